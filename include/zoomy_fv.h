/*
 * zoomy_fv.h — C ABI of libzoomyfv.so, the sm_100a implementation of
 * zoomy-amrex's per-level finite-volume right-hand side and SSP-RK2 time step.
 *
 * The reference runs this path as AMReX C++ (Source/ZoomyAmr.cpp +
 * Source/make_rhs.H) inside a compiled executable that zoomy_amrex/run_case.py
 * launches as a subprocess. This library replaces that executable's hot loop
 * with an in-process call: the caller (Python via ctypes, or any C caller)
 * owns every device buffer, the library owns only a small handle.
 *
 * Conventions
 *  - Every function returns an int status: 0 = OK, <0 = error
 *    (zfv_last_error() returns the message). No C++ exception crosses this ABI.
 *  - State arrays are structure-of-arrays, component-major, x fastest:
 *    Q[n][j][i], element (i,j,n) at Q + n*ny*nx + j*nx + i, i in [0,nx),
 *    j in [0,ny). This is Array4's (i,j,k,n) order with no ghost cells:
 *    ghost cells are never stored; they are rebuilt inside each kernel's
 *    tile load (mirror + Model::boundary_conditions).
 *  - Element type of Q: double for ZFV_PREC_FP64; float for ZFV_PREC_FP32,
 *    whose rows are [b, eta = h + b, hu, hv]. An FP32 state ping-pongs
 *    between Q rows 1..3 and a scratch buffer from step to step (the buffer
 *    in use is recorded on the device), so FP32 states are read only through
 *    zfv_state_export / zfv_batch_export, which convert to the reference
 *    layout [b, h, hu, hv] in FP64 and refresh aux's hinv row. aux is always
 *    double.
 *  - All device work is enqueued on the given stream (cudaStream_t passed as
 *    void*; NULL = legacy default stream). Functions never synchronize unless
 *    their comment says so.
 *  - A handle is used by one host thread at a time.
 */
#ifndef ZOOMY_FV_H
#define ZOOMY_FV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ZFV_MAX_PARAMS 16

/* Compiled model families (the Model::/Numerics:: pair a handle runs). */
enum {
    ZFV_MODEL_SWE1D = 1,   /* shallow water, 1 horizontal dim: Q=[b,h,hu],    aux 4 */
    ZFV_MODEL_SWE2D = 2,   /* shallow water, 2 horizontal dims: Q=[b,h,hu,hv], aux 7 */
    ZFV_MODEL_SME2D_L2 = 3,/* shallow-moment equations, level 2, 2 horizontal dims:
                              Q=[b,h,hu,hv,h*alpha1,h*alpha2,h*beta1,h*beta2], aux 1 (hinv);
                              Navier-slip bed friction (csrc/models/sme.H) */
    ZFV_MODEL_SME1D_L2 = 4 /* the same, 1 horizontal dim: Q=[b,h,hu,h*alpha1,h*alpha2], aux 1 */
};

/* Arithmetic form. */
enum {
    ZFV_PREC_FP64 = 0,     /* the plain form: FP64 everywhere, bit-compatible with the CPU path */
    ZFV_PREC_FP32 = 1      /* the chosen form (ZFV_MODEL_SWE2D, ZFV_MODEL_SME2D_L2): FP32 state
                              and flux arithmetic, Q = [b, eta = h + b, q_2, ...] as float,
                              compensation planes in scratch carry the low-order part of the
                              evolved rows (compensated update); FP64 for near-dry implicit
                              sources and the mass sum. 2-D SWE at order 2 without MOOD runs
                              on the column sweep (zfv_tile_variants); SME, order 1 and
                              MOOD run on the generic tile kernels (zfv_generic_tile_variants) */
};

/* Status flags (bitwise OR) reported by zfv_get_status(). */
enum {
    ZFV_FLAG_NONFINITE_DT   = 1,   /* the CFL reduction produced a non-finite dt            */
    ZFV_FLAG_MOOD_REDO      = 2,   /* a step was redone at order 1 (positivity = mood)      */
    ZFV_FLAG_DONE           = 4,   /* time >= time_end or step >= max_step: kernels idle   */
    ZFV_FLAG_DEVICE_WAIT    = 8    /* a bounded device-side wait (a TMA copy's barrier) ran
                                      out: the run was stopped and its last step is invalid */
};

/*
 * Solver configuration. Field meanings follow the reference's inputs deck
 * (ZoomyAmr.cpp:27-83 reads it; build.py:55-120 writes it) and its
 * generated MarchConstants.H (zoomy_amrex/_constants.py:59-88).
 */
typedef struct zfv_config {
    int model;              /* ZFV_MODEL_*                                          */
    int precision;          /* ZFV_PREC_*                                           */
    int nx, ny;             /* amr.n_cell (ny = 1 for 1-D models)                   */
    double prob_lo[2];      /* geometry.prob_lo                                     */
    double prob_hi[2];      /* geometry.prob_hi                                     */
    int spatial_order;      /* solver.spatial_order: 1 (PCM, 1 stage) or 2 (MUSCL/minmod, SSP-RK2) */
    int well_balanced;      /* solver.well_balanced: Audusse hydrostatic reconstruction */
    int implicit_source;    /* solver.implicit_source: point-implicit source after each stage */
    int clamp_positivity;   /* solver.clamp_positivity: h<0 -> 0 in UpdateState    */
    int positivity_mood;    /* solver.positivity == "mood": whole-step order-1 redo */
    int implicit_global;    /* solver.implicit_global: with implicit_source, the source
                               is solved for the whole field by Jacobian-free
                               Newton-Krylov (imex_solver.H) instead of per cell */
    double cfl;             /* solver.cfl (pure safety factor)                      */
    double dtmin, dtmax;    /* solver.dtmin / solver.dtmax                          */
    double time_end;        /* solver.time_end                                      */
    int max_step;           /* solver.max_step (<0: no cap)                         */
    int cfl_dimension;      /* ZoomyConstants::c_cfl_dimension (= d)                */
    int cfl_degree_factor;  /* ZoomyConstants::c_cfl_degree_factor (= 2k+1)         */
    int bc_tag[4];          /* bc.x_lo, bc.x_hi, bc.y_lo, bc.y_hi resolved to the
                               index in Model::get_boundary_tags()                  */
    int n_params;           /* Model::n_parameters                                  */
    double params[ZFV_MAX_PARAMS]; /* p_mat: Model::default_parameters() + params.* */
} zfv_config;

/* Device-side run status (read back by zfv_get_status; one 64-byte record). */
typedef struct zfv_status {
    double time;            /* simulated time reached                               */
    double dt;              /* dt of the NEXT step (already clamped to time_end)    */
    double mass;            /* sum(h) * dx * dy after the last completed step       */
    double max_inv;         /* max over cells, dirs of |lambda|/dx of the last reduction */
    int64_t step;           /* completed steps                                      */
    uint32_t flags;         /* ZFV_FLAG_*                                           */
    uint32_t mood_redos;    /* number of steps redone at order 1                    */
    uint32_t pad[4];
} zfv_status;

typedef struct zfv_handle zfv_handle;

/* Last error message of the calling thread ("" if none). */
const char* zfv_last_error(void);

/* Library build identification, e.g. "zoomyfv sm_100a fp64". */
const char* zfv_version(void);

/* sizeof(zfv_config) and sizeof(zfv_status) as compiled, for binding checks. */
size_t zfv_sizeof_config(void);
size_t zfv_sizeof_status(void);

/*
 * Create a solver handle for one level.
 * Replaces the ZoomyAmr constructor's deck parsing and parameter setup
 * (Source/ZoomyAmr.cpp:27-107). Validates the configuration; no device work.
 */
int zfv_create(const zfv_config* cfg, zfv_handle** out);
int zfv_destroy(zfv_handle* h);

/* Model shape: number of state rows, aux rows, parameters and space dims. */
int zfv_model_info(int model, int* n_q, int* n_aux, int* n_params, int* dimension);

/*
 * Bytes of caller-provided device scratch a handle needs (stage buffer,
 * reduction partials and the device-side status record). The scratch must
 * stay valid and unmodified between calls that share a run.
 */
size_t zfv_scratch_bytes(const zfv_handle* h);

/*
 * Initialise the device status record in scratch (time = 0, step = 0, flags
 * cleared) and compute the first dt from (Q, aux) exactly as
 * ZoomyAmr::ComputeDt does (Source/ZoomyAmr.cpp:448-515), reading the aux
 * as stored (the reference's first ComputeDt sees the aux that
 * init_solution wrote, before any UpdateState).
 */
int zfv_begin(zfv_handle* h, const void* Q, const void* aux, void* scratch, void* stream);

/*
 * ZoomyAmr::UpdateState (Source/ZoomyAmr.cpp:293-334) on every cell:
 * Model::update_variables, optional h>=0 clamp, Model::update_aux_variables.
 * Q and aux are updated in place.
 */
int zfv_update_state(zfv_handle* h, void* Q, void* aux, double time, void* stream);
/*
 * init_solution (Source/init_solution.cpp:78-116) on the device into a
 * (n_comp, ny, nx) float64 field of the handle's grid: zeros, and for
 * n_comp >= 2 the flat-bed dam break b = 0, h = 2 (x < x mid-point) | 1.
 * InitData applies it to Q and Qaux (ZoomyAmr.cpp:174-175); a caller uses
 * it to create aux0 on the device instead of copying it from the host.
 */
int zfv_init_solution(const zfv_handle* h, double* field, int n_comp, void* stream);
/* Work of the global implicit source (implicit_global; SolveImplicitSourceGlobal,
 * imex_solver.H:102-160) since the last zfv_begin: field solves (one per
 * stage), Newton iterations that ran a linear solve, and GMRES iterations.
 * Host counters; any pointer may be NULL. Zero for the point-implicit form. */
int zfv_implicit_global_stats(const zfv_handle* h, long long* solves, long long* newton, long long* gmres);

/*
 * ZoomyAmr::ComputeDt (Source/ZoomyAmr.cpp:448-515) on (Q, aux) as stored.
 * Writes the un-clamped-to-time_end dt and max_inv into the status record.
 */
int zfv_compute_dt(zfv_handle* h, const void* Q, const void* aux, void* scratch, void* stream);

/*
 * Up to n_steps iterations of ZoomyAmr::Evolve's loop body
 * (Source/ZoomyAmr.cpp:782-810) for a single level: TimeStep's dt clamp to
 * time_end (733-749), Advance (538-731: SSP-RK2 stages, implicit source,
 * Heun combine, MOOD redo, final UpdateState), time/step bookkeeping and the
 * mass sum (517-536). dt, time and the stop test live on the device, so the
 * call enqueues work without synchronizing; steps past the stop condition
 * are no-ops. Q is advanced in place; aux is written at the end of the call
 * (aux = Model::update_aux_variables of the final state).
 */
int zfv_evolve(zfv_handle* h, void* Q, void* aux, void* scratch, int n_steps, void* stream);

/*
 * One explicit right-hand side as compute_cell_rhs / assemble_cell_rhs
 * compute it (Source/make_rhs.H:234-290, 346-399) for the given stage
 * state: UpdateState + ghost fill + RHS. Writes rhs[n][j][i]. Validation
 * entry: the stepping kernels fuse this work and never store the RHS.
 */
int zfv_rhs(zfv_handle* h, const void* Q, const void* aux, void* rhs, double time, void* stream);

/*
 * Ghost fill as FillPatch + FillPhysicalBC_mf leave it
 * (Source/ZoomyAmr.cpp:258-277, 342-443), after UpdateState: writes the
 * grown arrays Qg[n][ny+2g][nx+2g], auxg[n][ny+2g][nx+2g] with g = ng
 * (ng = 1 at order 1, 2 at order 2; in 1-D models only x ghosts are
 * filled, as in the reference). Validation entry for the tile loaders.
 */
int zfv_fill_ghosts(zfv_handle* h, const void* Q, const void* aux, void* Qg, void* auxg,
                    double time, void* stream);

/*
 * Convert between the reference layout (Q64: [b, h, hu, (hv)] float64) and a
 * handle's state Q. FP64 handles copy. FP32 handles split eta = h + b, hu, hv
 * into a float part in Q and a float remainder in scratch (the compensation
 * planes), so the FP64 input is carried to ~48 bits; export recombines them
 * and writes aux's last row (hinv) for the exported state, the refresh that
 * FP64 handles do at the end of every zfv_evolve (FP32 stages evaluate hinv
 * from the face states and never read it).
 * zfv_state_import must precede zfv_begin for FP32 handles.
 */
int zfv_state_import(zfv_handle* h, const double* Q64, void* Q, void* scratch, void* stream);
int zfv_state_export(zfv_handle* h, const void* Q, const void* scratch, double* Q64, void* stream);

/* Sum(h) * dx * dy into the status record's mass field (ZoomyAmr.cpp:517-536). */
int zfv_total_mass(zfv_handle* h, const void* Q, void* scratch, void* stream);

/*
 * Copy the device status record to *out. Synchronizes the stream.
 */
int zfv_get_status(zfv_handle* h, const void* scratch, zfv_status* out, void* stream);

/*
 * Per-step log written by zfv_evolve: for step s (1-based) entry s-1 holds
 * {dt, time, mass} — the fields of the reference's "Step n dt: time: mass:"
 * line (ZoomyAmr.cpp:804-809). The log keeps the last zfv_log_capacity()
 * steps (ring buffer). Synchronizes the stream.
 */
int zfv_log_capacity(const zfv_handle* h);
int zfv_read_log(zfv_handle* h, const void* scratch, double* out3, int max_entries,
                 int64_t* first_step, int* n_out, void* stream);

/*
 * Batches: many independent FP32 SWE2D levels (the boxes of an AMR level or
 * the members of an ensemble; each with its own grid, bathymetry, parameters,
 * boundary conditions, dt, time and stop test) advanced together, one launch
 * per RK stage for all of them. Replaces the per-box launches of the
 * reference's MFIter loops (ZoomyAmr.cpp:579-637, one ParallelFor per box per
 * kernel) for the case where the boxes are independent runs.
 * All instances must be ZFV_MODEL_SWE2D / ZFV_PREC_FP32 / spatial_order 2 and
 * share well_balanced and implicit_source.
 *
 * zfv_batch_bind registers each instance's Q (4 float planes [b, eta, hu, hv])
 * and aux (double planes) and the caller's scratch, and uploads the work list
 * (synchronizes the stream). The bound buffers are used by every later call;
 * zfv_batch_begin / zfv_batch_evolve enqueue work without synchronizing and can
 * be captured in a CUDA graph.
 */
typedef struct zfv_batch zfv_batch;
int zfv_batch_create(const zfv_config* cfgs, int n_inst, zfv_batch** out);
int zfv_batch_destroy(zfv_batch* b);
size_t zfv_batch_scratch_bytes(const zfv_batch* b);
int zfv_batch_bind(zfv_batch* b, void* const* Q, double* const* aux, void* scratch, void* stream);
/* FP64 reference layout [b, h, hu, hv] <-> the bound FP32 states (synchronizes).
 * Export also refreshes each instance's aux hinv row; a NULL Q64[k] refreshes
 * only that. */
int zfv_batch_import(zfv_batch* b, const double* const* Q64, void* stream);
int zfv_batch_export(zfv_batch* b, double* const* Q64, void* stream);
/* zfv_begin for every instance (time 0, first dt from the stored aux). */
int zfv_batch_begin(zfv_batch* b, void* stream);
/* n_steps SSP-RK2 steps of every instance (an instance past its stop test idles):
 * exactly two kernel launches per step, whatever the step count before, so a
 * graph captured from a one-step call can be replayed any number of times. */
int zfv_batch_evolve(zfv_batch* b, int n_steps, void* stream);
/* Status records of all instances into out[n_inst] (synchronizes). */
int zfv_batch_status(zfv_batch* b, zfv_status* out, void* stream);
/* Work units of the current strip shape. */
int zfv_batch_units(const zfv_batch* b);
/*
 * Strip shapes compiled into the library: (warps per block, cells per thread
 * in y, columns per lane: 1 = scalar sweep, 2 = packed-FP32 column pairs,
 * flags: bit 0 = stage 2 stages its update inputs in shared memory with
 * asynchronous copies at the top of each row, bit 1 = the stage-2 kernel is
 * capped at 128 registers).
 * zfv_tile_variants writes up to max_n of them and returns how many exist;
 * zfv_batch_set_variant selects one for a batch, zfv_set_variant for a
 * single FP32 level (the autotuner in zoomy_amrex_b200/autotune.py measures
 * them and caches the fastest per n_dof_q). Until one is selected, batches and
 * FP32 levels use variant 9 (4 warps x 8 rows, column pairs, flags 3).
 * The FP64 form has one tile shape: zfv_set_variant fails with -2 there and
 * zfv_get_variant returns -1.
 */
int zfv_tile_variants(int* nw, int* cpt, int* cols, int* flags, int max_n);
/*
 * Tile variants of the generic FP32 kernels (the FP32 form of the
 * shallow-moment model, ZFV_MODEL_SME2D_L2, and of 2-D SWE at spatial order 1
 * or with positivity_mood): tile width and height in cells
 * and the staging (0 = plain coalesced loads, 1 = TMA boxes completing on an
 * mbarrier; needs nx % 4 == 0 and a 16-byte aligned state). Writes up to
 * max_n of them and returns how many exist; zfv_set_variant selects one for
 * such a level (default 0). Every variant gives the same bits.
 */
int zfv_generic_tile_variants(int* tx, int* ty, int* tma, int max_n);
int zfv_set_variant(zfv_handle* h, int variant, void* stream);
int zfv_get_variant(const zfv_handle* h);

/*
 * Batches whose instances are grouped: instances with the same group id
 * (0 .. n_inst-1) share one run record — one dt, one CFL / mass reduction over
 * all their cells, one step counter — as the boxes of one AMR level do
 * (ZoomyAmr::ComputeDt reduces over the level's boxes, ZoomyAmr.cpp:448-515).
 * Grouped instances must share the CFL constants.
 */
int zfv_batch_create_grouped(const zfv_config* cfgs, int n_inst, const int* groups, zfv_batch** out);
/* Per instance, a ghost frame ((nx+4) x (ny+4) x 4 floats, [b, eta, hu, hv]
 * planes) whose ring the kernels read instead of mirroring the box's own cells
 * (NULL entries / NULL array: physical mirror). Re-uploads the descriptors. */
int zfv_batch_set_frames(zfv_batch* b, const float* const* frames, void* stream);
/* Set each instance's next dt from dts (device, one per instance; enqueued,
 * no synchronization). AMR levels step with dt_0 / 2^l. */
int zfv_batch_set_dt(zfv_batch* b, const double* dts, void* stream);
/* ComputeDt of every run record's current state (ZoomyAmr::ComputeDt,
 * ZoomyAmr.cpp:448-515, over the record's instances, hinv from the state),
 * written as the record's next dt (enqueued, no synchronization): the
 * reference's per-level step law, ZoomyAmr.cpp:739. */
int zfv_batch_compute_dt(zfv_batch* b, void* stream);
/* One stage (1 or 2) of one SSP-RK2 step of every instance, so that ghost
 * frames can be refilled between the stages (Advance's per-stage FillPatch,
 * ZoomyAmr.cpp:561-572). */
int zfv_batch_stage(zfv_batch* b, int stage, void* stream);
/* Device address of the bound instance descriptors (for the AMR kernels). */
const void* zfv_batch_descriptors(const zfv_batch* b);

/*
 * Block-structured AMR over grouped batches (ZoomyAmr.cpp:161-288, 733-762:
 * FillPatch / FillPatchTwoLevels, average_down, ErrorEst, RemakeLevel). A
 * level is a batch of B x B boxes on a block grid; map[by * nbx + bx] is the
 * instance holding block (bx, by), -1 if absent; pos lists (bx, by) of the
 * boxes to work on (device int pairs); frames is a device array of the boxes'
 * ghost-frame pointers in the same order. Refinement ratio 2.
 */
typedef struct zfv_amr_level {
    const void* insts;   /* zfv_batch_descriptors() of the level's batch */
    const int* map;      /* device, nby * nbx: (instance << 10) | (block row offset << 5) |
                            block column offset inside the patch, -1 absent */
    int nbx, nby;        /* block grid */
    int B;               /* cells per block side (even) */
    int nx, ny;          /* the level's grid in cells */
    int wall;            /* bit s set: side s (x_lo, x_hi, y_lo, y_hi) is a reflective wall */
    int pad;
} zfv_amr_level;
/*
 * Patches: a level's blocks grouped into rectangles of nbx x nby blocks
 * (each side 1 .. 32), one batch instance of (nbx * B) x (nby * B) cells
 * each. `patches` (device) holds 4 ints per patch: first block x, first
 * block row y, nbx, nby; max_blocks bounds nbx * nby over the list (it sizes
 * the launch). Instance k of the level's batch is patch k.
 */
/* Ghost frames ((nby*B + 4) x (nbx*B + 4) x 4 floats per patch) before stage
 * `stage` (1: the stage input; 2: neighbours' stage-2 input): same-level
 * patches, else conservative linear interpolation of `coarse` (NULL on level
 * 0), physical boundaries by mirroring. */
int zfv_amr_fill(const zfv_amr_level* fine, const zfv_amr_level* coarse, const int* patches, float* const* frames,
                 int n_patches, int max_blocks, int stage, void* stream);
/* Replace the coarse cells under the listed fine patches by 2 x 2 averages. */
int zfv_amr_average_down(const zfv_amr_level* fine, const zfv_amr_level* coarse, const int* patches, int n_patches,
                         int max_blocks, void* stream);
/* flags[by * nbx + bx] = 1 (others untouched) for the blocks of the listed
 * patches with a tagged cell. criterion 0: |grad eta| > threshold;
 * criterion 1: the reference's ErrorEst (ZoomyAmr.cpp:224-252): b < b_max
 * and (undivided |(h(i+1)-h(i-1), h(j+1)-h(j-1))| > threshold or h > 1e-2). */
int zfv_amr_tag(const zfv_amr_level* level, const int* patches, int n_patches, int max_blocks, double dx, double dy,
                double threshold, int criterion, double b_max, int* flags, void* stream);
/* dt_0 = the largest step whose dt_0 / 2^l every level's CFL law allows (from
 * each level's last CFL maximum), clamped to [dtmin, dtmax] and then to land
 * on time_end (0 once *time >= time_end, ZoomyAmr.cpp:746-749); writes
 * dt_0 / 2^l into level l's per-instance dt array (device) and adds dt_0 to
 * *time (device; NULL: no time, no time_end clamp). level_descs:
 * zfv_batch_descriptors() of each level. Enqueued; no synchronization (a
 * coarse step can be captured in a graph). */
int zfv_amr_set_dt(const void* const* level_descs, double* const* dts, const int* n_inst, int n_levels,
                   double cfl, double cfl_divisor, double dtmin, double dtmax, double time_end, double* time,
                   void* stream);
/* The base level's step under the reference's per-level law
 * (ZoomyAmr.cpp:739-749): the dt in its run record (zfv_batch_compute_dt)
 * clamped to land on time_end (0 once *time >= time_end), added to *time
 * (device). level_desc: zfv_batch_descriptors() of the base level. */
int zfv_amr_level_dt(const void* level_desc, double time_end, double* time, void* stream);
/* Fill freshly created patches from the old patches of the level (where
 * present) or from the coarser level. */
int zfv_amr_regrid_fill(const zfv_amr_level* level, const zfv_amr_level* old_level, const zfv_amr_level* coarse,
                        const int* patches, int n_patches, int max_blocks, void* stream);
int zfv_batch_set_variant(zfv_batch* b, int variant, void* stream);

/*
 * Run record save / restore: the device-side time, dt, step and flags of a
 * handle's run (zfv_run_state_bytes() bytes, device to device, async). With
 * the state Q this is everything a run needs to continue: the checkpoint of
 * the adjoint's checkpoint-and-recompute.
 */
size_t zfv_run_state_bytes(void);
int zfv_save_run_state(zfv_handle* h, const void* scratch, void* dst, void* stream);
int zfv_load_run_state(zfv_handle* h, void* scratch, const void* src, void* stream);

/*
 * Adjoint of the FP64 ZFV_MODEL_SWE2D step (spatial_order 2, no clamp, no
 * MOOD). No counterpart in the reference, which has no derivatives; it
 * differentiates exactly the map zfv_evolve applies, dt included:
 *   Y1 = stage(Q^n), Y2 = stage(Y1), Q^{n+1} = (Q^n + Y2)/2, stage = explicit
 *   flux update then point-implicit source (ZoomyAmr.cpp:538-731,
 *   make_rhs.H:31-509), dt_n = cfl/(d (2k+1) max_inv(Q^n)) (ZoomyAmr.cpp:448-515).
 * zfv_adj_record runs n_steps steps exactly as zfv_evolve does (same kernels,
 * same results) and writes what the reverse needs onto `tape`
 * (zfv_adj_tape_bytes(h, n_steps) bytes, caller-allocated, device). The run
 * must not reach its stop test inside the recorded steps.
 * zfv_adj_step reverses recorded step k: on entry lam (n_q planes, like Q)
 * holds dL/dQ^{k+1}, on exit dL/dQ^k; grad[0] += dL/dn_m (Manning
 * coefficient), grad[1] += dL/ddt_k (diagnostic). aux0: the aux whose hinv row
 * the run's first dt was computed from (pass it for the run's first step, NULL
 * otherwise: later dts use the state's own hinv). work: zfv_adj_work_bytes(h)
 * bytes, zero-filled before first use. Neither call synchronizes.
 */
size_t zfv_adj_tape_bytes(const zfv_handle* h, int n_steps);
size_t zfv_adj_work_bytes(const zfv_handle* h);
int zfv_adj_record(zfv_handle* h, void* Q, void* aux, void* scratch, void* tape, int n_steps, void* stream);
int zfv_adj_step(zfv_handle* h, const void* tape, int k, void* lam, double* grad, const void* aux0,
                 void* work, void* stream);
/* zfv_adj_step for recorded steps n_steps - 1 down to 0 of `tape`, in one
 * call (aux0, or NULL, is passed for step 0 only). */
int zfv_adj_steps(zfv_handle* h, const void* tape, int n_steps, void* lam, double* grad, const void* aux0,
                  void* work, void* stream);
/* Tile shapes compiled for the adjoint's face-reverse kernel (a process-wide
 * tuning choice; every shape gives the same gradient up to rounding). */
int zfv_adj_variants(void);
int zfv_adj_set_variant(int variant);

/*
 * zfv_evolve without caller-provided scratch. No counterpart in the reference
 * (its AMReX driver allocates MultiFabs itself); it exists for callers that
 * cannot call cudaMalloc at all — code inside another framework's memory
 * pool, under a caching allocator that owns all device memory, or in a
 * plugin that must not allocate at call time.
 *
 * Scratch is a 64 MiB array compiled into the library (every GPU that loads
 * the library holds it until exit); levels whose zfv_scratch_bytes() exceeds
 * it (about 2 million cells for ZFV_MODEL_SWE2D) are rejected with an error.
 * Only FP64 handles are accepted: the FP32 form keeps a part of its state
 * (the compensation remainder) in scratch, where only zfv_state_import and
 * zfv_state_export reach it, so it needs caller-provided scratch.
 * restart != 0 starts a run like zfv_begin (clearing the device run record);
 * restart == 0 continues the run that the previous call on this device left
 * in the array, and is refused with an error unless the last restart on this
 * device was made with the same handle. Every call on a device shares the one
 * array: calls that overlap on the GPU (other streams, other handles) race,
 * and interleaving runs of different handles needs restart != 0. The first
 * call on each device looks up the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * If status_out is not NULL the run status is copied into it and the stream
 * is synchronized before the call returns; with status_out == NULL the call
 * only enqueues the work and returns before the stream has finished it.
 * Allocates no device memory.
 */
int zfv_evolve_static(zfv_handle* h, void* Q, void* aux, int n_steps, int restart,
                      zfv_status* status_out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* ZOOMY_FV_H */
