// The fused finite-volume stage kernel and the per-cell helper kernels.
//
// One CTA owns a TX x TY tile of cells. Per stage it
//   1. loads the tile plus its ng-cell halo from the state planes and applies
//      UpdateState on load (ZoomyAmr.cpp:293-334),
//   2. rebuilds the out-of-domain ghost cells in shared memory from their
//      mirrored interior cells and Model::boundary_conditions
//      (FillPhysicalBC_mf, ZoomyAmr.cpp:342-443) — ghost cells are never stored,
//   3. evaluates every face of the tile once (eval_face, make_rhs.H:31-131)
//      into shared memory,
//   4. assembles each cell's RHS (make_rhs.H:346-399), applies the stage
//      update Q += dt*RHS (ZoomyAmr.cpp:629-637) and the point-implicit source
//      (make_rhs.H:429-509),
//   5. depending on the stage: stores the stage state (RK stage 1); or applies
//      the Heun combine (ZoomyAmr.cpp:665-675), the final UpdateState
//      (ZoomyAmr.cpp:730) and contributes the CFL max and the mass sum to a
//      grid reduction whose last block advances time/step and computes the
//      next dt on the device (ComputeDt + TimeStep, ZoomyAmr.cpp:448-515,
//      733-751, 789-809).
// The step therefore touches HBM once per stage for the state (plus halo
// re-reads served mostly from L2) and never for RHS, face data or ghosts.
#pragma once
#include "fv_device.cuh"

namespace zfv {

enum StageMode : int {
    MODE_RHS = 0,   // write the RHS only (validation entry zfv_rhs)
    MODE_S1 = 1,    // SSP-RK2 stage 1: write the stage state
    MODE_S2 = 2,    // SSP-RK2 stage 2: Heun + final UpdateState + reduction
    MODE_ONE = 3,   // order 1: single stage + final UpdateState + reduction
    // positivity = "mood" (ZoomyAmr.cpp:685-720):
    MODE_S2M = 4,   // stage 2 writing the Heun candidate to a buffer and flagging troubled cells
    MODE_R1 = 5,    // order-1 redo, stage 1 (runs only when the step is troubled)
    MODE_R2 = 6,    // order-1 redo, stage 2 + final UpdateState + reduction (troubled only)
    // solver.implicit_global (imex_solver.H): the stage state after the flux
    // update, before any source; the global Newton-Krylov solve follows
    MODE_X = 7
};

// Face records in shared memory hold make_rhs.H:310-315's components
// (flux, D+, D-, h*_L, h*_R) for the rows the step evolves: with a static bed
// (and outside the RHS validation mode) the bed row is skipped.
template <class Model, int ORDER, int TX, int TY, bool SKIPB>
struct TileShape {
    static constexpr int dim = Model::dimension;
    static constexpr int nq = Model::n_dof_q;
    static constexpr int n0 = SKIPB ? 1 : 0;               // first evolved row
    static constexpr int NQE = nq - n0;
    static constexpr int G = (ORDER == 2) ? 2 : 1;        // ZoomyAmr.H:152 nghost()
    static constexpr int GY = (dim == 2) ? G : 0;
    static constexpr int RW = TX + 2 * G;
    static constexpr int RH = TY + 2 * GY;
    static constexpr int NFC = 3 * NQE + 2;                // make_rhs.H:315 n_face_comp
    static constexpr int NT = TX * TY;
    static constexpr int min_blocks = (dim == 2) ? 3 : 2;
    static constexpr size_t q_elems = size_t(nq) * RH * RW;
    static constexpr size_t fx_elems = size_t(TY) * (TX + 1) * NFC;
    static constexpr size_t fy_elems = (dim == 2) ? size_t(TY + 1) * TX * NFC : 0;
    // the x faces and then the y faces use one buffer; between the two
    // passes each cell keeps its x part of the balance (NQE values and the
    // WB x pressure term) in xp
    static constexpr size_t f_elems = fx_elems > fy_elems ? fx_elems : fy_elems;
    static constexpr size_t xp_elems = (dim == 2) ? size_t(NQE + 1) * NT : 0;
    static constexpr size_t smem_bytes = (q_elems + f_elems + xp_elems) * sizeof(double);
};

// Deterministic block reduction: max of m (NaN-ignoring, as the reference's
// `if (inv > max_inv)` accumulation) and sum of s in a fixed order.
template <int NT>
__device__ __forceinline__ void block_reduce_max_sum(double& m, double& s, double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const double om = __shfl_down_sync(0xffffffffu, m, off);
        const double os = __shfl_down_sync(0xffffffffu, s, off);
        if (om > m) m = om;
        s = s + os;
    }
    constexpr int NW = (NT + 31) / 32;
    __syncthreads();
    if (lane == 0) { red[2 * warp] = m; red[2 * warp + 1] = s; }
    __syncthreads();
    if (threadIdx.x == 0) {
        m = red[0]; s = red[1];
        for (int w = 1; w < NW; ++w) {
            if (red[2 * w] > m) m = red[2 * w];
            s = s + red[2 * w + 1];
        }
    }
}

// Last-block-done grid reduction + device-side TimeStep/Evolve bookkeeping.
// Every block writes (max, sum) to partials[blk]; the last block to finish
// reduces them in block order and advances the run state.
template <int NT, class PL>
__device__ __forceinline__ bool finish_step_units(double m, double s, double* red, double* partials,
                                                  double* log3, int log_cap, DevState* st, PL const& L,
                                                  double dt_used, double time_used, bool mood_redo,
                                                  unsigned nblk, unsigned blk);

template <int NT, class PL>
__device__ __forceinline__ void finish_step(double m, double s, double* red, double* partials,
                                            double* log3, int log_cap, DevState* st, PL const& L,
                                            double dt_used, double time_used, bool mood_redo = false) {
    finish_step_units<NT>(m, s, red, partials, log3, log_cap, st, L, dt_used, time_used, mood_redo,
                          gridDim.x * gridDim.y, blockIdx.y * gridDim.x + blockIdx.x);
}

// The same over an explicit set of `nblk` work units (this block is unit
// `blk`): lets one launch carry several independent runs (a batch), each with
// its own run record and partials. Returns true in the block that finished
// the step (the last unit to arrive).
template <int NT, class PL>
__device__ __forceinline__ bool finish_step_units(double m, double s, double* red, double* partials,
                                                  double* log3, int log_cap, DevState* st, PL const& L,
                                                  double dt_used, double time_used, bool mood_redo,
                                                  unsigned nblk, unsigned blk) {
    block_reduce_max_sum<NT>(m, s, red);
    __shared__ unsigned s_last;
    if (threadIdx.x == 0) {
        partials[2 * blk] = m;
        partials[2 * blk + 1] = s;
        __threadfence();
        const unsigned prev = atomicAdd(&st->counter, 1u);
        s_last = (prev == nblk - 1) ? 1u : 0u;
    }
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
    double gm = 0.0, gs = 0.0;
    // unrolled so that many loads are in flight: this loop is the serial tail
    // of every step (same order of additions as a plain loop)
#pragma unroll 8
    for (unsigned b = threadIdx.x; b < nblk; b += NT) {
        const double pm = __ldcg(&partials[2 * b]);
        const double ps = __ldcg(&partials[2 * b + 1]);
        if (pm > gm) gm = pm;
        gs = gs + ps;
    }
    block_reduce_max_sum<NT>(gm, gs, red);
    if (threadIdx.x == 0) {
        const double t_new = time_used + dt_used;                 // Evolve: time += dt0
        const long long step = st->step + 1;
        const double mass = gs * (L.dx * L.dy);                   // ComputeTotalMass
        if (log_cap > 0) {
            double* e = log3 + 3 * ((step - 1) % log_cap);
            e[0] = dt_used; e[1] = t_new; e[2] = mass;
        }
        const double dt_next = dt_from_max(gm, t_new, L);         // next TimeStep's ComputeDt + clamp
        unsigned flags = st->flags;
        if (!isfinite(dt_next)) flags |= kFlagNonfiniteDt;
        if (run_done(t_new, step, L)) flags |= kFlagDone;
        if (mood_redo) {
            flags |= kFlagMoodRedo;
            st->mood_redos = st->mood_redos + 1u;
            st->troubled = 0u;
        }
        st->time = t_new;
        st->step = step;
        st->mass = mass;
        st->max_inv = gm;
        st->dt = dt_next;
        st->flags = flags;
        st->counter = 0u;
        __threadfence();
    }
    return true;
}

// Blocks per SM the register budget aims at: 4 for 2-D tiles, so that 32
// warps (shallow water: 256 threads at 64 registers) or 16 (the models whose
// point-implicit system is solved by blocks: 128 threads at 128 registers,
// the dense fallback out of line) hide the FP64 latency; their shared
// memory, with the one face buffer, fits 4 blocks too; 2 for 1-D rows and
// for dense n x n eliminations, which must stay in registers.
template <class Model>
constexpr int stage_min_blocks() {
    if constexpr (Model::dimension == 2 && (Model::n_dof_q <= 4 || implicit_blocks<Model>::value)) return 4;
    else return 2;
}

template <class Model, class Numerics, int ORDER, int MODE, bool WB, bool IMPL, int TX, int TY>
__global__ void __launch_bounds__(TX * TY, stage_min_blocks<Model>())
k_stage(const double* __restrict__ qin, const double* __restrict__ qbed,
        const double* __restrict__ qold, double* __restrict__ qout,
        LevelParams<double, Model::n_parameters> L, DevState* st,
        double* __restrict__ partials, double* __restrict__ log3, int log_cap, double time_arg,
        double* __restrict__ qstar)
{
    constexpr bool sbed = static_bed<Model>::value;
    using Sh = TileShape<Model, ORDER, TX, TY, sbed && MODE != MODE_RHS>;
    using T = ModelTypes<Model>;
    using R = double;
    constexpr int nq = Sh::nq, dim = Sh::dim, n0 = Sh::n0, NQE = Sh::NQE;
    constexpr int G = Sh::G, GY = Sh::GY, RW = Sh::RW, RH = Sh::RH, NFC = Sh::NFC, NT = Sh::NT;
    constexpr bool pure = aux_pure<Model>::value;
    static_assert(pure, "the fused stage kernel needs Model::zb_aux_pure");
    // make_rhs.H:166-229 (add_diffusive_flux, compiled in when
    // Model::has_diffusion) is not part of these kernels: refuse such a model
    // at compile time rather than drop its viscous term.
    static_assert(!Model::has_diffusion, "diffusive models (Model::has_diffusion) are not built here");

    extern __shared__ __align__(16) double smem[];
    double* sQ = smem;                                  // [nq][RH][RW]
    double* sF = sQ + Sh::q_elems;                      // x faces [TY][TX+1][NFC], then y faces [TY+1][TX][NFC]
    double* sXp = sF + Sh::f_elems;                     // 2-D: [NQE+1][NT] x parts of the cells' balances
    __shared__ double red[2 * ((NT + 31) / 32)];

    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int nx = L.nx, ny = L.ny;
    const long long plane = L.plane;

    // The MOOD redo stages run only for a troubled step.
    if constexpr (MODE == MODE_R1 || MODE == MODE_R2) {
        if (*(volatile unsigned*)&st->troubled == 0u) return;
    }
    // Idle once the run is done (time_end / max_step reached).
    const unsigned flags0 = (MODE == MODE_RHS) ? 0u : *(volatile unsigned*)&st->flags;
    if (flags0 & kFlagDone) {
        if constexpr (MODE == MODE_ONE) {   // ping-pong: keep the state in the output buffer
            for (int k = tid; k < TX * TY; k += NT) {
                const int i = x0 + k % TX, j = y0 + k / TX;
                if (i < nx && j < ny) {
                    const long long c = (long long)j * nx + i;
#pragma unroll
                    for (int n = (sbed ? 1 : 0); n < nq; ++n) qout[n * plane + c] = qin[n * plane + c];
                }
            }
        }
        return;
    }
    // Read once: the last block of this grid rewrites them after every other
    // block has passed its reduction counter (finish_step).
    const R dt = (MODE == MODE_RHS) ? R(0) : *(volatile double*)&st->dt;
    const R time = (MODE == MODE_RHS) ? time_arg : *(volatile double*)&st->time;

    typename T::VP p;
#pragma unroll
    for (int k = 0; k < Model::n_parameters; ++k) p(k, 0) = L.p[k];
    typename T::VA azero{};

    // 1. tile + halo load with UpdateState applied (valid cells only)
    for (int k = tid; k < RW * RH; k += NT) {
        const int lx = k % RW, ly = k / RW;
        const int gi = x0 - G + lx, gj = y0 - GY + ly;
        if (gi >= 0 && gi < nx && gj >= 0 && gj < ny) {
            const long long c = (long long)gj * nx + gi;
            typename T::VQ q;
            q(0, 0) = sbed ? qbed[c] : qin[c];
#pragma unroll
            for (int n = 1; n < nq; ++n) q(n, 0) = qin[n * plane + c];
            typename T::VA a = azero;
            update_state_cell<Model, R>(q, a, p, L, time, cell_centre<Model, R>(L, gi, gj));
#pragma unroll
            for (int n = 0; n < nq; ++n) sQ[(n * RH + ly) * RW + lx] = q(n, 0);
        }
    }
    __syncthreads();

    // 2. ghost cells from mirrored interior cells + Model::boundary_conditions
    const bool edge_tile = (x0 - G < 0) || (x0 + TX + G > nx) ||
                           (dim == 2 && ((y0 - GY < 0) || (y0 + TY + GY > ny)));
    if (edge_tile) {
        for (int k = tid; k < RW * RH; k += NT) {
            const int lx = k % RW, ly = k / RW;
            const int gi = x0 - G + lx, gj = y0 - GY + ly;
            const bool in_x = gi >= 0 && gi < nx, in_y = gj >= 0 && gj < ny;
            if (in_x && in_y) continue;
            // only the ng-deep ghost frame exists in the reference's grown box
            if (gi < -G || gi > nx - 1 + G || gj < -GY || gj > ny - 1 + GY) continue;
            const GhostMap<dim> gm = ghost_map<dim>(gi, gj, nx, ny);
            if (gm.bc_side < 0) continue;
            const int mx = gm.ii - x0 + G, my = gm.jj - y0 + GY;
            if (mx < 0 || mx >= RW || my < 0 || my >= RH) continue;   // excluded by zfv_create
            typename T::VQ qi;
#pragma unroll
            for (int n = 0; n < nq; ++n) qi(n, 0) = sQ[(n * RH + my) * RW + mx];
            const auto Xi = cell_centre<Model, R>(L, gm.ii, gm.jj);
            const typename T::VA ai = Model::update_aux_variables(qi, azero, p, time, Xi);
            typename T::VN nh{};
            nh(gm.normal_dir, 0) = R(gm.normal_sign);
            const auto X = cell_centre<Model, R>(L, gi, gj);
            const typename T::VQ qg =
                Model::boundary_conditions(L.bc_tag[gm.bc_side], qi, ai, nh, X, time, L.dx);
#pragma unroll
            for (int n = 0; n < nq; ++n) sQ[(n * RH + ly) * RW + lx] = qg(n, 0);
        }
        __syncthreads();
    }

    const int tx = tid % TX, ty = tid / TX;
    const int i = x0 + tx, j = y0 + ty;
    const int iend = min(x0 + TX, nx);        // last face index needed in x
    const int jend = min(y0 + TY, ny);

    auto loadq = [&](int lx, int ly) {
        typename T::VQ q;
#pragma unroll
        for (int n = 0; n < nq; ++n) q(n, 0) = sQ[(n * RH + ly) * RW + lx];
        return q;
    };
    auto store_face = [&](double* F, typename T::VQ const& fl, typename T::V2Q const& fc, R hl, R hr) {
#pragma unroll
        for (int n = n0; n < nq; ++n) {
            F[n - n0] = fl(n, 0);                 // flux
            F[NQE + n - n0] = fc(n, 0);           // D+
            F[2 * NQE + n - n0] = fc(nq + n, 0);  // D-
        }
        F[3 * NQE] = hl;
        F[3 * NQE + 1] = hr;
    };
    // x-face f sits between cells f-1 and f of row jj (local row ly)
    auto x_face = [&](int f, int jj, int ly, double* F) {
        const int lx = f - x0 + G;
        typename T::VQ cLL, cRR;
        if constexpr (ORDER == 2) { cLL = loadq(lx - 2, ly); cRR = loadq(lx + 1, ly); }
        const typename T::VQ cL = loadq(lx - 1, ly), cR = loadq(lx, ly);
        typename T::VQ fl; typename T::V2Q fc; R hl, hr;
        eval_face<Model, Numerics, ORDER, 0, WB, R>(cLL, cL, cR, cRR, azero, azero, p, L, time,
                                                    f - 1, jj, f, jj, fl, fc, hl, hr);
        store_face(F, fl, fc, hl, hr);
    };
    auto y_face = [&](int ii, int f, int lx, double* F) {
        const int ly = f - y0 + GY;
        typename T::VQ cLL, cRR;
        if constexpr (ORDER == 2) { cLL = loadq(lx, ly - 2); cRR = loadq(lx, ly + 1); }
        const typename T::VQ cL = loadq(lx, ly - 1), cR = loadq(lx, ly);
        typename T::VQ fl; typename T::V2Q fc; R hl, hr;
        eval_face<Model, Numerics, ORDER, 1, WB, R>(cLL, cL, cR, cRR, azero, azero, p, L, time,
                                                    ii, f - 1, ii, f, fl, fc, hl, hr);
        store_face(F, fl, fc, hl, hr);
    };

    // 3. faces, each once: the x faces, each cell's x part of its balance,
    // then the y faces in the same buffer. The x part is Fx / dx and the WB
    // x pressure term, each formed exactly as the one-pass assembly forms
    // it, so the balance below is the same IEEE arithmetic in the same order.
    const bool valid = (i < nx) && (j < ny);
    if (j < jend) {
        const int ly = ty + GY;
        if (i <= iend) x_face(i, j, ly, sF + (ty * (TX + 1) + tx) * NFC);
        if (tx == TX - 1 && x0 + TX <= iend)
            x_face(x0 + TX, j, ly, sF + (ty * (TX + 1) + TX) * NFC);
    }
    __syncthreads();
    R xdiv[NQE], xwb = R(0.0);
    if (valid) {
        const double* FxL = sF + (ty * (TX + 1) + tx) * NFC;
        const double* FxR = FxL + NFC;
#pragma unroll
        for (int k = 0; k < NQE; ++k) {
            const R Fx = -(FxR[k] - FxL[k]) - FxR[2 * NQE + k] - FxL[NQE + k];
            xdiv[k] = Fx / L.dx;
        }
        if constexpr (WB)
            xwb = R(0.5) * p(0, 0) * (FxR[3 * NQE] * FxR[3 * NQE] - FxL[3 * NQE + 1] * FxL[3 * NQE + 1]) / L.dx;
    }
    if constexpr (dim == 2) {
        if (valid) {
#pragma unroll
            for (int k = 0; k < NQE; ++k) sXp[k * NT + tid] = xdiv[k];
            sXp[NQE * NT + tid] = xwb;
        }
        __syncthreads();   // every x face read: the buffer takes the y faces
        if (i < iend) {
            const int lx = tx + G;
            if (j <= jend) y_face(i, j, lx, sF + (ty * TX + tx) * NFC);
            if (ty == TY - 1 && y0 + TY <= jend)
                y_face(i, y0 + TY, lx, sF + (TY * TX + tx) * NFC);
        }
        __syncthreads();
        if (valid) {
#pragma unroll
            for (int k = 0; k < NQE; ++k) xdiv[k] = sXp[k * NT + tid];
            xwb = sXp[NQE * NT + tid];
        }
    }

    // 4. assemble (make_rhs.H:346-399), update, implicit source, epilogue
    double m_loc = 0.0, s_loc = 0.0;
    if (valid) {
        const double* FyL = (dim == 2) ? sF + (ty * TX + tx) * NFC : nullptr;
        const double* FyR = (dim == 2) ? FyL + TX * NFC : nullptr;
        const typename T::VQ qc = loadq(tx + G, ty + GY);
        const auto X = cell_centre<Model, R>(L, i, j);
        const typename T::VA ac = Model::update_aux_variables(qc, azero, p, time, X);
        typename T::VQ S;
#pragma unroll
        for (int n = 0; n < nq; ++n) S(n, 0) = R(0.0);
        if constexpr (!IMPL) S = Model::source(qc, ac, p, time, X);
        typename T::VQ rhs;
        if constexpr (n0 == 1) rhs(0, 0) = R(0.0);   // static bed: never used
#pragma unroll
        for (int n = n0; n < nq; ++n) {
            const int k = n - n0;
            R Fy = R(0.0);
            if constexpr (dim == 2) Fy = -(FyR[k] - FyL[k]) - FyR[2 * NQE + k] - FyL[NQE + k];
            rhs(n, 0) = xdiv[k] + Fy / L.dy;
            if constexpr (!IMPL) rhs(n, 0) += S(n, 0);
        }
        if constexpr (WB) {
            const R g = p(0, 0);
            rhs(kIdxH + 1, 0) += xwb;
            if constexpr (dim == 2)
                rhs(kIdxH + 2, 0) += R(0.5) * g * (FyR[3 * NQE] * FyR[3 * NQE] - FyL[3 * NQE + 1] * FyL[3 * NQE + 1]) / L.dy;
        }
        const long long c = (long long)j * nx + i;
        if constexpr (MODE == MODE_RHS) {
#pragma unroll
            for (int n = 0; n < nq; ++n) qout[n * plane + c] = rhs(n, 0);
        } else {
            typename T::VQ q;
#pragma unroll
            for (int n = 0; n < nq; ++n) q(n, 0) = qc(n, 0) + dt * rhs(n, 0);
            if (qstar) {   // adjoint tape: the stage state before the implicit source
#pragma unroll
                for (int n = n0; n < nq; ++n) qstar[(n - n0) * plane + c] = q(n, 0);
            }
            if constexpr (IMPL && MODE != MODE_X) implicit_source_cell<Model, R>(q, ac, dt, p, time, X);
            if constexpr (MODE == MODE_S1 || MODE == MODE_R1 || MODE == MODE_X) {
#pragma unroll
                for (int n = (sbed ? 1 : 0); n < nq; ++n) qout[n * plane + c] = q(n, 0);
            } else if constexpr (MODE == MODE_S2M) {
                // Heun candidate; the MOOD test (ZoomyAmr.cpp:706-708) runs on it
                // before the final UpdateState, as in the reference
#pragma unroll
                for (int n = 0; n < nq; ++n) q(n, 0) = R(0.5) * qold[n * plane + c] + R(0.5) * q(n, 0);
#pragma unroll
                for (int n = (sbed ? 1 : 0); n < nq; ++n) qout[n * plane + c] = q(n, 0);
                const R hh = q(kIdxH, 0);
                if (!(hh >= R(0.0)) || !(hh < R(1.0e300))) atomicOr(&st->troubled, 1u);
            } else {
                if constexpr (MODE == MODE_S2 || MODE == MODE_R2) {
                    // Heun: Q = 0.5*Q^n + 0.5*Q** (the bed row of Q^n is qbed == qold row 0)
#pragma unroll
                    for (int n = 0; n < nq; ++n) q(n, 0) = R(0.5) * qold[n * plane + c] + R(0.5) * q(n, 0);
                }
                // final UpdateState (ZoomyAmr.cpp:730) and this cell's CFL / mass terms
                typename T::VA a2 = azero;
                update_state_cell<Model, R>(q, a2, p, L, time, X);
#pragma unroll
                for (int n = (sbed ? 1 : 0); n < nq; ++n) qout[n * plane + c] = q(n, 0);
                m_loc = cell_max_inv<Model, Numerics, R>(q, a2, p, L);
                s_loc = q(kIdxH, 0);
            }
        }
    }
    if constexpr (MODE == MODE_S2 || MODE == MODE_ONE || MODE == MODE_R2)
        finish_step<NT>(m_loc, s_loc, red, partials, log3, log_cap, st, L, dt, time, MODE == MODE_R2);
}

// MOOD commit (positivity = "mood", ZoomyAmr.cpp:699-730): when no cell of the
// order-2 candidate is troubled, the candidate becomes Q^{n+1} after the final
// UpdateState, and this kernel contributes the CFL / mass reduction. When the
// step is troubled it does nothing; the order-1 redo stages finish the step.
template <class Model, class Numerics, int NT>
__global__ void __launch_bounds__(NT)
k_mood_commit(const double* __restrict__ qcand, double* __restrict__ qout,
              LevelParams<double, Model::n_parameters> L, DevState* st,
              double* __restrict__ partials, double* __restrict__ log3, int log_cap) {
    using T = ModelTypes<Model>;
    constexpr bool sbed = static_bed<Model>::value;
    constexpr int nq = Model::n_dof_q;
    __shared__ double red[2 * ((NT + 31) / 32)];
    if (*(volatile unsigned*)&st->troubled != 0u) return;
    if (*(volatile unsigned*)&st->flags & kFlagDone) return;
    const double dt = *(volatile double*)&st->dt;
    const double time = *(volatile double*)&st->time;
    typename T::VP p;
    for (int k = 0; k < Model::n_parameters; ++k) p(k, 0) = L.p[k];
    const long long c = (long long)blockIdx.x * NT + threadIdx.x;
    double m_loc = 0.0, s_loc = 0.0;
    if (c < L.plane) {
        const int i = int(c % L.nx), j = int(c / L.nx);
        typename T::VQ q;
        q(0, 0) = sbed ? qout[c] : qcand[c];
#pragma unroll
        for (int n = 1; n < nq; ++n) q(n, 0) = qcand[n * L.plane + c];
        typename T::VA a{};
        update_state_cell<Model, double>(q, a, p, L, time, cell_centre<Model, double>(L, i, j));
#pragma unroll
        for (int n = (sbed ? 1 : 0); n < nq; ++n) qout[n * L.plane + c] = q(n, 0);
        m_loc = cell_max_inv<Model, Numerics, double>(q, a, p, L);
        s_loc = q(kIdxH, 0);
    }
    finish_step<NT>(m_loc, s_loc, red, partials, log3, log_cap, st, L, dt, time, false);
}

// ---------------------------------------------------------------------------
// Per-cell kernels with the reference's general aux handling (aux read from
// and written to memory). Used outside the stepping loop.
// ---------------------------------------------------------------------------
template <class Model>
__device__ __forceinline__ void load_cell(const double* Q, const double* A, long long plane,
                                          long long c, typename ModelTypes<Model>::VQ& q,
                                          typename ModelTypes<Model>::VA& a) {
#pragma unroll
    for (int n = 0; n < Model::n_dof_q; ++n) q(n, 0) = Q[n * plane + c];
#pragma unroll
    for (int n = 0; n < Model::n_dof_qaux; ++n) a(n, 0) = A[n * plane + c];
}

// ZoomyAmr::UpdateState in place on the valid cells.
template <class Model>
__global__ void k_update_state(double* Q, double* A, LevelParams<double, Model::n_parameters> L,
                               double time) {
    using T = ModelTypes<Model>;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= L.plane) return;
    const int i = int(c % L.nx), j = int(c / L.nx);
    typename T::VP p;
    for (int k = 0; k < Model::n_parameters; ++k) p(k, 0) = L.p[k];
    typename T::VQ q; typename T::VA a;
    load_cell<Model>(Q, A, L.plane, c, q, a);
    update_state_cell<Model, double>(q, a, p, L, time, cell_centre<Model, double>(L, i, j));
    for (int n = 0; n < Model::n_dof_q; ++n) Q[n * L.plane + c] = q(n, 0);
    for (int n = 0; n < Model::n_dof_qaux; ++n) A[n * L.plane + c] = a(n, 0);
}

// Grown arrays as UpdateState + FillPatch + FillPhysicalBC_mf leave them
// (validation entry). One thread per grown cell; ghost rows of 1-D models
// (j outside [0,ny)) are written as zeros, as they hold no data in the reference.
template <class Model>
__global__ void k_fill_ghosts(const double* Q, const double* A, double* Qg, double* Ag,
                              LevelParams<double, Model::n_parameters> L, int ng, double time) {
    using T = ModelTypes<Model>;
    constexpr int dim = Model::dimension;
    const int gxw = L.nx + 2 * ng, gyw = L.ny + 2 * ng;
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long gplane = (long long)gxw * gyw;
    if (k >= gplane) return;
    const int i = int(k % gxw) - ng, j = int(k / gxw) - ng;
    typename T::VP p;
    for (int n = 0; n < Model::n_parameters; ++n) p(n, 0) = L.p[n];
    const bool in_x = i >= 0 && i < L.nx, in_y = j >= 0 && j < L.ny;
    typename T::VQ q; typename T::VA a;
    if (in_x && in_y) {
        load_cell<Model>(Q, A, L.plane, (long long)j * L.nx + i, q, a);
        update_state_cell<Model, double>(q, a, p, L, time, cell_centre<Model, double>(L, i, j));
    } else {
        const GhostMap<dim> gm = ghost_map<dim>(i, j, L.nx, L.ny);
        const bool reach = gm.bc_side >= 0 && gm.ii >= 0 && gm.ii < L.nx && gm.jj >= 0 && gm.jj < L.ny;
        if (!reach) {
            for (int n = 0; n < Model::n_dof_q; ++n) Qg[n * gplane + k] = 0.0;
            for (int n = 0; n < Model::n_dof_qaux; ++n) Ag[n * gplane + k] = 0.0;
            return;
        }
        typename T::VQ qi; typename T::VA ai;
        load_cell<Model>(Q, A, L.plane, (long long)gm.jj * L.nx + gm.ii, qi, ai);
        update_state_cell<Model, double>(qi, ai, p, L, time, cell_centre<Model, double>(L, gm.ii, gm.jj));
        typename T::VN nh{};
        nh(gm.normal_dir, 0) = double(gm.normal_sign);
        const auto X = cell_centre<Model, double>(L, i, j);
        q = Model::boundary_conditions(L.bc_tag[gm.bc_side], qi, ai, nh, X, time, L.dx);
        a = Model::aux_boundary_conditions(L.bc_tag[gm.bc_side], qi, ai, nh, X, time, L.dx);
    }
    for (int n = 0; n < Model::n_dof_q; ++n) Qg[n * gplane + k] = q(n, 0);
    for (int n = 0; n < Model::n_dof_qaux; ++n) Ag[n * gplane + k] = a(n, 0);
}

// ZoomyAmr::ComputeDt on (Q, aux) as stored (WHAT 0) or the mass sum (WHAT 1);
// the last block writes st->dt / st->mass. With CLAMP_TO_END the dt is also
// clamped to land on time_end from st->time, as TimeStep does (ZoomyAmr.cpp:746-749).
template <class Model, class Numerics, int NT, int WHAT, bool CLAMP_TO_END>
__global__ void __launch_bounds__(NT)
k_reduce(const double* Q, const double* A, LevelParams<double, Model::n_parameters> L,
         DevState* st, double* partials) {
    using T = ModelTypes<Model>;
    __shared__ double red[2 * ((NT + 31) / 32)];
    __shared__ unsigned s_last;
    typename T::VP p;
    for (int k = 0; k < Model::n_parameters; ++k) p(k, 0) = L.p[k];
    double m = 0.0, s = 0.0;
    const long long stride = (long long)gridDim.x * NT;
    for (long long c = (long long)blockIdx.x * NT + threadIdx.x; c < L.plane; c += stride) {
        if constexpr (WHAT == 0) {
            typename T::VQ q; typename T::VA a;
            load_cell<Model>(Q, A, L.plane, c, q, a);
            const double v = cell_max_inv<Model, Numerics, double>(q, a, p, L);
            if (v > m) m = v;
        } else {
            s = s + Q[kIdxH * L.plane + c];
        }
    }
    block_reduce_max_sum<NT>(m, s, red);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = m;
        partials[2 * blockIdx.x + 1] = s;
        __threadfence();
        s_last = (atomicAdd(&st->counter, 1u) == gridDim.x - 1) ? 1u : 0u;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    double gm = 0.0, gs = 0.0;
#pragma unroll 8
    for (unsigned b = threadIdx.x; b < gridDim.x; b += NT) {
        const double pm = __ldcg(&partials[2 * b]), ps = __ldcg(&partials[2 * b + 1]);
        if (pm > gm) gm = pm;
        gs = gs + ps;
    }
    block_reduce_max_sum<NT>(gm, gs, red);
    if (threadIdx.x == 0) {
        if constexpr (WHAT == 0) {
            const double dt = CLAMP_TO_END ? dt_from_max(gm, st->time, L)
                                           : dt_from_max(gm, -1.0e300, L);
            st->max_inv = gm;
            st->dt = dt;
            if (!isfinite(dt)) st->flags |= kFlagNonfiniteDt;
        } else {
            st->mass = gs * (L.dx * L.dy);
        }
        st->counter = 0u;
        __threadfence();
    }
}

// Aux after a run: aux = update_aux_variables(Q, aux) on every cell (the
// reference's final UpdateState leaves exactly this in Qaux).
template <class Model>
__global__ void k_aux_from_state(const double* Q, double* A, LevelParams<double, Model::n_parameters> L,
                                 const DevState* st) {
    using T = ModelTypes<Model>;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= L.plane) return;
    const int i = int(c % L.nx), j = int(c / L.nx);
    typename T::VP p;
    for (int k = 0; k < Model::n_parameters; ++k) p(k, 0) = L.p[k];
    typename T::VQ q; typename T::VA a;
    load_cell<Model>(Q, A, L.plane, c, q, a);
    a = Model::update_aux_variables(q, a, p, st->time, cell_centre<Model, double>(L, i, j));
    for (int n = 0; n < Model::n_dof_qaux; ++n) A[n * L.plane + c] = a(n, 0);
}

// Start-of-run state: time = 0, step = 0, flags from the stop test.
template <class PL>
__global__ void k_begin(DevState* st, PL L) {
    st->time = 0.0; st->dt = 0.0; st->mass = 0.0; st->max_inv = 0.0;
    st->step = 0; st->flags = run_done(0.0, 0, L) ? kFlagDone : 0u; st->mood_redos = 0;
    st->counter = 0u;
    st->troubled = 0u;
}

}  // namespace zfv
