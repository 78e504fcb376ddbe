// Internals shared by the translation units of libzoomyfv.so (not installed).
#pragma once
#include <cstddef>
#include <memory>
#include <cuda_runtime.h>
#include "zoomy_fv.h"

namespace zfvi {

// Record an error message for zfv_last_error() and return `code`.
int fail(int code, const char* fmt, ...);
// 0 if e == cudaSuccess, else fail(-3, "<what>: <cuda message>").
int cuda_check(cudaError_t e, const char* what);

constexpr size_t kAlign = 256;
inline size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

constexpr int kLogCap = 4096;            // per-step log ring buffer entries
constexpr int kReduceNT = 256;
constexpr int kReduceBlocksMax = 1184;   // 8 x 148 SMs

// Scratch layout (byte offsets from the caller's scratch base).
struct ScratchLayout {
    size_t state = 0;        // DevState (128 B; first 64 B = zfv_status)
    size_t partials = 0;     // 2 doubles per block
    size_t log = 0;          // 3 doubles per entry
    size_t stage = 0;        // FP64: n_q stage planes; FP32: increment planes
    size_t alt = 0;          // FP32: ping-pong state planes
    size_t lo = 0;           // FP32: compensation planes
    size_t lo2 = 0;          // FP32 with MOOD: the order-2 candidate's compensation planes
    size_t jfnk = 0;         // FP64 with implicit_global: the Newton-Krylov work area
    size_t total = 0;
};

// Adjoint tape and work layout of one FP64 SWE2D level (zoomy_adj.cu).
// Tape, per recorded step: Q^n (4 planes), Y1 (4 planes, bed row unused),
// q* of stage 1 and of stage 2 (3 planes each: h, hu, hv), and the (time, dt)
// the step used.
struct AdjLayout {
    size_t off_X = 0, off_Y1 = 0, off_qs1 = 0, off_qs2 = 0, off_meta = 0, step_bytes = 0;
    size_t w_lamq = 0, w_loc = 0, w_lamY1 = 0, w_part = 0, w_amax = 0, w_counter = 0, w_total = 0;
    int nbA = 0, nbD = 0;       // blocks of the per-cell pass and of the dt pass
};
AdjLayout adj_layout(long long plane);
// Reverse of one recorded step (see fv_adjoint.cuh). `Lp` points to the
// level's zfv::LevelParams<double, 6>.
int adj_step_swe2d(const void* Lp, bool wb, bool impl, const AdjLayout& A, const char* tape_step,
                   double* lam, double* grad, const double* aux0, int n_aux, char* work,
                   cudaStream_t s);
// Process-wide tile shape of the face-reverse kernel (tuning).
int adj_set_variant(int v);
int adj_variants();

// One compiled model/precision: owns its kernel instantiations.
struct Runner {
    virtual ~Runner() = default;
    virtual int setup() = 0;
    virtual void layout(ScratchLayout& L) const = 0;
    virtual int begin(const void* Q, const void* A, char* scratch, cudaStream_t s) = 0;
    virtual int update_state(void* Q, void* A, double time, cudaStream_t s) = 0;
    virtual int compute_dt(const void* Q, const void* A, char* scratch, cudaStream_t s) = 0;
    virtual int total_mass(const void* Q, char* scratch, cudaStream_t s) = 0;
    virtual int evolve(void* Q, void* A, char* scratch, int n, cudaStream_t s) = 0;
    virtual int rhs(const void* Q, void* out, double time, cudaStream_t s) = 0;
    virtual int fill_ghosts(const void* Q, const void* A, void* Qg, void* Ag, double time,
                            cudaStream_t s) = 0;
    virtual int state_import(const double* Q64, void* Q, char* scratch, cudaStream_t s) = 0;
    virtual int state_export(const void* Q, const char* scratch, double* Q64, cudaStream_t s) = 0;
    // Adjoint (FP64 SWE2D, order 2): record n forward steps onto a tape, and
    // the reverse of recorded step k.
    virtual int adj_record(void*, void*, char*, char*, int, cudaStream_t) {
        return fail(-2, "zfv_adj_record: the adjoint is implemented for the FP64 SWE2D form, order 2");
    }
    virtual int adj_step(const char*, int, double*, double*, const double*, char*, cudaStream_t) {
        return fail(-2, "zfv_adj_step: the adjoint is implemented for the FP64 SWE2D form, order 2");
    }
    // Strip shape of the FP32 stage kernels (zfv_set_variant); the FP64 form
    // has one tile shape.
    virtual int set_variant(int, cudaStream_t) {
        return fail(-2, "zfv_set_variant: strip shapes are a property of the FP32 form");
    }
    virtual int variant() const { return -1; }
    // Global implicit source (implicit_global): iteration counts since the
    // last begin (Newton iterations, GMRES iterations, source solves).
    long long jfnk_newton = 0, jfnk_gmres = 0, jfnk_solves = 0;
};

}  // namespace zfvi

struct zfv_handle {
    zfv_config cfg;
    zfvi::ScratchLayout lay;
    std::unique_ptr<zfvi::Runner> run;
};

namespace zfvi {
// FP32 chosen-form runner for ZFV_MODEL_SWE2D (zoomy_fv32.cu).
Runner* make_runner_fp32_swe2d(zfv_handle* h);
// FP32 chosen-form runner of the generic tile kernels (zoomy_fv32_tile.cu):
// any compiled model family; ZFV_MODEL_SME2D_L2.
Runner* make_runner_fp32_generic(zfv_handle* h);
int fp32_tile_variants();
// FP64 plain-form runners (zoomy_fv64_swe.cu, zoomy_fv64_sme.cu).
Runner* make_runner_fp64_swe1d(zfv_handle* h);
Runner* make_runner_fp64_swe2d(zfv_handle* h);
Runner* make_runner_fp64_sme2d_l2(zfv_handle* h);
Runner* make_runner_fp64_sme1d_l2(zfv_handle* h);
}
