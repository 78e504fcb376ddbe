// libzoomyfv.so: the C ABI of include/zoomy_fv.h over the sm_100a kernels.
//
// Build (see zoomy_amrex_b200/build.py):
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 --fmad=false -std=c++17
//        -Xcompiler -fPIC -shared ...
// --fmad=false matches the reference's CUDA build (build.py:33-41) and keeps
// the FP64 arithmetic bitwise equal to the CPU build of the same expressions.
#include <atomic>
#include <cstdio>
#include <cstring>
#include <cstdarg>
#include <new>
#include <memory>
#include <string>
#include <algorithm>
#include <type_traits>
#include <cuda_runtime.h>

#include "zoomy_fv.h"
#include "zfv_internal.H"
#include "swe.H"
#include "sme.H"
#include "fv_kernels.cuh"

namespace zfvi {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int cuda_check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return 0;
    return fail(-3, "%s: %s", what, cudaGetErrorString(e));
}

}  // namespace zfvi

using namespace zfvi;

namespace {

template <class M>
int shape_of(int* nq, int* na, int* np, int* dim) {
    *nq = M::n_dof_q; *na = M::n_dof_qaux; *np = M::n_parameters; *dim = M::dimension;
    return 0;
}

int model_shape(int model, int* nq, int* na, int* np, int* dim) {
    switch (model) {
    case ZFV_MODEL_SWE1D: return shape_of<zb::SWE<double, 1>>(nq, na, np, dim);
    case ZFV_MODEL_SWE2D: return shape_of<zb::SWE<double, 2>>(nq, na, np, dim);
    case ZFV_MODEL_SME2D_L2: return shape_of<zb::SME<double, 2, 2>>(nq, na, np, dim);
    case ZFV_MODEL_SME1D_L2: return shape_of<zb::SME<double, 1, 2>>(nq, na, np, dim);
    default: return -1;
    }
}

// init_solution (Source/init_solution.cpp:78-116) on the device, as the
// reference's InitData applies it to Q and Qaux (ZoomyAmr.cpp:174-175): every
// component zero, and for a field of >= 2 components the flat-bed dam break
// b = 0, h = 2 | 1 split at the x mid-point. Component-major (n_comp, ny, nx).
__global__ void k_init_solution(double* __restrict__ f, int n_comp, long long plane, int nx, double lo,
                                double hi) {
    const double dx = (hi - lo) / nx;
    const double x_mid = 0.5 * (lo + hi);
    const long long total = plane * n_comp;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        double v = 0.0;
        if (n_comp >= 2 && e >= plane && e < 2 * plane) {
            const int i = int((e - plane) % nx);
            const double x = lo + (i + 0.5) * dx;
            v = (x < x_mid) ? 2.0 : 1.0;
        }
        f[e] = v;
    }
}

// Drops a destroyed handle from the static-scratch ownership record, so a
// later handle allocated at the same address cannot continue its run.
void static_scratch_forget(const zfv_handle* h);

}  // namespace

extern "C" {

const char* zfv_last_error(void) { return g_err.c_str(); }

int zfv_init_solution(const zfv_handle* h, double* field, int n_comp, void* stream) {
    if (!h || !field) return fail(-1, "zfv_init_solution: null argument");
    if (n_comp < 1) return fail(-1, "zfv_init_solution: n_comp must be >= 1");
    const long long plane = (long long)h->cfg.nx * h->cfg.ny;
    const long long total = plane * n_comp;
    const long long want = (total + 255) / 256;
    const int blocks = int(want < 148LL * 16 ? (want > 0 ? want : 1) : 148LL * 16);
    k_init_solution<<<blocks, 256, 0, (cudaStream_t)stream>>>(field, n_comp, plane, h->cfg.nx, h->cfg.prob_lo[0],
                                                              h->cfg.prob_hi[0]);
    return cuda_check(cudaGetLastError(), "zfv_init_solution launch");
}

const char* zfv_version(void) { return "zoomyfv 0.1 sm_100a fp64"; }

size_t zfv_sizeof_config(void) { return sizeof(zfv_config); }
size_t zfv_sizeof_status(void) { return sizeof(zfv_status); }

int zfv_model_info(int model, int* n_q, int* n_aux, int* n_params, int* dimension) {
    int a, b, c, d;
    if (model_shape(model, &a, &b, &c, &d) != 0) return fail(-1, "unknown model id %d", model);
    if (n_q) *n_q = a;
    if (n_aux) *n_aux = b;
    if (n_params) *n_params = c;
    if (dimension) *dimension = d;
    return 0;
}

int zfv_create(const zfv_config* cfg, zfv_handle** out) {
    g_err.clear();
    if (!cfg || !out) return fail(-1, "zfv_create: null argument");
    *out = nullptr;
    int nq, na, np, dim;
    if (model_shape(cfg->model, &nq, &na, &np, &dim) != 0)
        return fail(-1, "zfv_create: unknown model id %d", cfg->model);
    if (cfg->precision != ZFV_PREC_FP64 && cfg->precision != ZFV_PREC_FP32)
        return fail(-1, "zfv_create: unsupported precision %d", cfg->precision);
    if (cfg->precision == ZFV_PREC_FP32) {
        if (cfg->model != ZFV_MODEL_SWE2D && cfg->model != ZFV_MODEL_SME2D_L2)
            return fail(-1, "zfv_create: the FP32 form is built for ZFV_MODEL_SWE2D and ZFV_MODEL_SME2D_L2");
        if (cfg->clamp_positivity)
            return fail(-1, "zfv_create: the FP32 form does not implement clamp_positivity");
    }
    if (cfg->implicit_global && cfg->implicit_source) {
        if (cfg->precision != ZFV_PREC_FP64)
            return fail(-1, "zfv_create: implicit_global is built for the FP64 form");
        if (cfg->positivity_mood)
            return fail(-1, "zfv_create: implicit_global with positivity mood is not built");
    }
    if (cfg->nx < 1 || cfg->ny < 1) return fail(-1, "zfv_create: bad grid %d x %d", cfg->nx, cfg->ny);
    if (dim == 1 && cfg->ny != 1) return fail(-1, "zfv_create: 1-D model needs ny == 1 (got %d)", cfg->ny);
    if ((long long)cfg->nx * cfg->ny > (1LL << 31))
        return fail(-1, "zfv_create: grid too large for one level (%lld cells)", (long long)cfg->nx * cfg->ny);
    if (cfg->spatial_order != 1 && cfg->spatial_order != 2)
        return fail(-1, "zfv_create: spatial_order must be 1 or 2 (got %d)", cfg->spatial_order);
    {
        // Every ghost layer must mirror onto a valid cell (ZoomyAmr.cpp:399-406);
        // with fewer cells than ghost layers the reference mirrors a ghost onto
        // another ghost, which has no defined value.
        const int ng = (cfg->spatial_order == 2) ? 2 : 1;
        if (cfg->nx < ng || (dim == 2 && cfg->ny < ng))
            return fail(-1, "zfv_create: order %d needs at least %d cells per direction (grid %d x %d)",
                        cfg->spatial_order, ng, cfg->nx, cfg->ny);
    }
    if (cfg->n_params != np)
        return fail(-1, "zfv_create: model takes %d parameters, config has %d", np, cfg->n_params);
    if (!(cfg->prob_hi[0] > cfg->prob_lo[0]) || !(cfg->prob_hi[1] > cfg->prob_lo[1]))
        return fail(-1, "zfv_create: empty domain");
    if (cfg->cfl_dimension < 1 || cfg->cfl_degree_factor < 1)
        return fail(-1, "zfv_create: march constants must be >= 1");
    for (int s = 0; s < 4; ++s)
        if (cfg->bc_tag[s] < 0 || cfg->bc_tag[s] >= 2)
            return fail(-1, "zfv_create: bc tag %d on side %d is not declared by the model", cfg->bc_tag[s], s);

    zfv_handle* h = new (std::nothrow) zfv_handle();
    if (!h) return fail(-4, "zfv_create: out of host memory");
    h->cfg = *cfg;
    if (cfg->precision == ZFV_PREC_FP32) {
        // the shallow-water sweep is order 2 without MOOD; order 1 and MOOD run on
        // the generic tile kernels
        if (cfg->model == ZFV_MODEL_SWE2D && cfg->spatial_order == 2 && !cfg->positivity_mood)
            h->run.reset(make_runner_fp32_swe2d(h));
        else h->run.reset(make_runner_fp32_generic(h));
    } else {
        switch (cfg->model) {
        case ZFV_MODEL_SWE1D: h->run.reset(make_runner_fp64_swe1d(h)); break;
        case ZFV_MODEL_SWE2D: h->run.reset(make_runner_fp64_swe2d(h)); break;
        case ZFV_MODEL_SME2D_L2: h->run.reset(make_runner_fp64_sme2d_l2(h)); break;
        case ZFV_MODEL_SME1D_L2: h->run.reset(make_runner_fp64_sme1d_l2(h)); break;
        }
    }
    if (!h->run) {
        delete h;
        return fail(-2, "zfv_create: precision %d is not built for model %d", cfg->precision, cfg->model);
    }
    int rc = h->run->setup();
    if (rc) { delete h; return rc; }
    h->run->layout(h->lay);
    *out = h;
    return 0;
}

int zfv_destroy(zfv_handle* h) {
    static_scratch_forget(h);
    delete h;
    return 0;
}

size_t zfv_scratch_bytes(const zfv_handle* h) { return h ? h->lay.total : 0; }

int zfv_begin(zfv_handle* h, const void* Q, const void* aux, void* scratch, void* stream) {
    if (!h || !Q || !aux || !scratch) return fail(-1, "zfv_begin: null argument");
    return h->run->begin(Q, aux, (char*)scratch, (cudaStream_t)stream);
}

int zfv_set_variant(zfv_handle* h, int variant, void* stream) {
    if (!h) return fail(-1, "zfv_set_variant: null handle");
    return h->run->set_variant(variant, (cudaStream_t)stream);
}

int zfv_get_variant(const zfv_handle* h) { return h ? h->run->variant() : -1; }

int zfv_implicit_global_stats(const zfv_handle* h, long long* solves, long long* newton, long long* gmres) {
    if (!h) return fail(-1, "zfv_implicit_global_stats: null handle");
    if (solves) *solves = h->run->jfnk_solves;
    if (newton) *newton = h->run->jfnk_newton;
    if (gmres) *gmres = h->run->jfnk_gmres;
    return 0;
}

int zfv_update_state(zfv_handle* h, void* Q, void* aux, double time, void* stream) {
    if (!h || !Q || !aux) return fail(-1, "zfv_update_state: null argument");
    return h->run->update_state(Q, aux, time, (cudaStream_t)stream);
}

int zfv_compute_dt(zfv_handle* h, const void* Q, const void* aux, void* scratch, void* stream) {
    if (!h || !Q || !aux || !scratch) return fail(-1, "zfv_compute_dt: null argument");
    return h->run->compute_dt(Q, aux, (char*)scratch, (cudaStream_t)stream);
}

int zfv_evolve(zfv_handle* h, void* Q, void* aux, void* scratch, int n_steps, void* stream) {
    if (!h || !Q || !aux || !scratch) return fail(-1, "zfv_evolve: null argument");
    if (n_steps < 0) return fail(-1, "zfv_evolve: negative step count");
    return h->run->evolve(Q, aux, (char*)scratch, n_steps, (cudaStream_t)stream);
}

int zfv_rhs(zfv_handle* h, const void* Q, const void* aux, void* rhs, double time, void* stream) {
    if (!h || !Q || !rhs) return fail(-1, "zfv_rhs: null argument");
    (void)aux;
    return h->run->rhs(Q, rhs, time, (cudaStream_t)stream);
}

int zfv_fill_ghosts(zfv_handle* h, const void* Q, const void* aux, void* Qg, void* auxg,
                    double time, void* stream) {
    if (!h || !Q || !aux || !Qg || !auxg) return fail(-1, "zfv_fill_ghosts: null argument");
    return h->run->fill_ghosts(Q, aux, Qg, auxg, time, (cudaStream_t)stream);
}

int zfv_state_import(zfv_handle* h, const double* Q64, void* Q, void* scratch, void* stream) {
    if (!h || !Q64 || !Q || !scratch) return fail(-1, "zfv_state_import: null argument");
    return h->run->state_import(Q64, Q, (char*)scratch, (cudaStream_t)stream);
}

int zfv_state_export(zfv_handle* h, const void* Q, const void* scratch, double* Q64, void* stream) {
    if (!h || !Q64 || !Q || !scratch) return fail(-1, "zfv_state_export: null argument");
    return h->run->state_export(Q, (const char*)scratch, Q64, (cudaStream_t)stream);
}

int zfv_total_mass(zfv_handle* h, const void* Q, void* scratch, void* stream) {
    if (!h || !Q || !scratch) return fail(-1, "zfv_total_mass: null argument");
    return h->run->total_mass(Q, (char*)scratch, (cudaStream_t)stream);
}

int zfv_get_status(zfv_handle* h, const void* scratch, zfv_status* out, void* stream) {
    if (!h || !scratch || !out) return fail(-1, "zfv_get_status: null argument");
    static_assert(sizeof(zfv_status) == 64, "zfv_status is 64 bytes");
    cudaStream_t s = (cudaStream_t)stream;
    int rc = cuda_check(cudaMemcpyAsync(out, (const char*)scratch + h->lay.state, sizeof(zfv_status),
                                        cudaMemcpyDeviceToHost, s), "zfv_get_status copy");
    if (rc) return rc;
    return cuda_check(cudaStreamSynchronize(s), "zfv_get_status sync");
}

int zfv_save_run_state(zfv_handle* h, const void* scratch, void* dst, void* stream) {
    if (!h || !scratch || !dst) return fail(-1, "zfv_save_run_state: null argument");
    return cuda_check(cudaMemcpyAsync(dst, static_cast<const char*>(scratch) + h->lay.state,
                                      sizeof(zfv::DevState), cudaMemcpyDeviceToDevice, (cudaStream_t)stream),
                      "zfv_save_run_state copy");
}

int zfv_load_run_state(zfv_handle* h, void* scratch, const void* src, void* stream) {
    if (!h || !scratch || !src) return fail(-1, "zfv_load_run_state: null argument");
    return cuda_check(cudaMemcpyAsync(static_cast<char*>(scratch) + h->lay.state, src,
                                      sizeof(zfv::DevState), cudaMemcpyDeviceToDevice, (cudaStream_t)stream),
                      "zfv_load_run_state copy");
}

size_t zfv_run_state_bytes(void) { return sizeof(zfv::DevState); }

size_t zfv_adj_tape_bytes(const zfv_handle* h, int n_steps) {
    if (!h || n_steps < 0) return 0;
    return adj_layout((long long)h->cfg.nx * h->cfg.ny).step_bytes * size_t(n_steps);
}

size_t zfv_adj_work_bytes(const zfv_handle* h) {
    return h ? adj_layout((long long)h->cfg.nx * h->cfg.ny).w_total : 0;
}

int zfv_adj_record(zfv_handle* h, void* Q, void* aux, void* scratch, void* tape, int n_steps, void* stream) {
    if (!h || !Q || !aux || !scratch || !tape) return fail(-1, "zfv_adj_record: null argument");
    if (n_steps < 0) return fail(-1, "zfv_adj_record: negative step count");
    return h->run->adj_record(Q, aux, static_cast<char*>(scratch), static_cast<char*>(tape), n_steps,
                              (cudaStream_t)stream);
}

int zfv_adj_step(zfv_handle* h, const void* tape, int k, void* lam, double* grad, const void* aux0,
                 void* work, void* stream) {
    if (!h || !tape || !lam || !grad || !work) return fail(-1, "zfv_adj_step: null argument");
    if (k < 0) return fail(-1, "zfv_adj_step: negative step index");
    return h->run->adj_step(static_cast<const char*>(tape), k, static_cast<double*>(lam), grad,
                            static_cast<const double*>(aux0), static_cast<char*>(work), (cudaStream_t)stream);
}

int zfv_adj_steps(zfv_handle* h, const void* tape, int n_steps, void* lam, double* grad, const void* aux0,
                  void* work, void* stream) {
    if (!h || !tape || !lam || !grad || !work) return fail(-1, "zfv_adj_steps: null argument");
    if (n_steps < 0) return fail(-1, "zfv_adj_steps: negative step count");
    for (int k = n_steps - 1; k >= 0; --k) {
        const int rc = h->run->adj_step(static_cast<const char*>(tape), k, static_cast<double*>(lam), grad,
                                        k == 0 ? static_cast<const double*>(aux0) : nullptr,
                                        static_cast<char*>(work), (cudaStream_t)stream);
        if (rc) return rc;
    }
    return 0;
}

int zfv_adj_set_variant(int variant) { return adj_set_variant(variant); }

int zfv_adj_variants(void) { return adj_variants(); }

int zfv_log_capacity(const zfv_handle* h) { return h ? kLogCap : 0; }

int zfv_read_log(zfv_handle* h, const void* scratch, double* out3, int max_entries,
                 int64_t* first_step, int* n_out, void* stream) {
    if (!h || !scratch || !out3 || !first_step || !n_out) return fail(-1, "zfv_read_log: null argument");
    zfv_status stt;
    int rc = zfv_get_status(h, scratch, &stt, stream);
    if (rc) return rc;
    const long long steps = stt.step;
    const long long avail = steps < kLogCap ? steps : kLogCap;
    const long long n = avail < max_entries ? avail : max_entries;
    const long long first = steps - n;   // 0-based index of the first returned step
    static thread_local double ring[3 * kLogCap];
    rc = cuda_check(cudaMemcpyAsync(ring, (const char*)scratch + h->lay.log, sizeof(double) * 3 * kLogCap,
                                    cudaMemcpyDeviceToHost, (cudaStream_t)stream), "zfv_read_log copy");
    if (rc) return rc;
    rc = cuda_check(cudaStreamSynchronize((cudaStream_t)stream), "zfv_read_log sync");
    if (rc) return rc;
    for (long long k = 0; k < n; ++k) {
        const long long s = first + k;
        std::memcpy(out3 + 3 * k, ring + 3 * (s % kLogCap), 3 * sizeof(double));
    }
    *first_step = first + 1;
    *n_out = int(n);
    return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free entry point.
//
// For callers that cannot call cudaMalloc: code running where a device
// allocation is not allowed or not possible, e.g. inside another framework's
// memory pool that forbids foreign allocations, a host that has handed all
// device memory to a caching allocator, or a plugin that must not grow the
// process's footprint at call time. The step's scratch (run record, reduction
// partials, step log and the SSP-RK2 stage buffer) lives in a fixed array
// compiled into this library; the caller only passes Q and aux.
// ---------------------------------------------------------------------------
namespace {

// 64 MiB per GPU that loads the library, held until process exit. Enough for
// about 2 million cells of the 2-D shallow-water model (4 state planes of
// FP64 in the stage buffer plus a few hundred KB of bookkeeping).
constexpr size_t kStaticScratchBytes = size_t(64) << 20;
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// Device address of g_static_scratch per device ordinal. In host code the
// symbol's name is only a host-side stand-in, never a device address.
constexpr int kMaxDevices = 64;
std::atomic<void*> g_static_scratch_addr[kMaxDevices];
// The handle whose run the array holds, per device: set by a restart, checked
// by a continuation (restart == 0), so a call never continues a run record
// laid out for another handle or one that no restart ever initialised.
std::atomic<const zfv_handle*> g_static_scratch_owner[kMaxDevices];

void static_scratch_forget(const zfv_handle* h) {
    for (int d = 0; d < kMaxDevices; ++d) {
        const zfv_handle* expect = h;
        g_static_scratch_owner[d].compare_exchange_strong(expect, nullptr, std::memory_order_acq_rel);
    }
}

}  // namespace

extern "C" int zfv_evolve_static(zfv_handle* h, void* Q, void* aux, int n_steps, int restart,
                                 zfv_status* status_out, void* stream) {
    if (!h || !Q || !aux) return fail(-1, "zfv_evolve_static: null argument");
    if (n_steps < 0) return fail(-1, "zfv_evolve_static: negative step count");
    if (h->cfg.precision != ZFV_PREC_FP64)
        return fail(-1, "zfv_evolve_static: only FP64 handles are accepted (the FP32 form keeps its "
                        "state remainder in scratch, which only zfv_state_import/export reach; use "
                        "zfv_evolve with caller-provided scratch)");
    if (h->lay.total > kStaticScratchBytes)
        return fail(-5, "zfv_evolve_static: this level needs %zu bytes of scratch; the static "
                        "scratch holds %zu bytes (grid %d x %d is too large for this entry point, "
                        "use zfv_evolve with caller-provided scratch)",
                    h->lay.total, kStaticScratchBytes, h->cfg.nx, h->cfg.ny);
    int dev = -1;
    int rc = cuda_check(cudaGetDevice(&dev), "zfv_evolve_static: cudaGetDevice");
    if (rc) return rc;
    if (dev < 0 || dev >= kMaxDevices) return fail(-1, "zfv_evolve_static: device %d out of range", dev);
    void* base = g_static_scratch_addr[dev].load(std::memory_order_acquire);
    if (!base) {   // once per device, with that device current
        void* addr = nullptr;
        rc = cuda_check(cudaGetSymbolAddress(&addr, g_static_scratch),
                        "zfv_evolve_static: cudaGetSymbolAddress");
        if (rc) return rc;
        g_static_scratch_addr[dev].store(addr, std::memory_order_release);
        base = addr;
    }
    char* scratch = static_cast<char*>(base);
    cudaStream_t s = (cudaStream_t)stream;
    if (restart) {
        // the run record (time, step, flags, reduction counter) must start at zero
        g_static_scratch_owner[dev].store(nullptr, std::memory_order_release);
        rc = h->run->begin(Q, aux, scratch, s);
        if (rc) return rc;
        g_static_scratch_owner[dev].store(h, std::memory_order_release);
    } else if (g_static_scratch_owner[dev].load(std::memory_order_acquire) != h) {
        return fail(-1, "zfv_evolve_static: restart == 0 continues the run this handle started on "
                        "device %d, but the array holds no run of this handle (no restart yet, or "
                        "another handle restarted since)", dev);
    }
    rc = h->run->evolve(Q, aux, scratch, n_steps, s);
    if (rc) return rc;
    if (status_out) {
        rc = cuda_check(cudaMemcpyAsync(status_out, scratch + h->lay.state, sizeof(zfv_status),
                                        cudaMemcpyDeviceToHost, s), "zfv_evolve_static status copy");
        if (rc) return rc;
        rc = cuda_check(cudaStreamSynchronize(s), "zfv_evolve_static sync");
    }
    return rc;
}

