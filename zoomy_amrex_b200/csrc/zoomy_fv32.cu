// The FP32 chosen form of the 2-D shallow-water step (ZFV_PREC_FP32).
//
// Same scheme as the FP64 plain form — MUSCL/minmod reconstruction of b and h,
// Audusse hydrostatic reconstruction, central flux + Rusanov D± fluctuations,
// point-implicit Manning source, SSP-RK2 (Heun) — evaluated so that FP32
// storage and arithmetic lose as little as possible:
//  * the state is stored as [b, eta = h + b, hu, hv] in FP32, and the slopes of
//    h are taken as d(eta) - d(b), so a lake at rest (eta constant, u = 0)
//    reconstructs eta at every face bit for bit: the face depths on both sides
//    of a face are equal and the hydrostatic pressure P(h) = (g/2) h^2 enters
//    the flux and the well-balancing bed source as the same FP32 values, which
//    cancel exactly;
//  * the update is compensated: stage 1 stores only its FP32 increment inc1,
//    stage 2 forms Q^{n+1} = (hi + lo) + (inc1 + inc2)/2 in FP64 per cell and
//    splits it again into an FP32 value (hi, the state the fluxes read) and an
//    FP32 remainder (lo, kept in scratch); so round-off of the stored state
//    does not accumulate step after step;
//  * FP64 is used only in the point-implicit source solve of near-dry cells
//    (h < 1e-3) and in the mass sum.
// Kernels are compiled with FMA contraction on (this file only).
#include <algorithm>
#include <cuda_runtime.h>

#include "zfv_internal.H"
#include "fv_kernels.cuh"
#include "swe.H"
#include "zb_portable_math.H"

using namespace zfvi;

namespace zfv32 {

struct Params {
    int nx, ny;
    long long plane;
    double dx, dy, plox, ploy;       // FP64 (reductions, dt)
    float fdx, fdy, rdx, rdy;
    float g, ex, ey, nm, hfloor, eps;
    double gd, exd, eyd, nmd, hfloord, epsd;
    int bc_tag[4];
    double cfl, dtmin, dtmax, time_end;
    int max_step, cfl_dimension, cfl_degree_factor;
};

struct C4 { float b, e, u, v; };   // bed, surface eta = h + b, hu, hv

constexpr float kNearDry = 1.0e-3f;   // FP64 implicit solve below this depth

__device__ __forceinline__ float mm(float a, float b) {
    if (a * b <= 0.0f) return 0.0f;
    return (fabsf(a) < fabsf(b)) ? a : b;
}

// Kurganov-Petrova desingularised 1/h (the model's update_aux_variables), FP32.
__device__ __forceinline__ float kp_hinv(float h, float eps) {
    const float h2 = h * h;
    const float x0 = h2 * h2;
    return 1.41421356237f * h * rsqrtf(x0 + fmaxf(x0, eps));
}
__device__ __forceinline__ double kp_hinv_d(double h, double eps) {
    const double h2 = h * h;
    const double x0 = h2 * h2;
    return 1.4142135623730951 * h / sqrt(x0 + fmax(x0, eps));
}

// Face record: flux (h, hu, hv), D+ (3), D- (3), P(h*_L), P(h*_R).
constexpr int NFC = 11;

template <int ORDER, int DIR, bool WB>
__device__ __forceinline__ void face(const C4& LL, const C4& Lc, const C4& Rc, const C4& RR,
                                     const Params& L, float* __restrict__ F) {
    float bL, bR, eL, eR, hL, hR, uL, uR, vL, vR;
    if constexpr (ORDER == 2) {
        const float db1 = Lc.b - LL.b, db2 = Rc.b - Lc.b, db3 = RR.b - Rc.b;
        const float de1 = Lc.e - LL.e, de2 = Rc.e - Lc.e, de3 = RR.e - Rc.e;
        const float gbL = mm(db1, db2), gbR = mm(db2, db3);
        const float ghL = mm(de1 - db1, de2 - db2), ghR = mm(de2 - db2, de3 - db3);
        bL = Lc.b + 0.5f * gbL;  bR = Rc.b - 0.5f * gbR;
        hL = (Lc.e - Lc.b) + 0.5f * ghL;  hR = (Rc.e - Rc.b) - 0.5f * ghR;
        eL = Lc.e + 0.5f * (ghL + gbL);  eR = Rc.e - 0.5f * (ghR + gbR);
        uL = Lc.u + 0.5f * mm(Lc.u - LL.u, Rc.u - Lc.u);
        uR = Rc.u - 0.5f * mm(Rc.u - Lc.u, RR.u - Rc.u);
        vL = Lc.v + 0.5f * mm(Lc.v - LL.v, Rc.v - Lc.v);
        vR = Rc.v - 0.5f * mm(Rc.v - Lc.v, RR.v - Rc.v);
    } else {
        bL = Lc.b; bR = Rc.b; eL = Lc.e; eR = Rc.e;
        hL = Lc.e - Lc.b; hR = Rc.e - Rc.b;
        uL = Lc.u; uR = Rc.u; vL = Lc.v; vR = Rc.v;
    }
    float db = 0.0f;
    if constexpr (WB) {
        const float bf = fmaxf(bL, bR);
        const float hsL = fmaxf(0.0f, eL - bf), hsR = fmaxf(0.0f, eR - bf);
        const float sL = (hL > 0.0f) ? hsL / hL : 0.0f;
        const float sR = (hR > 0.0f) ? hsR / hR : 0.0f;
        uL *= sL; vL *= sL; uR *= sR; vR *= sR;
        hL = hsL; hR = hsR;
    } else {
        db = bR - bL;
    }
    const float g = L.g, hg = 0.5f * L.g;
    const float hiL = kp_hinv(hL, L.eps), hiR = kp_hinv(hR, L.eps);
    const float unL = (DIR == 0) ? uL : vL, unR = (DIR == 0) ? uR : vR;
    const float pL = hg * hL * hL, pR = hg * hR * hR;
    float fuL, fvL, fuR, fvR;
    if constexpr (DIR == 0) {
        fuL = uL * uL * hiL + pL;  fvL = vL * uL * hiL;
        fuR = uR * uR * hiR + pR;  fvR = vR * uR * hiR;
    } else {
        fuL = uL * vL * hiL;  fvL = vL * vL * hiL + pL;
        fuR = uR * vR * hiR;  fvR = vR * vR * hiR + pR;
    }
    F[0] = 0.5f * (unL + unR);
    F[1] = 0.5f * (fuL + fuR);
    F[2] = 0.5f * (fvL + fvR);
    const float evL = fabsf(unL * hiL) + sqrtf(g * fmaxf(hL, 0.0f));
    const float evR = fabsf(unR * hiR) + sqrtf(g * fmaxf(hR, 0.0f));
    const float hs = 0.5f * fmaxf(evL, evR);
    const float dh = hR - hL, du = uR - uL, dv = vR - vL;
    float bu = 0.0f, bv = 0.0f;
    if constexpr (!WB) {
        const float Bn = g * (0.5f * (hL + hR)) * db;
        if (DIR == 0) bu = 0.5f * Bn; else bv = 0.5f * Bn;
    }
    F[3] = hs * dh;        F[6] = -hs * dh;          // D+ / D-, h
    F[4] = bu + hs * du;   F[7] = bu - hs * du;      // hu
    F[5] = bv + hs * dv;   F[8] = bv - hs * dv;      // hv
    F[9] = pL;
    F[10] = pR;
}

// Manning friction S_m = g e_m h - k u_m |u|, k = g n^2 max(h, h_floor)^(-1/3),
// and its Jacobian w.r.t. (hu, hv) with hinv held fixed; the point-implicit
// update solves (I - dt J) dq = dt S on the momentum block (the bed and depth
// rows of J are zero, so the reference's 4x4 elimination reduces to it).
template <class T>
__device__ __forceinline__ void manning_implicit(T h, T u, T v, T hinv, T dt, T g, T ex, T ey, T nm,
                                                 T hfloor, T& du, T& dv) {
    const T m = (h > hfloor) ? h : hfloor;
    const T k = g * nm * nm * zb::inv_cbrt_pos(m);
    const T ux = u * hinv, uy = v * hinv;
    const T sp = sqrt(ux * ux + uy * uy);
    const T Su = g * ex * h - k * ux * sp;
    const T Sv = g * ey * h - k * uy * sp;
    const T rsp = (sp > T(0)) ? T(1) / sp : T(0);
    const T dsx = ux * hinv * rsp, dsy = uy * hinv * rsp;
    const T J22 = -k * (hinv * sp + ux * dsx), J23 = -k * (ux * dsy);
    const T J32 = -k * (uy * dsx), J33 = -k * (hinv * sp + uy * dsy);
    const T a = T(1) - dt * J22, b = -dt * J23, c = -dt * J32, d = T(1) - dt * J33;
    const T det = a * d - b * c;
    const T r0 = dt * Su, r1 = dt * Sv;
    bool ok = (fabs(det) > T(0)) && isfinite(det);
    T x0 = T(0), x1 = T(0);
    if (ok) {
        x0 = (r0 * d - b * r1) / det;
        x1 = (a * r1 - c * r0) / det;
        ok = isfinite(x0) && isfinite(x1);
    }
    if (!ok) {   // explicit fallback, as make_rhs.H:501-508
        x0 = isfinite(r0) ? r0 : T(0);
        x1 = isfinite(r1) ? r1 : T(0);
    }
    du = x0;
    dv = x1;
}

enum Mode { S1 = 1, S2 = 2 };

}  // namespace zfv32

#include "fv32_sweep.cuh"

namespace zfv32 {

// FP64 reference layout [b, h, hu, hv] -> FP32 [b, eta, hu, hv] + remainders.
__global__ void k32_import(const double* __restrict__ Q64, float* __restrict__ Q, float* __restrict__ lo,
                           long long plane) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= plane) return;
    // eta from the FP64 bed: a surface that is constant in FP64 (a lake at rest)
    // rounds to the same FP32 value in every cell. The FP32 form's depth is
    // eta - b32, within half an FP32 ulp of b of the FP64 depth.
    const float b = float(Q64[c]);
    const double eta = Q64[plane + c] + Q64[c];
    const double hu = Q64[2 * plane + c], hv = Q64[3 * plane + c];
    const float e = float(eta), u = float(hu), v = float(hv);
    Q[c] = b; Q[plane + c] = e; Q[2 * plane + c] = u; Q[3 * plane + c] = v;
    lo[c] = float(eta - double(e));
    lo[plane + c] = float(hu - double(u));
    lo[2 * plane + c] = float(hv - double(v));
}

__global__ void k32_export(const float* __restrict__ Q, const float* __restrict__ lo,
                           double* __restrict__ Q64, long long plane) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= plane) return;
    const double b = double(Q[c]);
    const double eta = double(Q[plane + c]) + double(lo[c]);
    Q64[c] = b;
    Q64[plane + c] = eta - b;
    Q64[2 * plane + c] = double(Q[2 * plane + c]) + double(lo[plane + c]);
    Q64[3 * plane + c] = double(Q[3 * plane + c]) + double(lo[2 * plane + c]);
}

// Final aux: hinv of the FP64 state (the carried rows stay untouched).
__global__ void k32_aux(const float* __restrict__ Q, const float* __restrict__ lo, double* __restrict__ A,
                        long long plane, int n_aux, double eps) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= plane) return;
    const double h = (double(Q[plane + c]) + double(lo[c])) - double(Q[c]);
    A[(n_aux - 1) * plane + c] = kp_hinv_d(h, eps);
}

// ComputeDt on the stored state and aux (WHAT 0, clamped to time_end) or the
// FP64 mass (WHAT 1).
template <int NT, int WHAT>
__global__ void __launch_bounds__(NT)
k32_reduce(const float* __restrict__ Q, const float* __restrict__ lo, const double* __restrict__ A,
           int n_aux, Params L, zfv::DevState* st, double* partials) {
    __shared__ double red[2 * ((NT + 31) / 32)];
    __shared__ unsigned s_last;
    const long long plane = L.plane;
    double m = 0.0, s = 0.0;
    const long long stride = (long long)gridDim.x * NT;
    for (long long c = (long long)blockIdx.x * NT + threadIdx.x; c < plane; c += stride) {
        const double b = double(Q[c]);
        const double h = (double(Q[plane + c]) + double(lo[c])) - b;
        if constexpr (WHAT == 0) {
            const double hinv = A[(n_aux - 1) * plane + c];
            const double c0 = sqrt(L.gd * fmax(h, 0.0));
            const double hu = double(Q[2 * plane + c]) + double(lo[plane + c]);
            const double hv = double(Q[3 * plane + c]) + double(lo[2 * plane + c]);
            const double ix = (fabs(hu * hinv) + c0) / L.dx, iy = (fabs(hv * hinv) + c0) / L.dy;
            if (ix > m) m = ix;
            if (iy > m) m = iy;
        } else {
            s = s + h;
        }
    }
    zfv::block_reduce_max_sum<NT>(m, s, red);
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
    for (unsigned bb = threadIdx.x; bb < gridDim.x; bb += NT) {
        const double pm = __ldcg(&partials[2 * bb]), ps = __ldcg(&partials[2 * bb + 1]);
        if (pm > gm) gm = pm;
        gs = gs + ps;
    }
    zfv::block_reduce_max_sum<NT>(gm, gs, red);
    if (threadIdx.x == 0) {
        if constexpr (WHAT == 0) {
            const double dt = zfv::dt_from_max(gm, st->time, L);
            st->max_inv = gm;
            st->dt = dt;
            if (!isfinite(dt)) st->flags |= zfv::kFlagNonfiniteDt;
        } else {
            st->mass = gs * (L.dx * L.dy);
        }
        st->counter = 0u;
        __threadfence();
    }
}

// ---------------------------------------------------------------------------
template <int NW, int CPT>
struct Runner32 final : Runner {
    zfv_handle* h;
    Params L;
    dim3 grid, block;
    static constexpr int n_aux = zb::SWE<double, 2>::n_dof_qaux;

    explicit Runner32(zfv_handle* hh) : h(hh) {
        const zfv_config& c = h->cfg;
        L.nx = c.nx; L.ny = c.ny; L.plane = (long long)c.nx * c.ny;
        L.dx = (c.prob_hi[0] - c.prob_lo[0]) / c.nx;
        L.dy = (c.prob_hi[1] - c.prob_lo[1]) / c.ny;
        L.plox = c.prob_lo[0]; L.ploy = c.prob_lo[1];
        L.fdx = float(L.dx); L.fdy = float(L.dy);
        L.rdx = float(1.0 / L.dx); L.rdy = float(1.0 / L.dy);
        L.gd = c.params[zb::swe_g]; L.exd = c.params[zb::swe_ex]; L.eyd = c.params[zb::swe_ey];
        L.nmd = c.params[zb::swe_n_m]; L.hfloord = c.params[zb::swe_h_floor]; L.epsd = c.params[zb::swe_eps];
        L.g = float(L.gd); L.ex = float(L.exd); L.ey = float(L.eyd); L.nm = float(L.nmd);
        L.hfloor = float(L.hfloord); L.eps = float(L.epsd);
        for (int s = 0; s < 4; ++s) L.bc_tag[s] = c.bc_tag[s];
        L.cfl = c.cfl; L.dtmin = c.dtmin; L.dtmax = c.dtmax; L.time_end = c.time_end;
        L.max_step = c.max_step; L.cfl_dimension = c.cfl_dimension; L.cfl_degree_factor = c.cfl_degree_factor;
        grid = dim3((c.nx + 30) / 31, (c.ny + NW * CPT - 1) / (NW * CPT), 1);
        block = dim3(32 * NW, 1, 1);
    }

    void layout(ScratchLayout& S) const override {
        const size_t pb = size_t(L.plane) * sizeof(float);
        const int nblk = std::max(int(grid.x * grid.y), kReduceBlocksMax);
        S.state = 0;
        S.partials = align_up(sizeof(zfv::DevState));
        S.log = S.partials + align_up(sizeof(double) * 2 * nblk);
        S.stage = S.log + align_up(sizeof(double) * 3 * kLogCap);    // inc1: 3 planes
        S.alt = S.stage + align_up(pb * 3);                           // ping-pong: 3 planes
        S.lo = S.alt + align_up(pb * 3);                               // remainders: 3 planes
        S.total = S.lo + align_up(pb * 3);
    }

    template <int M, bool W, bool I>
    static auto kfn() { return &k32s_stage<2, M, W, I, NW, CPT>; }

    template <int O, bool W, bool I>
    int setup_combo() { return 0; }

    template <class F>
    int with_combo(F&& f) {
        const zfv_config& c = h->cfg;
        const bool wb = c.well_balanced != 0, im = c.implicit_source != 0;
        if (c.spatial_order == 2) {
            if (wb) return im ? f.template operator()<2, true, true>() : f.template operator()<2, true, false>();
            return im ? f.template operator()<2, false, true>() : f.template operator()<2, false, false>();
        }
        if (wb) return im ? f.template operator()<1, true, true>() : f.template operator()<1, true, false>();
        return im ? f.template operator()<1, false, true>() : f.template operator()<1, false, false>();
    }

    struct SetupF {
        Runner32* r;
        template <int O, bool W, bool I> int operator()() { return r->template setup_combo<O, W, I>(); }
    };
    int setup() override {
        if (h->cfg.spatial_order == 1) {
            // order 1 (PCM) is a single forward-Euler stage in the reference
            // (ZoomyAmr.cpp:677-678); the FP32 form implements the SSP-RK2 path
            return fail(-2, "zfv_create: the FP32 form implements spatial_order 2 only");
        }
        if (h->cfg.positivity_mood) return fail(-2, "zfv_create: the FP32 form does not implement MOOD");
        return with_combo(SetupF{this});
    }

    zfv::DevState* st(char* s) const { return reinterpret_cast<zfv::DevState*>(s + h->lay.state); }
    double* partials(char* s) const { return reinterpret_cast<double*>(s + h->lay.partials); }
    double* log3(char* s) const { return reinterpret_cast<double*>(s + h->lay.log); }
    float* inc(char* s) const { return reinterpret_cast<float*>(s + h->lay.stage); }
    float* alt(char* s) const { return reinterpret_cast<float*>(s + h->lay.alt); }
    float* lo(char* s) const { return reinterpret_cast<float*>(s + h->lay.lo); }
    const float* lo(const char* s) const { return reinterpret_cast<const float*>(s + h->lay.lo); }

    int reduce_blocks() const {
        long long need = (L.plane + kReduceNT - 1) / kReduceNT;
        return int(need < kReduceBlocksMax ? (need > 0 ? need : 1) : kReduceBlocksMax);
    }

    int begin(const void* Q, const void* A, char* scratch, cudaStream_t s) override {
        zfv::k_begin<<<1, 1, 0, s>>>(st(scratch), L);
        k32_reduce<kReduceNT, 0><<<reduce_blocks(), kReduceNT, 0, s>>>(
            (const float*)Q, lo(scratch), (const double*)A, n_aux, L, st(scratch), partials(scratch));
        return cuda_check(cudaGetLastError(), "zfv_begin (fp32) launch");
    }
    int update_state(void*, void*, double, cudaStream_t) override {
        return fail(-2, "zfv_update_state: validation entry of the FP64 form only");
    }
    int compute_dt(const void* Q, const void* A, char* scratch, cudaStream_t s) override {
        return fail(-2, "zfv_compute_dt: validation entry of the FP64 form only");
    }
    int total_mass(const void* Q, char* scratch, cudaStream_t s) override {
        k32_reduce<kReduceNT, 1><<<reduce_blocks(), kReduceNT, 0, s>>>(
            (const float*)Q, lo(scratch), nullptr, n_aux, L, st(scratch), partials(scratch));
        return cuda_check(cudaGetLastError(), "zfv_total_mass (fp32) launch");
    }
    int rhs(const void*, void*, double, cudaStream_t) override {
        return fail(-2, "zfv_rhs: validation entry of the FP64 form only");
    }
    int fill_ghosts(const void*, const void*, void*, void*, double, cudaStream_t) override {
        return fail(-2, "zfv_fill_ghosts: validation entry of the FP64 form only");
    }

    template <int O, bool W, bool I>
    void launch_step(float* Qf, float* Xs, float* Ys, char* scratch, cudaStream_t s) {
        const float* bedp = Qf;
        auto k1 = kfn<S1, W, I>();
        k1<<<grid, block, 0, s>>>(bedp, Xs, nullptr, inc(scratch), nullptr, nullptr, L,
                                  st(scratch), partials(scratch), log3(scratch), kLogCap);
        auto k2 = kfn<S2, W, I>();
        k2<<<grid, block, 0, s>>>(bedp, Xs, inc(scratch), nullptr, Ys, lo(scratch), L,
                                  st(scratch), partials(scratch), log3(scratch), kLogCap);
    }

    struct EvolveF {
        Runner32* r; float* Qf; char* scratch; int n; cudaStream_t s;
        template <int O, bool W, bool I> int operator()() {
            const long long plane = r->L.plane;
            float* A = Qf + plane;            // eta, hu, hv planes of the caller's Q
            float* B = r->alt(scratch);
            bool in_b = false;
            for (int k = 0; k < n; ++k) {
                r->template launch_step<O, W, I>(Qf, in_b ? B : A, in_b ? A : B, scratch, s);
                in_b = !in_b;
            }
            if (in_b) {
                cudaError_t e = cudaMemcpyAsync(A, B, size_t(plane) * 3 * sizeof(float),
                                                cudaMemcpyDeviceToDevice, s);
                if (e != cudaSuccess) return cuda_check(e, "zfv_evolve (fp32) copy-back");
            }
            return cuda_check(cudaGetLastError(), "zfv_evolve (fp32) launch");
        }
    };

    int evolve(void* Qv, void* Av, char* scratch, int n, cudaStream_t s) override {
        int rc = with_combo(EvolveF{this, (float*)Qv, scratch, n, s});
        if (rc) return rc;
        const int nb = int((L.plane + 255) / 256);
        k32_aux<<<nb, 256, 0, s>>>((const float*)Qv, lo(scratch), (double*)Av, L.plane, n_aux, L.epsd);
        return cuda_check(cudaGetLastError(), "zfv_evolve (fp32) aux launch");
    }

    int state_import(const double* Q64, void* Q, char* scratch, cudaStream_t s) override {
        const int nb = int((L.plane + 255) / 256);
        k32_import<<<nb, 256, 0, s>>>(Q64, (float*)Q, lo(scratch), L.plane);
        return cuda_check(cudaGetLastError(), "zfv_state_import (fp32) launch");
    }
    int state_export(const void* Q, const char* scratch, double* Q64, cudaStream_t s) override {
        const int nb = int((L.plane + 255) / 256);
        k32_export<<<nb, 256, 0, s>>>((const float*)Q, lo(scratch), Q64, L.plane);
        return cuda_check(cudaGetLastError(), "zfv_state_export (fp32) launch");
    }
};

}  // namespace zfv32

namespace zfvi {
Runner* make_runner_fp32_swe2d(zfv_handle* h) { return new zfv32::Runner32<4, 16>(h); }
}
