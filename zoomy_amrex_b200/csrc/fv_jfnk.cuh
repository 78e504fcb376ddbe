// Global implicit source by Jacobian-free Newton-Krylov (the reference's
// solver.implicit_global, imex_solver.H:19-160), FP64.
//
// After a stage's flux update Q = Qexp (the stage kernel in MODE_X, which
// stops before the point-implicit source), the whole field solves
//     F(Q) = Q - Qexp - dt S(Q) = 0
// by Newton steps J delta = -F with restarted GMRES, J applied matrix-free as
//     J x = x - (dt / eps) (S(Qbase + eps x) - S(Qbase)),
//     eps = 1e-7 (1 + |Qbase|) / |x|                  (imex_solver.H:79-87)
// S is evaluated with the aux refreshed from the state (ComputeSourceField,
// imex_solver.H:21-58). The host drives the iteration (zoomy_fv.cu); these
// are its kernels.
//
// Vectors are the state rows the step evolves (rows n0 .. n_q-1; the static
// bed row of SWE is constant, so its F, J x and Newton update are identically
// zero), stored row after row: length N = (n_q - n0) * plane. Every reduction
// writes per-block partials that a one-block kernel sums in block order, so
// the iteration is deterministic.
#pragma once
#include "fv_device.cuh"

namespace zfv {
namespace jfnk {

constexpr int kNT = 256;         // threads per block of every kernel here
constexpr int kMaxDots = 32;     // vectors per multi-dot / multi-axpy launch

template <class Model>
__device__ __forceinline__ typename ModelTypes<Model>::VQ source_of(const typename ModelTypes<Model>::VQ& q,
                                                                    const typename ModelTypes<Model>::VP& p,
                                                                    const LevelParams<double, Model::n_parameters>& L,
                                                                    double time, int i, int j) {
    typename ModelTypes<Model>::VA a{};
    const auto X = cell_centre<Model, double>(L, i, j);
    a = Model::update_aux_variables(q, a, p, time, X);
    return Model::source(q, a, p, time, X);
}

// Block sum in a fixed order; thread 0 holds the result.
__device__ __forceinline__ double block_sum(double v, double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        v = red[0];
        for (int w = 1; w < kNT / 32; ++w) v += red[w];
    }
    return v;
}

// S = S(Q), F = Q - Qexp - dt S; partials[block] = sum of F^2 over the block
// (imex_solver.H:129-131). Q, Qexp, S, F: vectors (rows n0 ..); qbed: the
// state whose row 0 is the bed.
template <class Model>
__global__ void __launch_bounds__(kNT)
k_residual(const double* __restrict__ Q, const double* __restrict__ qbed, const double* __restrict__ Qexp,
           double* __restrict__ S, double* __restrict__ F, LevelParams<double, Model::n_parameters> L,
           const DevState* st, double* __restrict__ partials) {
    using T = ModelTypes<Model>;
    constexpr int nq = Model::n_dof_q, n0 = static_bed<Model>::value ? 1 : 0;
    __shared__ double red[kNT / 32];
    const double dt = *(volatile const double*)&st->dt;
    const double time = *(volatile const double*)&st->time;
    const long long pl = L.plane;
    const long long c = (long long)blockIdx.x * kNT + threadIdx.x;
    double f2 = 0.0;
    if (c < pl) {
        typename T::VP p;
        for (int k = 0; k < Model::n_parameters; ++k) p(k, 0) = L.p[k];
        typename T::VQ q;
        if constexpr (n0 == 1) q(0, 0) = qbed[c];
#pragma unroll
        for (int n = n0; n < nq; ++n) q(n, 0) = Q[(n - n0) * pl + c];
        const auto s = source_of<Model>(q, p, L, time, int(c % L.nx), int(c / L.nx));
#pragma unroll
        for (int n = n0; n < nq; ++n) {
            const long long e = (n - n0) * pl + c;
            const double f = (q(n, 0) - Qexp[e]) + (-dt) * s(n, 0);
            S[e] = s(n, 0);
            F[e] = f;
            f2 += f * f;
        }
    }
    const double b = block_sum(f2, red);
    if (threadIdx.x == 0) partials[blockIdx.x] = b;
}

// Ax = x - (dt / eps) (S(Qbase + eps x) - Sbase)  (ImpSrcOp::apply,
// imex_solver.H:79-89: LinComb(Ax, 1, x, -dt/eps, Spert), then
// Saxpy(Ax, dt/eps, Sbase)).
template <class Model>
__global__ void __launch_bounds__(kNT)
k_jvp(const double* __restrict__ Qbase, const double* __restrict__ qbed, const double* __restrict__ Sbase,
      const double* __restrict__ x, double eps, double* __restrict__ Ax,
      LevelParams<double, Model::n_parameters> L, const DevState* st) {
    using T = ModelTypes<Model>;
    constexpr int nq = Model::n_dof_q, n0 = static_bed<Model>::value ? 1 : 0;
    const double dt = *(volatile const double*)&st->dt;
    const double time = *(volatile const double*)&st->time;
    const long long pl = L.plane;
    const long long c = (long long)blockIdx.x * kNT + threadIdx.x;
    if (c >= pl) return;
    typename T::VP p;
    for (int k = 0; k < Model::n_parameters; ++k) p(k, 0) = L.p[k];
    typename T::VQ q;
    if constexpr (n0 == 1) q(0, 0) = qbed[c];
#pragma unroll
    for (int n = n0; n < nq; ++n) {
        const long long e = (n - n0) * pl + c;
        q(n, 0) = Qbase[e] + eps * x[e];
    }
    const auto s = source_of<Model>(q, p, L, time, int(c % L.nx), int(c / L.nx));
    const double a = dt / eps;
#pragma unroll
    for (int n = n0; n < nq; ++n) {
        const long long e = (n - n0) * pl + c;
        Ax[e] = (x[e] + (-a) * s(n, 0)) + a * Sbase[e];
    }
}

// partials[k * nblk + block] = sum over the block of w . V_k for k <
// gridDim.y (blockIdx.y = k; V_k = V + k * vstride); with self_last the last
// k is w . w instead.
static __global__ void __launch_bounds__(kNT)
k_dots(const double* __restrict__ w, const double* __restrict__ V, long long vstride, long long N,
       double* __restrict__ partials, int self_last) {
    __shared__ double red[kNT / 32];
    const double* v = (self_last && blockIdx.y == gridDim.y - 1) ? w : V + blockIdx.y * vstride;
    double s = 0.0;
    for (long long e = (long long)blockIdx.x * kNT + threadIdx.x; e < N; e += (long long)gridDim.x * kNT)
        s += w[e] * v[e];
    const double b = block_sum(s, red);
    if (threadIdx.x == 0) partials[(long long)blockIdx.y * gridDim.x + blockIdx.x] = b;
}

// out[k] = sum of partials[k * nblk + b] over b in order (one block per k).
static __global__ void __launch_bounds__(kNT)
k_sum_partials(const double* __restrict__ partials, int nblk, double* __restrict__ out) {
    __shared__ double red[kNT / 32];
    const double* p = partials + (long long)blockIdx.x * nblk;
    double s = 0.0;
    for (int b = threadIdx.x; b < nblk; b += kNT) s += p[b];
    const double t = block_sum(s, red);
    if (threadIdx.x == 0) out[blockIdx.x] = t;
}

struct Coefs {
    double c[kMaxDots];
};

// y = a y + sum_k coef_k V_k (k < nv; a = 1: accumulate).
static __global__ void __launch_bounds__(kNT)
k_combine(double* __restrict__ y, double a, const double* __restrict__ V, long long vstride, int nv, Coefs cf,
          long long N) {
    for (long long e = (long long)blockIdx.x * kNT + threadIdx.x; e < N; e += (long long)gridDim.x * kNT) {
        double v = (a == 1.0) ? y[e] : a * y[e];
        for (int k = 0; k < nv; ++k) v += cf.c[k] * V[k * vstride + e];
        y[e] = v;
    }
}

// dst = s * src
static __global__ void __launch_bounds__(kNT)
k_scale(double* __restrict__ dst, const double* __restrict__ src, double s, long long N) {
    for (long long e = (long long)blockIdx.x * kNT + threadIdx.x; e < N; e += (long long)gridDim.x * kNT)
        dst[e] = s * src[e];
}

// End of a step whose stages took the global implicit source: the Heun
// combine Q = 0.5 Q^n + 0.5 Q** (order 2, ZoomyAmr.cpp:665-675) or Q = Q**
// (order 1), the final UpdateState (:730) and the CFL / mass reduction that
// advances the run record (as the fused stage kernel's epilogue does).
template <class Model, class Numerics, bool HEUN>
__global__ void __launch_bounds__(kNT)
k_finish(const double* __restrict__ qss, double* __restrict__ Q, LevelParams<double, Model::n_parameters> L,
         DevState* st, double* __restrict__ partials, double* __restrict__ log3, int log_cap) {
    using T = ModelTypes<Model>;
    constexpr int nq = Model::n_dof_q, n0 = static_bed<Model>::value ? 1 : 0;
    __shared__ double red[2 * (kNT / 32)];
    if (*(volatile unsigned*)&st->flags & kFlagDone) return;
    const double dt = *(volatile double*)&st->dt;
    const double time = *(volatile double*)&st->time;
    const long long pl = L.plane;
    const long long c = (long long)blockIdx.x * kNT + threadIdx.x;
    double m_loc = 0.0, s_loc = 0.0;
    if (c < pl) {
        typename T::VP p;
        for (int k = 0; k < Model::n_parameters; ++k) p(k, 0) = L.p[k];
        typename T::VQ q;
        if constexpr (n0 == 1) q(0, 0) = Q[c];
#pragma unroll
        for (int n = n0; n < nq; ++n) {
            const double v = qss[(n - n0) * pl + c];
            q(n, 0) = HEUN ? 0.5 * Q[n * pl + c] + 0.5 * v : v;
        }
        typename T::VA a{};
        update_state_cell<Model, double>(q, a, p, L, time,
                                         cell_centre<Model, double>(L, int(c % L.nx), int(c / L.nx)));
#pragma unroll
        for (int n = n0; n < nq; ++n) Q[n * pl + c] = q(n, 0);
        m_loc = cell_max_inv<Model, Numerics, double>(q, a, p, L);
        s_loc = q(kIdxH, 0);
    }
    finish_step<kNT>(m_loc, s_loc, red, partials, log3, log_cap, st, L, dt, time, false);
}

}  // namespace jfnk
}  // namespace zfv
