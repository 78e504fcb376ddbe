// Definitions shared by the translation units of the FP32 chosen form
// (zoomy_fv32.cu and the per-strip-shape units zoomy_fv32_shape.cu): the
// level parameters, the FP32 helper arithmetic and the point-implicit
// Manning solve. The scheme itself is described in zoomy_fv32.cu.
#pragma once
#include <cuda_runtime.h>
#include "fv_kernels.cuh"
#include "swe.H"
#include "zb_portable_math.H"

namespace zfv32 {

struct Params {
    int nx, ny;
    long long plane;
    double dx, dy, plox, ploy;       // FP64 (reductions, dt)
    float fdx, fdy, rdx, rdy, rfdx, rfdy;
    float g, ex, ey, nm, hfloor, eps;
    float hwet;                      // above this depth h^4 > eps: the KP hinv is 1/h
    double gd, exd, eyd, nmd, hfloord, epsd;
    int bc_tag[4];
    double cfl, dtmin, dtmax, time_end;
    int max_step, cfl_dimension, cfl_degree_factor;
    // Ghost frame (AMR boxes): when set, the cells just outside the box are
    // read from this (nx+4) x (ny+4) x 4 array ([b, eta, hu, hv] planes, ring
    // filled by the caller before each stage, stage input already summed)
    // instead of mirrored from the box's own cells.
    const float* frame;
};

struct C4 { float b, e, u, v; };   // bed, surface eta = h + b, hu, hv

constexpr float kNearDry = 1.0e-3f;   // FP64 implicit solve below this depth

// minmod (make_rhs.H:9-13) as the median of (a, b, 0): 0 when the signs
// differ or either is 0, else the one of smaller magnitude; four min/max
// operations and no multiply or compare-and-select.
__device__ __forceinline__ float mm(float a, float b) {
    return fmaxf(fminf(a, b), fminf(fmaxf(a, b), 0.0f));
}

// Knuth's two-sum: s + e == a + b exactly (round-to-nearest, no contraction:
// the _rn intrinsics are never fused into FMAs).
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
    s = __fadd_rn(a, b);
    const float bp = __fsub_rn(s, a);
    const float ap = __fsub_rn(s, bp);
    e = __fadd_rn(__fsub_rn(a, ap), __fsub_rn(b, bp));
}

// Kurganov-Petrova desingularised 1/h (the model's update_aux_variables), FP32.
__device__ __forceinline__ float kp_hinv(float h, float eps) {
    const float h2 = h * h;
    const float x0 = h2 * h2;
    return 1.41421356237f * h * rsqrtf(x0 + fmaxf(x0, eps));
}
// The same, 1/h (one reciprocal) where every active lane's depth exceeds
// hwet (h^4 > eps), decided by a warp vote.
__device__ __forceinline__ float kp_hinv_w(float h, float eps, float hwet) {
    if (__all_sync(__activemask(), h > hwet)) return 1.0f / h;
    return kp_hinv(h, eps);
}
__device__ __forceinline__ double kp_hinv_d(double h, double eps) {
    const double h2 = h * h;
    const double x0 = h2 * h2;
    return 1.4142135623730951 * h / sqrt(x0 + fmax(x0, eps));
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

// A near-dry cell at rest with no source: u = v = 0 and no slope forcing
// (ex = ey = 0) or no depth. manning_implicit then returns exactly +0 in
// both rows (ux = uy = 0, sp = 0, det = 1 and x0 = 0 - (+-0) = +0), so the
// FP64 solve can be skipped: dry cells are a tenth of a wet/dry level, and a
// warp with one of them would otherwise run the FP64 path.
__device__ __forceinline__ bool rest_without_source(float h, float u, float v, const Params& L) {
    return u == 0.0f && v == 0.0f && (h == 0.0f || (L.exd == 0.0 && L.eyd == 0.0));
}

enum Mode { S1 = 1, S2 = 2 };

}  // namespace zfv32

