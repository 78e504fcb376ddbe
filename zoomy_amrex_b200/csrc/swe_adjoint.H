// Hand-written reverse mode of one SSP-RK2 stage of the 2-D shallow-water
// scheme (FP64): the per-face reconstruction / hydrostatic reconstruction /
// flux / fluctuation map of make_rhs.H:31-131 with the SWE model functions of
// models/swe.H, and the point-implicit Manning update of make_rhs.H:429-509.
//
// Conventions
//  * A face's stencil is c[k][n], k = 0..3 the cells iL-1, iL, iR, iR+1 along
//    the normal D, n = 0..3 the components (b, h, hu, hv).
//  * A face's outputs are o[11] = (flux h, hu, hv; D+ h, hu, hv; D- h, hu, hv;
//    h*_L, h*_R): the same numbers the forward kernels keep per face (the bed
//    row of flux and D+- is identically zero).
//  * Non-smooth points take the subgradient of the branch the forward code
//    takes: minmod's selected argument (0 on a sign change), max's selected
//    argument (amrex::max picks its first argument on ties), 0 for the
//    derivative of sqrt(g max(h, 0)) and |x| at 0.
//  * The implicit update q = q* + dq with (I - dt J(q*)) dq = dt S(q*), hv
//    (the stage aux 1/h) held fixed inside S and J, is differentiated by the
//    implicit-function theorem: mu = A^{-T} lam, then every input theta gets
//    dt mu . d(S + J dq)/dtheta with dq held fixed (second derivatives of the
//    Manning law written out below).
#pragma once
#include <cmath>
#include "AMReX_Algorithm.H"
#include "zb_portable_math.H"

#ifdef __CUDACC__
#  define ZADJ_UNROLL _Pragma("unroll")
#  define ZADJ_INLINE __forceinline__
#else
#  define ZADJ_UNROLL
#  define ZADJ_INLINE inline
#endif

#ifndef PORTABLE_FN
#  ifdef __CUDACC__
#    define PORTABLE_FN __host__ __device__
#  else
#    define PORTABLE_FN
#  endif
#endif

namespace zadj {

template <class R>
struct SweP {
    R g, ex, ey, nm, hfloor, eps;
};

constexpr int kFaceOut = 11;

// minmod with the index of the selected argument (0: none, 1: a, 2: b).
template <class R>
PORTABLE_FN ZADJ_INLINE R mm_sel(R a, R b, int& s) {
    if (a * b <= R(0)) { s = 0; return R(0); }
    if (std::fabs(a) < std::fabs(b)) { s = 1; return a; }
    s = 2;
    return b;
}

// models/swe.H hinv_of and its derivative.
template <class R>
PORTABLE_FN ZADJ_INLINE R hinv(R h, R eps) {
    const R h2 = h * h;
    const R x0 = h2 * h2;
    return std::sqrt(R(2)) * h / std::sqrt(x0 + amrex::max(x0, eps));
}
template <class R>
PORTABLE_FN ZADJ_INLINE R dhinv(R h, R eps) {
    const R h2 = h * h;
    const R x0 = h2 * h2;
    const bool big = !(x0 < eps);          // amrex::max(x0, eps) takes x0
    const R D = x0 + (big ? x0 : eps);
    if (!(D > R(0))) return R(0);
    const R den = std::sqrt(D);
    const R dD = R(4) * h * h2 * (big ? R(2) : R(1));
    return std::sqrt(R(2)) / den * (R(1) - h * dD / (R(2) * D));
}

// 1 / sqrt(x): the device's reciprocal square root (at most 1 ulp off in
// FP64), 1 / sqrt on the host.
template <class R>
PORTABLE_FN ZADJ_INLINE R rsqrt_of(R x) {
#ifdef __CUDA_ARCH__
    return ::rsqrt(x);
#else
    return R(1) / std::sqrt(x);
#endif
}

// dhinv from one reciprocal square root: with D = x0 + max(x0, eps),
// dhinv = sqrt2 D^(-1/2) (1 - h D' / (2 D)). A derivative coefficient only.
template <class R>
PORTABLE_FN ZADJ_INLINE R dhinv_r(R h, R eps) {
    const R h2 = h * h;
    const R x0 = h2 * h2;
    const bool big = !(x0 < eps);
    const R D = x0 + (big ? x0 : eps);
    if (!(D > R(0))) return R(0);
    const R r = rsqrt_of(D);
    const R dD = R(4) * h * h2 * (big ? R(2) : R(1));
    return std::sqrt(R(2)) * r * (R(1) - R(0.5) * h * dD * (r * r));
}

// hinv from one reciprocal square root, sqrt2 h D^(-1/2) (within an ulp or
// two of hinv): the face reverse's coefficient. The only branch it feeds is
// the Rusanov speed's max(evL, evR), which it can turn only where the two
// speeds agree to an ulp without being equal (equal inputs still give equal
// speeds).
template <class R>
PORTABLE_FN ZADJ_INLINE R hinv_r(R h, R eps) {
    const R h2 = h * h;
    const R x0 = h2 * h2;
    return std::sqrt(R(2)) * h * rsqrt_of(x0 + amrex::max(x0, eps));
}

// Rounded product and sum that the compiler may not fuse (the forward
// kernels are built without contraction).
template <class R>
PORTABLE_FN ZADJ_INLINE R mul_rn(R a, R b) {
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
template <class R>
PORTABLE_FN ZADJ_INLINE R add_rn(R a, R b) {
#ifdef __CUDA_ARCH__
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}

// A face side's Rusanov speed |m_n hinv(h)| + sqrt(g max(h, 0)) in the
// forward's own operations (make_rhs.H:77-131 with the model's eigenvalue):
// qh, qm the reconstructed depth and normal momentum, h the depth the flux
// sees (h* with WB, where m = qm (h* / qh)).
template <bool WB, class R>
PORTABLE_FN ZADJ_INLINE R speed_fwd(R qh, R h, R qm, R g, R eps) {
    R m = qm;
    if constexpr (WB) m = mul_rn(qm, (qh > R(0)) ? h / qh : R(0));
    const R h2 = mul_rn(h, h);
    const R x0 = mul_rn(h2, h2);
    const R hi = mul_rn(std::sqrt(R(2)), h) / std::sqrt(add_rn(x0, amrex::max(x0, eps)));
    return add_rn(std::fabs(mul_rn(m, hi)), std::sqrt(mul_rn(g, amrex::max(h, R(0)))));
}

template <class R>
PORTABLE_FN ZADJ_INLINE R sgn(R x) { return (x > R(0)) ? R(1) : ((x < R(0)) ? R(-1) : R(0)); }

// Forward face map (the values eval_face produces for SWE2D).
template <int D, bool WB, class R>
PORTABLE_FN ZADJ_INLINE void face_fwd(const R c[4][4], SweP<R> const& p, R o[kFaceOut]) {
    R qL[4], qR[4];
    ZADJ_UNROLL
    for (int n = 0; n < 4; ++n) {
        int s;
        const R gL = mm_sel(c[1][n] - c[0][n], c[2][n] - c[1][n], s);
        const R gR = mm_sel(c[2][n] - c[1][n], c[3][n] - c[2][n], s);
        qL[n] = c[1][n] + R(0.5) * gL;
        qR[n] = c[2][n] - R(0.5) * gR;
    }
    R hL = qL[1], hR = qR[1];
    R mL[2] = {qL[2], qL[3]}, mR[2] = {qR[2], qR[3]};
    R bL = qL[0], bR = qR[0];
    if constexpr (WB) {
        const R bf = amrex::max(qL[0], qR[0]);
        const R hsL = amrex::max(R(0), qL[1] + qL[0] - bf);
        const R hsR = amrex::max(R(0), qR[1] + qR[0] - bf);
        const R sL = (qL[1] > R(0)) ? hsL / qL[1] : R(0);
        const R sR = (qR[1] > R(0)) ? hsR / qR[1] : R(0);
        mL[0] *= sL; mL[1] *= sL; mR[0] *= sR; mR[1] *= sR;
        hL = hsL; hR = hsR; bL = bf; bR = bf;
    }
    const R g = p.g;
    const R hiL = hinv(hL, p.eps), hiR = hinv(hR, p.eps);
    R FL[3], FR[3];
    FL[0] = mL[D]; FR[0] = mR[D];
    ZADJ_UNROLL
    for (int k = 0; k < 2; ++k) {
        FL[1 + k] = mL[k] * mL[D] * hiL + ((k == D) ? R(0.5) * g * hL * hL : R(0));
        FR[1 + k] = mR[k] * mR[D] * hiR + ((k == D) ? R(0.5) * g * hR * hR : R(0));
    }
    const R evL = std::fabs(mL[D] * hiL) + std::sqrt(g * amrex::max(hL, R(0)));
    const R evR = std::fabs(mR[D] * hiR) + std::sqrt(g * amrex::max(hR, R(0)));
    const R s = amrex::max(evL, evR);
    const R db = bR - bL;
    const R Bn = g * (R(0.5) * (hL + hR));
    const R dq[3] = {hR - hL, mR[0] - mL[0], mR[1] - mL[1]};
    ZADJ_UNROLL
    for (int n = 0; n < 3; ++n) {
        o[n] = R(0.5) * (FL[n] + FR[n]);
        const R bdq = (n == 1 + D) ? Bn * db : R(0);
        o[3 + n] = R(0.5) * bdq + R(0.5) * s * dq[n];
        o[6 + n] = R(0.5) * bdq - R(0.5) * s * dq[n];
    }
    o[9] = hL;
    o[10] = hR;
}

// Reverse face map: lc[k][n] += (d o / d c[k][n])^T lo. The well-balancing
// bed source enters a cell as +-0.5 g h*^2: its adjoint weights are passed as
// wA, wB (lo[9] += wA h*_L, lo[10] += wB h*_R, the derivative of 0.5 g h^2
// being g h), since h*_L, h*_R are only known inside.
template <int D, bool WB, class R>
PORTABLE_FN ZADJ_INLINE void face_rev(const R c[4][4], SweP<R> const& p, const R lo[kFaceOut],
                                 R wA, R wB, R lc[4][4]) {
    // -- forward, keeping what the reverse needs
    R qL[4], qR[4];
    int sLsel[4], sRsel[4];
    ZADJ_UNROLL
    for (int n = 0; n < 4; ++n) {
        const R gL = mm_sel(c[1][n] - c[0][n], c[2][n] - c[1][n], sLsel[n]);
        const R gR = mm_sel(c[2][n] - c[1][n], c[3][n] - c[2][n], sRsel[n]);
        qL[n] = c[1][n] + R(0.5) * gL;
        qR[n] = c[2][n] - R(0.5) * gR;
    }
    R hL = qL[1], hR = qR[1];
    R mL[2] = {qL[2], qL[3]}, mR[2] = {qR[2], qR[3]};
    R bL = qL[0], bR = qR[0];
    R bf = 0, tL = 0, tR = 0, hsL = 0, hsR = 0, sL = 1, sR = 1, iqL = 0, iqR = 0;
    if constexpr (WB) {
        bf = amrex::max(qL[0], qR[0]);
        tL = qL[1] + qL[0] - bf;
        tR = qR[1] + qR[0] - bf;
        hsL = amrex::max(R(0), tL);
        hsR = amrex::max(R(0), tR);
        // iq = 1 / q_h; s = h* iq (the forward divides: s is within an ulp
        // of the forward's, and the branches below depend on it only through
        // the Rusanov speed's max)
        iqL = (qL[1] > R(0)) ? R(1) / qL[1] : R(0);
        iqR = (qR[1] > R(0)) ? R(1) / qR[1] : R(0);
        sL = hsL * iqL;
        sR = hsR * iqR;
        mL[0] *= sL; mL[1] *= sL; mR[0] *= sR; mR[1] *= sR;
        hL = hsL; hR = hsR; bL = bf; bR = bf;
    }
    const R g = p.g;
    const R hiL = hinv_r(hL, p.eps), hiR = hinv_r(hR, p.eps);
    const R uL = mL[D] * hiL, uR = mR[D] * hiR;
    // c = sqrt(g h) exactly as the forward forms it; dc/dh = g r / 2 with
    // r = (g h)^(-1/2)
    const R ghL = mul_rn(g, amrex::max(hL, R(0))), ghR = mul_rn(g, amrex::max(hR, R(0)));
    const R cL = std::sqrt(ghL), cR = std::sqrt(ghR);
    const R rcL = (ghL > R(0)) ? rsqrt_of(ghL) : R(0), rcR = (ghR > R(0)) ? rsqrt_of(ghR) : R(0);
    const R evL = std::fabs(uL) + cL, evR = std::fabs(uR) + cR;
    bool pickR = evL < evR;                // amrex::max(evL, evR)
    const R aL = std::fabs(uL), aR = std::fabs(uR);
#ifdef ZADJ_FORWARD_BRANCHES
    // test build: every face recomputes both speeds with the forward's
    // operations (the near-tie rule below must give the same branches)
    constexpr bool kTieRule = false;
    pickR = speed_fwd<WB>(qL[1], hL, qL[2 + D], g, p.eps) < speed_fwd<WB>(qR[1], hR, qR[2 + D], g, p.eps);
#else
    constexpr bool kTieRule = true;
#endif
    if (kTieRule && std::fabs(evL - evR) <= R(1e-13) * (aL + aR) + R(1e-15) * (evL + evR)) {
        // Near a tie the branch is decided as the forward decides it. c is
        // the forward's and |u| is within 1e-13 relative of the forward's
        // |u| (a few ulps), so each forward speed fl(|u| + c) lies between
        // the sums of c with |u| -+ 1e-13 |u|: where those agree (always for
        // a side with |u| far below an ulp of c, as in water nearly at rest)
        // it is known exactly.
        const R loL = (aL - R(1e-13) * aL) + cL, upL = (aL + R(1e-13) * aL) + cL;
        const R loR = (aR - R(1e-13) * aR) + cR, upR = (aR + R(1e-13) * aR) + cR;
        if (loL == upL && loR == upR) {
            pickR = loL < loR;
        } else {
            // else from the forward's own arithmetic: equal speeds where both
            // sides' inputs agree (a mirrored wall face; the forward keeps
            // evL), else the speeds recomputed as the forward computes them
            const R nL = qL[2 + D], nR = qR[2 + D];
            const bool same = hL == hR && qL[1] == qR[1] && std::fabs(nL) == std::fabs(nR);
            pickR = !same && speed_fwd<WB>(qL[1], hL, nL, g, p.eps) < speed_fwd<WB>(qR[1], hR, nR, g, p.eps);
        }
    }
    const R s = pickR ? evR : evL;
    const R db = bR - bL;
    const R Bn = g * (R(0.5) * (hL + hR));
    const R dq[3] = {hR - hL, mR[0] - mL[0], mR[1] - mL[1]};

    // -- reverse
    R lhL = lo[9] + wA * hL, lhR = lo[10] + wB * hR;
    R lmL[2] = {0, 0}, lmR[2] = {0, 0};
    R lbL = 0, lbR = 0, ls = 0, lhiL = 0, lhiR = 0;
    ZADJ_UNROLL
    for (int n = 0; n < 3; ++n) {
        const R lp = lo[3 + n], lm = lo[6 + n];
        ls += R(0.5) * dq[n] * (lp - lm);
        const R ldq = R(0.5) * s * (lp - lm);
        if (n == 0) { lhR += ldq; lhL -= ldq; }
        else { lmR[n - 1] += ldq; lmL[n - 1] -= ldq; }
        if (n == 1 + D) {
            const R lbdq = R(0.5) * (lp + lm);
            const R lBn = lbdq * db;
            const R ldb = lbdq * Bn;
            lhL += R(0.5) * g * lBn;
            lhR += R(0.5) * g * lBn;
            lbR += ldb;
            lbL -= ldb;
        }
        // flux: o[n] = 0.5 (FL[n] + FR[n])
        const R lF = R(0.5) * lo[n];
        if (n == 0) { lmL[D] += lF; lmR[D] += lF; }
        else {
            const int k = n - 1;
            lmL[k] += lF * mL[D] * hiL; lmL[D] += lF * mL[k] * hiL; lhiL += lF * mL[k] * mL[D];
            lmR[k] += lF * mR[D] * hiR; lmR[D] += lF * mR[k] * hiR; lhiR += lF * mR[k] * mR[D];
            if (k == D) { lhL += lF * g * hL; lhR += lF * g * hR; }
        }
    }
    // s = max(evL, evR), ev = |m_D hi| + sqrt(g max(h, 0))
    {
        const R lev = ls;
        if (pickR) {
            const R lu = sgn(uR) * lev;
            lmR[D] += lu * hiR; lhiR += lu * mR[D];
            if (hR > R(0)) lhR += lev * g * R(0.5) * rcR;
        } else {
            const R lu = sgn(uL) * lev;
            lmL[D] += lu * hiL; lhiL += lu * mL[D];
            if (hL > R(0)) lhL += lev * g * R(0.5) * rcL;
        }
    }
    lhL += lhiL * dhinv_r(hL, p.eps);
    lhR += lhiR * dhinv_r(hR, p.eps);

    // hydrostatic reconstruction
    R lqL[4], lqR[4];
    if constexpr (WB) {
        // m = q_m * s, h = hs, b = bf
        R lsL = lmL[0] * qL[2] + lmL[1] * qL[3];
        R lsR = lmR[0] * qR[2] + lmR[1] * qR[3];
        lqL[2] = lmL[0] * sL; lqL[3] = lmL[1] * sL;
        lqR[2] = lmR[0] * sR; lqR[3] = lmR[1] * sR;
        R lhsL = lhL, lhsR = lhR;
        lqL[1] = 0; lqR[1] = 0;
        if (qL[1] > R(0)) { lhsL += lsL * iqL; lqL[1] -= lsL * sL * iqL; }
        if (qR[1] > R(0)) { lhsR += lsR * iqR; lqR[1] -= lsR * sR * iqR; }
        const R ltL = (R(0) < tL) ? lhsL : R(0);
        const R ltR = (R(0) < tR) ? lhsR : R(0);
        R lbf = lbL + lbR - ltL - ltR;
        lqL[1] += ltL; lqL[0] = ltL;
        lqR[1] += ltR; lqR[0] = ltR;
        if (qL[0] < qR[0]) lqR[0] += lbf; else lqL[0] += lbf;
    } else {
        lqL[0] = lbL; lqR[0] = lbR;
        lqL[1] = lhL; lqR[1] = lhR;
        lqL[2] = lmL[0]; lqL[3] = lmL[1];
        lqR[2] = lmR[0]; lqR[3] = lmR[1];
    }
    // MUSCL / minmod
    ZADJ_UNROLL
    for (int n = 0; n < 4; ++n) {
        lc[1][n] += lqL[n];
        const R lgL = R(0.5) * lqL[n];
        if (sLsel[n] == 1) { lc[1][n] += lgL; lc[0][n] -= lgL; }
        else if (sLsel[n] == 2) { lc[2][n] += lgL; lc[1][n] -= lgL; }
        lc[2][n] += lqR[n];
        const R lgR = -R(0.5) * lqR[n];
        if (sRsel[n] == 1) { lc[2][n] += lgR; lc[1][n] -= lgR; }
        else if (sRsel[n] == 2) { lc[3][n] += lgR; lc[2][n] -= lgR; }
    }
}

// Manning friction and its Jacobian on the momentum block, hv fixed.
template <class R>
struct Manning {
    R k, dk_dh, ic, S[2], J[2][2];
};
template <class R>
PORTABLE_FN ZADJ_INLINE Manning<R> manning(R h, R mx, R my, R hv, SweP<R> const& p) {
    Manning<R> M;
    const R m = amrex::max(h, p.hfloor);
    M.ic = zb::inv_cbrt_pos(m);
    M.k = p.g * p.nm * p.nm * M.ic;
    const R heav = (h - p.hfloor > R(0)) ? R(1) : ((h - p.hfloor < R(0)) ? R(0) : R(0.5));
    M.dk_dh = -M.k * (M.ic * M.ic * M.ic) * R(1.0 / 3.0) * heav;
    const R ux = mx * hv, uy = my * hv;
    const R s2 = ux * ux + uy * uy;
    const R rsp = (s2 > R(0)) ? rsqrt_of(s2) : R(0);   // 1 / |u|
    const R sp = s2 * rsp;                              // |u|
    M.S[0] = p.g * p.ex * h - M.k * ux * sp;
    M.S[1] = p.g * p.ey * h - M.k * uy * sp;
    const R dsx = ux * hv * rsp, dsy = uy * hv * rsp;
    M.J[0][0] = -M.k * (hv * sp + ux * dsx);
    M.J[0][1] = -M.k * (ux * dsy);
    M.J[1][0] = -M.k * (uy * dsx);
    M.J[1][1] = -M.k * (hv * sp + uy * dsy);
    return M;
}

// Forward implicit update of the momenta (the 2x2 block the reference's 4x4
// elimination reduces to: the bed and depth rows of J and S are zero).
// Returns false when the explicit fallback of make_rhs.H:501-508 is taken.
template <class R>
PORTABLE_FN ZADJ_INLINE bool implicit_fwd(R h, R mx, R my, R hv, R dt, SweP<R> const& p, R dq[2]) {
    const Manning<R> M = manning(h, mx, my, hv, p);
    const R a = R(1) - dt * M.J[0][0], b = -dt * M.J[0][1];
    const R c = -dt * M.J[1][0], d = R(1) - dt * M.J[1][1];
    const R det = a * d - b * c;
    const R r0 = dt * M.S[0], r1 = dt * M.S[1];
    if (std::fabs(det) > R(0) && std::isfinite(det)) {
        dq[0] = (r0 * d - b * r1) / det;
        dq[1] = (a * r1 - c * r0) / det;
        if (std::isfinite(dq[0]) && std::isfinite(dq[1])) return true;
    }
    dq[0] = std::isfinite(r0) ? r0 : R(0);
    dq[1] = std::isfinite(r1) ? r1 : R(0);
    return false;
}

// Reverse of q_out = q* + dq(q*, hv, n_m, dt) on one cell. lam: adjoint of
// q_out's momenta (the h and b rows pass through unchanged). Adds to
// lq[1..3] (h, hu, hv of q*), lhv, lnm, ldt.
template <class R>
PORTABLE_FN ZADJ_INLINE void implicit_rev(R h, R mx, R my, R hv, R dt, SweP<R> const& p, const R lam[2],
                                     R lq[4], R& lhv, R& lnm, R& ldt) {
    const Manning<R> M = manning(h, mx, my, hv, p);
    const R a = R(1) - dt * M.J[0][0], b = -dt * M.J[0][1];
    const R c = -dt * M.J[1][0], d = R(1) - dt * M.J[1][1];
    const R det = a * d - b * c;
    R dq[2] = {0, 0}, mu[2];
    bool ok = false;
    R rdet = R(0);
    if (std::fabs(det) > R(0) && std::isfinite(det)) {
        const R r0 = dt * M.S[0], r1 = dt * M.S[1];
        rdet = R(1) / det;
        dq[0] = (r0 * d - b * r1) * rdet;
        dq[1] = (a * r1 - c * r0) * rdet;
        ok = std::isfinite(dq[0]) && std::isfinite(dq[1]);
    }
    if (ok) {
        // A^T mu = lam, A = [[a, b], [c, d]]
        mu[0] = (lam[0] * d - c * lam[1]) * rdet;
        mu[1] = (a * lam[1] - b * lam[0]) * rdet;
    } else {       // explicit fallback: q_out = q* + dt S (dq = 0 in the terms below)
        mu[0] = lam[0]; mu[1] = lam[1];
        dq[0] = dq[1] = R(0);
        if (!std::isfinite(dt * M.S[0]) || !std::isfinite(dt * M.S[1])) return;
    }
    // phi = S + J dq = g e h - k Psi(u, w), u = hv m, w = hv dq,
    // Psi = |u| u + |u| w + u (u.w)/|u|
    const R ux = mx * hv, uy = my * hv;
    const R wx = hv * dq[0], wy = hv * dq[1];
    const R s2 = ux * ux + uy * uy;
    R Psi[2] = {0, 0}, lu[2] = {0, 0}, lw[2] = {0, 0};
    const R k = M.k;
    if (s2 > R(0)) {
        const R rs = rsqrt_of(s2);          // 1 / |u|
        const R sp = s2 * rs;
        const R ex = ux * rs, ey = uy * rs;
        const R uw = ux * wx + uy * wy;
        const R uwr = uw * rs, umr = (ux * mu[0] + uy * mu[1]) * rs;
        Psi[0] = sp * ux + sp * wx + ux * uwr;
        Psi[1] = sp * uy + sp * wy + uy * uwr;
        const R umu = ux * mu[0] + uy * mu[1];
        const R wmu = wx * mu[0] + wy * mu[1];
        // (dPsi/du)^T mu
        const R gu0 = sp * mu[0] + ex * umu + ex * wmu + uwr * mu[0] + wx * umr - ex * uwr * umr;
        const R gu1 = sp * mu[1] + ey * umu + ey * wmu + uwr * mu[1] + wy * umr - ey * uwr * umr;
        // (dPsi/dw)^T mu = (|u| I + u e^T)^T mu
        const R gw0 = sp * mu[0] + ex * umu;
        const R gw1 = sp * mu[1] + ey * umu;
        lu[0] = -k * dt * gu0; lu[1] = -k * dt * gu1;
        lw[0] = -k * dt * gw0; lw[1] = -k * dt * gw1;
    }
    lq[1] += dt * (mu[0] * (p.g * p.ex - M.dk_dh * Psi[0]) + mu[1] * (p.g * p.ey - M.dk_dh * Psi[1]));
    lq[2] += hv * lu[0];
    lq[3] += hv * lu[1];
    lhv += mx * lu[0] + my * lu[1] + dq[0] * lw[0] + dq[1] * lw[1];
    // dk/dn_m = 2 g n_m ic
    lnm += -dt * R(2) * p.g * p.nm * M.ic * (mu[0] * Psi[0] + mu[1] * Psi[1]);
    // explicit dependence on dt: A dq = dt S -> d dq/d dt = A^{-1} (S + J dq)
    const R phi0 = M.S[0] + M.J[0][0] * dq[0] + M.J[0][1] * dq[1];
    const R phi1 = M.S[1] + M.J[1][0] * dq[0] + M.J[1][1] * dq[1];
    ldt += mu[0] * phi0 + mu[1] * phi1;
}

}  // namespace zadj
