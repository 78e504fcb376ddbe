// FP32 chosen form: the paired-column warp sweep (sm_100 packed FP32).
//
// The same column sweep as fv32_sweep.cuh, with each lane holding TWO
// adjacent columns (A = x0-2+2L, B = A+1) and doing their arithmetic as
// float2 pairs through Blackwell's packed FP32 instructions (FADD2/FMUL2/FFMA2
// via __fadd2_rn/__fmul2_rn/__ffma2_rn): one instruction advances both
// columns' reconstruction, faces and update. A strip is 60 owned columns
// (lanes 1..30); lanes 0 and 31 hold the neighbour column pairs, and, unlike
// the one-column sweep, need no extra loads (the x-stencil of every face a
// lane evaluates lies inside the 64 columns the warp holds).
//
// Per row a lane
//   * reconstructs A and B in x (neighbours: lane-1's B, lane+1's A by shuffle)
//     and the next row in y (register window, as before),
//   * evaluates, packed, the x-faces left of A and between A and B, and the
//     y-faces above A and B,
//   * takes the face right of B from lane+1 (its face left of A),
//   * assembles, applies the point-implicit Manning update (packed; cells
//     below h = 1e-3 fall back to the per-cell FP64 solve) and writes.
// Loads and stores are float2 (8-byte) when the strip is interior and nx is
// even; otherwise per-element with the ghost-cell mirror of fetch().
#pragma once

namespace zfv32 {
namespace pk {

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 s2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
__device__ __forceinline__ float2 mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 neg(float2 a) { return f2(-a.x, -a.y); }
__device__ __forceinline__ float2 mm(float2 a, float2 b) { return f2(zfv32::mm(a.x, b.x), zfv32::mm(a.y, b.y)); }
__device__ __forceinline__ float2 fmax2(float2 a, float2 b) { return f2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }
__device__ __forceinline__ float2 fabs2(float2 a) { return f2(fabsf(a.x), fabsf(a.y)); }
__device__ __forceinline__ float2 sqrt2(float2 a) { return f2(sqrtf(a.x), sqrtf(a.y)); }
__device__ __forceinline__ float2 rsqrt2(float2 a) { return f2(rsqrtf(a.x), rsqrtf(a.y)); }

struct C42 { float2 b, e, u, v; };          // cells A, B: bed, eta, hu, hv
struct RS2 { float2 b, h, e, u, v; };       // reconstructed face states of A, B

// KP desingularised 1/h (the model's update_aux_variables), packed. Where
// every active lane's depths exceed hwet (h^4 > eps) the formula is 1/h:
// one reciprocal each, decided by a warp vote.
__device__ __forceinline__ float2 kp_hinv2(float2 h, const Params& L) {
    if (__all_sync(__activemask(), fminf(h.x, h.y) > L.hwet)) return f2(1.0f / h.x, 1.0f / h.y);
    const float2 h2 = mul(h, h);
    const float2 x0 = mul(h2, h2);
    return mul(mul(s2(1.41421356237f), h), rsqrt2(add(x0, fmax2(x0, s2(L.eps)))));
}

__device__ __forceinline__ void reconstruct2(const C42& m, const C42& c, const C42& p, RS2& lo, RS2& hi) {
    const float2 dbm = sub(c.b, m.b), dbp = sub(p.b, c.b);
    const float2 dem = sub(c.e, m.e), dep = sub(p.e, c.e);
    const float2 gb = mm(dbm, dbp);
    const float2 gh = mm(sub(dem, dbm), sub(dep, dbp));
    const float2 gu = mm(sub(c.u, m.u), sub(p.u, c.u));
    const float2 gv = mm(sub(c.v, m.v), sub(p.v, c.v));
    const float2 h = sub(c.e, c.b);
    const float2 half = s2(0.5f);
    const float2 hb = mul(half, gb), hh = mul(half, gh), he = mul(half, add(gh, gb));
    const float2 hu = mul(half, gu), hv = mul(half, gv);
    hi = RS2{add(c.b, hb), add(h, hh), add(c.e, he), add(c.u, hu), add(c.v, hv)};
    lo = RS2{sub(c.b, hb), sub(h, hh), sub(c.e, he), sub(c.u, hu), sub(c.v, hv)};
}

// What a face contributes to the balance of its two cells (make_rhs.H:346-399):
// the cell on its high side gets  l = f - D+ (- P(h*_R) in the momentum
// normal to the face, the WB bed source), the cell on its low side loses
// r = f + D- (- P(h*_L)); a cell's balance is l(low face) - r(high face).
// D+ and D- differ only in the sign of the Rusanov term for h (so l0 = r0)
// and in the bed term of the normal momentum, so 5 values describe a face.
struct FaceLR {
    float2 l0, l1, l2;
    float2 r1, r2;
};

// Two faces at once from their reconstructed left (a) / right (c) states.
template <int DIR, bool WB>
__device__ __forceinline__ FaceLR face2(RS2 a, RS2 c, const Params& L) {
    float2 db = s2(0.0f);
    float2 qL, qR;          // normal velocities of the face states
    if constexpr (WB) {
        const float2 bf = fmax2(a.b, c.b);
        const float2 hsL = fmax2(s2(0.0f), sub(a.e, bf)), hsR = fmax2(s2(0.0f), sub(c.e, bf));
        const float hs_min = fminf(fminf(hsL.x, hsL.y), fminf(hsR.x, hsR.y));
        const float h_min = fminf(fminf(a.h.x, a.h.y), fminf(c.h.x, c.h.y));
        if (__all_sync(__activemask(), hs_min > L.hwet && h_min > 0.0f)) {
            // every face depth wet: with r = 1/h the Audusse factor is
            // s = h* r and the normal velocity (s m_n) / h* is m_n r, so one
            // reciprocal per side serves both
            const float2 rL = f2(1.0f / a.h.x, 1.0f / a.h.y), rR = f2(1.0f / c.h.x, 1.0f / c.h.y);
            const float2 sL = mul(hsL, rL), sR = mul(hsR, rR);
            qL = mul((DIR == 0) ? a.u : a.v, rL);
            qR = mul((DIR == 0) ? c.u : c.v, rR);
            a.u = mul(a.u, sL); a.v = mul(a.v, sL); c.u = mul(c.u, sR); c.v = mul(c.v, sR);
        } else {
            const float2 sL = f2((a.h.x > 0.0f) ? __fdividef(hsL.x, a.h.x) : 0.0f,
                                 (a.h.y > 0.0f) ? __fdividef(hsL.y, a.h.y) : 0.0f);
            const float2 sR = f2((c.h.x > 0.0f) ? __fdividef(hsR.x, c.h.x) : 0.0f,
                                 (c.h.y > 0.0f) ? __fdividef(hsR.y, c.h.y) : 0.0f);
            a.u = mul(a.u, sL); a.v = mul(a.v, sL); c.u = mul(c.u, sR); c.v = mul(c.v, sR);
            qL = mul((DIR == 0) ? a.u : a.v, kp_hinv2(hsL, L));
            qR = mul((DIR == 0) ? c.u : c.v, kp_hinv2(hsR, L));
        }
        a.h = hsL; c.h = hsR;
    } else {
        db = sub(c.b, a.b);
        qL = mul((DIR == 0) ? a.u : a.v, kp_hinv2(a.h, L));
        qR = mul((DIR == 0) ? c.u : c.v, kp_hinv2(c.h, L));
    }
    const float2 g = s2(L.g), hg = s2(0.5f * L.g), half = s2(0.5f);
    const float2 unL = (DIR == 0) ? a.u : a.v, unR = (DIR == 0) ? c.u : c.v;
    const float2 pL = mul(mul(hg, a.h), a.h), pR = mul(mul(hg, c.h), c.h);
    float2 fuL, fvL, fuR, fvR;
    if constexpr (DIR == 0) {
        fuL = fma(a.u, qL, pL);  fvL = mul(a.v, qL);
        fuR = fma(c.u, qR, pR);  fvR = mul(c.v, qR);
    } else {
        fuL = mul(a.u, qL);  fvL = fma(a.v, qL, pL);
        fuR = mul(c.u, qR);  fvR = fma(c.v, qR, pR);
    }
    const float2 f0 = mul(half, add(unL, unR));
    const float2 f1 = mul(half, add(fuL, fuR));
    const float2 f2_ = mul(half, add(fvL, fvR));
    const float2 evL = add(fabs2(qL), sqrt2(mul(g, fmax2(a.h, s2(0.0f)))));
    const float2 evR = add(fabs2(qR), sqrt2(mul(g, fmax2(c.h, s2(0.0f)))));
    const float2 nhs = neg(mul(half, fmax2(evL, evR)));    // -(Rusanov speed) / 2
    const float2 dh = sub(c.h, a.h), du = sub(c.u, a.u), dv = sub(c.v, a.v);
    FaceLR F;
    F.l0 = fma(nhs, dh, f0);
    const float2 b1 = fma(nhs, du, f1), b2 = fma(nhs, dv, f2_);
    F.l1 = F.r1 = b1;
    F.l2 = F.r2 = b2;
    // the normal momentum: WB pressure terms P(h*_R) / P(h*_L), else the
    // path-conservative bed product g (hL + hR)/2 (bR - bL) in D+ and D-
    const float2 kl = WB ? pR : mul(mul(hg, mul(half, add(a.h, c.h))), db);
    const float2 kr = WB ? pL : neg(kl);
    if constexpr (DIR == 0) { F.l1 = sub(b1, kl); F.r1 = sub(b1, kr); }
    else                    { F.l2 = sub(b2, kl); F.r2 = sub(b2, kr); }
    return F;
}

// Stage input of the column pair (cA, cA+1) in row j.
template <int MODE, bool INTERIOR, bool VEC>
__device__ __forceinline__ C42 fetch2(const float* __restrict__ bed, const float* __restrict__ X,
                                      const float* __restrict__ inc, const Params& L, int cA, int j) {
    if constexpr (INTERIOR && VEC) {
        const long long pl = L.plane;
        const long long c = (long long)j * L.nx + cA;
        C42 q;
        q.b = __ldg(reinterpret_cast<const float2*>(bed + c));
        q.e = __ldg(reinterpret_cast<const float2*>(X + c));
        q.u = __ldg(reinterpret_cast<const float2*>(X + pl + c));
        q.v = __ldg(reinterpret_cast<const float2*>(X + 2 * pl + c));
        if constexpr (MODE == S2) {
            q.e = add(q.e, __ldg(reinterpret_cast<const float2*>(inc + c)));
            q.u = add(q.u, __ldg(reinterpret_cast<const float2*>(inc + pl + c)));
            q.v = add(q.v, __ldg(reinterpret_cast<const float2*>(inc + 2 * pl + c)));
        }
        return q;
    } else {
        const C4 a = fetch<MODE, INTERIOR>(bed, X, inc, L, cA, j);
        const C4 b = fetch<MODE, INTERIOR>(bed, X, inc, L, cA + 1, j);
        return C42{f2(a.b, b.b), f2(a.e, b.e), f2(a.u, b.u), f2(a.v, b.v)};
    }
}

// Packed point-implicit Manning update of two cells (FP32; the caller routes
// near-dry pairs to the per-cell solve). Explicit fallback per cell as in
// make_rhs.H:501-508.
__device__ __forceinline__ void manning_implicit2(float2 h, float2 u, float2 v, float2 hinv, float dt,
                                                  const Params& L, float2& du, float2& dv) {
    const float2 m = fmax2(h, s2(L.hfloor));
    // m^(-1/3) from the hardware log2 / exp2 (relative error ~1e-7)
    const float2 ic = f2(exp2f(-0.333333343f * __log2f(m.x)), exp2f(-0.333333343f * __log2f(m.y)));
    const float2 k = mul(s2(L.g * L.nm * L.nm), ic);
    const float2 ux = mul(u, hinv), uy = mul(v, hinv);
    const float2 sp = sqrt2(fma(ux, ux, mul(uy, uy)));
    const float2 Su = sub(mul(s2(L.g * L.ex), h), mul(mul(k, ux), sp));
    const float2 Sv = sub(mul(s2(L.g * L.ey), h), mul(mul(k, uy), sp));
    // the hardware reciprocal (1/x is approximate under -prec-div=false):
    // rcp(0) = inf and rcp(inf) = 0 keep the non-finite test below exact
    const float2 rsp = f2(sp.x > 0.0f ? 1.0f / sp.x : 0.0f, sp.y > 0.0f ? 1.0f / sp.y : 0.0f);
    const float2 dsx = mul(mul(ux, hinv), rsp), dsy = mul(mul(uy, hinv), rsp);
    const float2 nk = neg(k), vdt = s2(dt), one = s2(1.0f);
    const float2 J22 = mul(nk, fma(hinv, sp, mul(ux, dsx))), J23 = mul(nk, mul(ux, dsy));
    const float2 J32 = mul(nk, mul(uy, dsx)), J33 = mul(nk, fma(hinv, sp, mul(uy, dsy)));
    const float2 a = fma(neg(vdt), J22, one), b = mul(neg(vdt), J23);
    const float2 c = mul(neg(vdt), J32), d = fma(neg(vdt), J33, one);
    const float2 det = sub(mul(a, d), mul(b, c));
    const float2 r0 = mul(vdt, Su), r1 = mul(vdt, Sv);
    const float2 rdet = f2(1.0f / det.x, 1.0f / det.y);
    const float2 x0 = mul(sub(mul(r0, d), mul(b, r1)), rdet);
    const float2 x1 = mul(sub(mul(a, r1), mul(c, r0)), rdet);
    // a zero, infinite or NaN determinant makes the solution non-finite
    const float2 xs = add(x0, x1);
    const bool okx = isfinite(xs.x), oky = isfinite(xs.y);
    du = f2(okx ? x0.x : (isfinite(r0.x) ? r0.x : 0.0f), oky ? x0.y : (isfinite(r0.y) ? r0.y : 0.0f));
    dv = f2(okx ? x1.x : (isfinite(r1.x) ? r1.x : 0.0f), oky ? x1.y : (isfinite(r1.y) ? r1.y : 0.0f));
}

// Two-sum on both columns: s + e == a + b exactly per lane pair.
__device__ __forceinline__ void two_sum2(float2 a, float2 b, float2& s, float2& e) {
    s = add(a, b);
    const float2 bp = sub(s, a);
    const float2 ap = sub(s, bp);
    e = add(sub(a, ap), sub(b, bp));
}

__device__ __forceinline__ float2 shfl_up2(float2 v, int d) {
    return f2(__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d));
}

// One warp's sub-strip of the paired sweep: column pairs x0-2+2L, rows j0 .. j0+CPT-1.
template <int MODE, bool WB, bool IMPL, int CPT, bool INTERIOR, bool VEC, bool PF>
__device__ __forceinline__ void sweep_strip2(const float* __restrict__ bed, const float* __restrict__ X,
                                             const float* __restrict__ inc_in, float* __restrict__ inc_out,
                                             float* __restrict__ Y, float* __restrict__ lo, const Params& L,
                                             int x0, int j0, float dt, double dtd, double& m_loc,
                                             double& s_loc, float2* __restrict__ cstage) {
    const int lane = threadIdx.x & 31;
    const int nx = L.nx, ny = L.ny;
    const long long pl = L.plane;
    const int cA = x0 - 2 + 2 * lane;
    const bool inner = (lane >= 1) && (lane <= 30);
    const bool ownA = inner && (cA < nx), ownB = inner && (cA + 1 < nx);
    const bool vec_io = VEC && INTERIOR;    // both cells in the domain, 8-byte aligned

    C42 wm = fetch2<MODE, INTERIOR, VEC>(bed, X, inc_in, L, cA, j0 - 2);
    C42 w0 = fetch2<MODE, INTERIOR, VEC>(bed, X, inc_in, L, cA, j0 - 1);
    C42 w1 = fetch2<MODE, INTERIOR, VEC>(bed, X, inc_in, L, cA, j0);
    C42 w2 = fetch2<MODE, INTERIOR, VEC>(bed, X, inc_in, L, cA, j0 + 1);
    RS2 lo_m, hi_m, lo_0, hi_0;
    reconstruct2(wm, w0, w1, lo_m, hi_m);
    reconstruct2(w0, w1, w2, lo_0, hi_0);
    // The face below the current row enters the y balance only through
    // f - D+ (and - P(h*_R) with WB): carry those three values from row to row
    // instead of the whole face (6 registers instead of 14).
    float2 gb0, gb1, gb2;
    {
        const FaceLR fb = face2<1, WB>(hi_m, lo_0, L);
        gb0 = fb.l0; gb1 = fb.l1; gb2 = fb.l2;
    }
    float m_f = 0.0f;    // CFL max of this sweep (>= 0, never NaN), merged into m_loc at the end
    RS2 top = hi_0;
    const float2 rdx = s2(L.rdx), rdy = s2(L.rdy), vdt = s2(dt);
    C42 w3 = fetch2<MODE, INTERIOR, VEC>(bed, X, inc_in, L, cA, j0 + 2);

#pragma unroll 1
    for (int r = 0; r < CPT; ++r) {
        const int j = j0 + r;
        if (j >= ny) break;                  // uniform across the warp
        // row j+3 is loaded one iteration ahead (latency hidden behind this row)
        const C42 w4 = (r + 1 < CPT) ? fetch2<MODE, INTERIOR, VEC>(bed, X, inc_in, L, cA, j + 3) : w3;
        // stage 2: the pair's FP32 state, stage-1 increment and remainder for
        // the compensated update. PF: copied asynchronously into this warp's
        // shared staging area (cp.async, no registers held) at the top of the
        // row so that they arrive during the face work; otherwise loaded where
        // they are used.
        float2 cx[3], ci[3], cl[3];
        auto load_comp = [&]() {
            const long long c = (long long)j * nx + cA;
            if (vec_io && (ownA || ownB)) {
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    cx[q] = __ldg(reinterpret_cast<const float2*>(X + q * pl + c));
                    ci[q] = __ldg(reinterpret_cast<const float2*>(inc_in + q * pl + c));
                    cl[q] = *reinterpret_cast<const float2*>(lo + q * pl + c);
                }
            } else {
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    cx[q] = f2(ownA ? __ldg(X + q * pl + c) : 0.0f, ownB ? __ldg(X + q * pl + c + 1) : 0.0f);
                    ci[q] = f2(ownA ? __ldg(inc_in + q * pl + c) : 0.0f, ownB ? __ldg(inc_in + q * pl + c + 1) : 0.0f);
                    cl[q] = f2(ownA ? lo[q * pl + c] : 0.0f, ownB ? lo[q * pl + c + 1] : 0.0f);
                }
            }
        };
        if constexpr (MODE == S2 && PF) {
            if (vec_io && (ownA || ownB)) {
                const long long c = (long long)j * nx + cA;
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    __pipeline_memcpy_async(cstage + q * 32 + lane, X + q * pl + c, 8);
                    __pipeline_memcpy_async(cstage + (3 + q) * 32 + lane, inc_in + q * pl + c, 8);
                    __pipeline_memcpy_async(cstage + (6 + q) * 32 + lane, lo + q * pl + c, 8);
                }
                __pipeline_commit();
            }
        }
        RS2 lo_1, hi_1;
        reconstruct2(w1, w2, w3, lo_1, hi_1);
        const FaceLR ft = face2<1, WB>(top, lo_1, L);

        // x: A's left neighbour is lane-1's B, B's right neighbour is lane+1's A
        const float pb = __shfl_up_sync(0xffffffffu, w1.b.y, 1), pe = __shfl_up_sync(0xffffffffu, w1.e.y, 1);
        const float pu = __shfl_up_sync(0xffffffffu, w1.u.y, 1), pv = __shfl_up_sync(0xffffffffu, w1.v.y, 1);
        const float nb = __shfl_down_sync(0xffffffffu, w1.b.x, 1), ne = __shfl_down_sync(0xffffffffu, w1.e.x, 1);
        const float nu = __shfl_down_sync(0xffffffffu, w1.u.x, 1), nv = __shfl_down_sync(0xffffffffu, w1.v.x, 1);
        const C42 m{f2(pb, w1.b.x), f2(pe, w1.e.x), f2(pu, w1.u.x), f2(pv, w1.v.x)};
        const C42 p{f2(w1.b.y, nb), f2(w1.e.y, ne), f2(w1.u.y, nu), f2(w1.v.y, nv)};
        RS2 xlo, xhi;
        reconstruct2(m, w1, p, xlo, xhi);
        // left states: (lane-1's B at its upper face, A at its upper face)
        const RS2 xl{f2(__shfl_up_sync(0xffffffffu, xhi.b.y, 1), xhi.b.x),
                     f2(__shfl_up_sync(0xffffffffu, xhi.h.y, 1), xhi.h.x),
                     f2(__shfl_up_sync(0xffffffffu, xhi.e.y, 1), xhi.e.x),
                     f2(__shfl_up_sync(0xffffffffu, xhi.u.y, 1), xhi.u.x),
                     f2(__shfl_up_sync(0xffffffffu, xhi.v.y, 1), xhi.v.x)};
        const FaceLR fl = face2<0, WB>(xl, xlo, L);   // faces left of A and between A and B
        // r of the faces right of A and B: (A|B, lane+1's left-of-A)
        const float2 fr0 = f2(fl.l0.y, __shfl_down_sync(0xffffffffu, fl.l0.x, 1));
        const float2 fr1 = f2(fl.r1.y, __shfl_down_sync(0xffffffffu, fl.r1.x, 1));
        const float2 fr2 = f2(fl.r2.y, __shfl_down_sync(0xffffffffu, fl.r2.x, 1));

        if (ownA || ownB) {
            // make_rhs.H:346-399 (WB bed source folded into l / r before the 1/dx scaling)
            const float2 Ax0 = sub(fl.l0, fr0), Ax1 = sub(fl.l1, fr1), Ax2 = sub(fl.l2, fr2);
            const float2 Ay0 = sub(gb0, ft.l0), Ay1 = sub(gb1, ft.r1), Ay2 = sub(gb2, ft.r2);
            const float2 r0 = fma(Ax0, rdx, mul(Ay0, rdy));
            const float2 r1 = fma(Ax1, rdx, mul(Ay1, rdy));
            const float2 r2 = fma(Ax2, rdx, mul(Ay2, rdy));
            const float2 h = sub(w1.e, w1.b);
            const float2 hinv = kp_hinv2(h, L);
            float2 inc_e = mul(vdt, r0), inc_u = mul(vdt, r1), inc_v = mul(vdt, r2);
            if constexpr (!IMPL) {
                const float2 mh = fmax2(h, s2(L.hfloor));
                const float2 k = mul(s2(L.g * L.nm * L.nm),
                                     f2(zb::inv_cbrt_pos(mh.x), zb::inv_cbrt_pos(mh.y)));
                const float2 ux = mul(w1.u, hinv), uy = mul(w1.v, hinv);
                const float2 sp = sqrt2(fma(ux, ux, mul(uy, uy)));
                inc_u = fma(vdt, sub(mul(s2(L.g * L.ex), h), mul(mul(k, ux), sp)), inc_u);
                inc_v = fma(vdt, sub(mul(s2(L.g * L.ey), h), mul(mul(k, uy), sp)), inc_v);
            } else {
                const float2 he = add(h, inc_e), ue = add(w1.u, inc_u), ve = add(w1.v, inc_v);
                if (he.x < kNearDry || he.y < kNearDry) {
                    float du[2], dv[2];
                    const float hh[2] = {he.x, he.y}, uu[2] = {ue.x, ue.y}, vv[2] = {ve.x, ve.y};
                    const float hi[2] = {hinv.x, hinv.y};
#pragma unroll
                    for (int k = 0; k < 2; ++k) {
                        if (hh[k] < kNearDry) {
                            double a = 0.0, b = 0.0;
                            if (!rest_without_source(hh[k], uu[k], vv[k], L))
                                manning_implicit<double>(double(hh[k]), double(uu[k]), double(vv[k]),
                                                         double(hi[k]), dtd, L.gd, L.exd, L.eyd, L.nmd,
                                                         L.hfloord, a, b);
                            du[k] = float(a); dv[k] = float(b);
                        } else {
                            manning_implicit<float>(hh[k], uu[k], vv[k], hi[k], dt, L.g, L.ex, L.ey, L.nm,
                                                    L.hfloor, du[k], dv[k]);
                        }
                    }
                    inc_u = add(inc_u, f2(du[0], du[1]));
                    inc_v = add(inc_v, f2(dv[0], dv[1]));
                } else {
                    float2 du, dv;
                    manning_implicit2(he, ue, ve, hinv, dt, L, du, dv);
                    inc_u = add(inc_u, du);
                    inc_v = add(inc_v, dv);
                }
            }
            const long long c = (long long)j * nx + cA;
            if constexpr (MODE == S1) {
                if (vec_io) {
                    *reinterpret_cast<float2*>(inc_out + c) = inc_e;
                    *reinterpret_cast<float2*>(inc_out + pl + c) = inc_u;
                    *reinterpret_cast<float2*>(inc_out + 2 * pl + c) = inc_v;
                } else {
                    if (ownA) { inc_out[c] = inc_e.x; inc_out[pl + c] = inc_u.x; inc_out[2 * pl + c] = inc_v.x; }
                    if (ownB) { inc_out[c + 1] = inc_e.y; inc_out[pl + c + 1] = inc_u.y; inc_out[2 * pl + c + 1] = inc_v.y; }
                }
            } else {
                // stage 2: the update's own inputs (hi, inc1, lo)
                if constexpr (PF) {
                    if (vec_io) {
                        __pipeline_wait_prior(0);
#pragma unroll
                        for (int q = 0; q < 3; ++q) {
                            cx[q] = cstage[q * 32 + lane];
                            ci[q] = cstage[(3 + q) * 32 + lane];
                            cl[q] = cstage[(6 + q) * 32 + lane];
                        }
                    } else {
                        load_comp();   // edge strips: plain loads
                    }
                } else {
                    load_comp();
                }
                // compensated Heun update Q^{n+1} = (hi + lo) + (inc1 + inc2) / 2: the
                // small part t = lo + (inc1 + inc2) / 2 in packed FP32, then an
                // exact two-sum hi + t -> (hi', lo')
                const float2 i2[3] = {inc_e, inc_u, inc_v};
                float2 nf2[3], nl2[3];
#pragma unroll
                for (int q = 0; q < 3; ++q)
                    two_sum2(cx[q], add(cl[q], mul(s2(0.5f), add(ci[q], i2[q]))), nf2[q], nl2[q]);
                float nf[2][3], nl[2][3];
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    nf[0][q] = nf2[q].x; nf[1][q] = nf2[q].y;
                    nl[0][q] = nl2[q].x; nl[1][q] = nl2[q].y;
                }
                // CFL terms of the new state (ZoomyAmr.cpp:472-487), packed, and its FP64 mass
                const float2 hn = sub(nf2[0], w1.b);
                const float2 hin = kp_hinv2(hn, L);
                const float2 c0 = sqrt2(mul(s2(L.g), fmax2(hn, s2(0.0f))));
                const float2 evx = mul(add(fabs2(mul(nf2[1], hin)), c0), s2(L.rfdx));
                const float2 evy = mul(add(fabs2(mul(nf2[2], hin)), c0), s2(L.rfdy));
                const float2 ev = fmax2(fmax2(evx, evy), s2(0.0f));
                if (ownA) {
                    m_f = fmaxf(m_f, ev.x);
                    s_loc = s_loc + ((double(nf[0][0]) - double(w1.b.x)) + double(nl[0][0]));
                }
                if (ownB) {
                    m_f = fmaxf(m_f, ev.y);
                    s_loc = s_loc + ((double(nf[1][0]) - double(w1.b.y)) + double(nl[1][0]));
                }
                if (vec_io) {
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        *reinterpret_cast<float2*>(Y + q * pl + c) = f2(nf[0][q], nf[1][q]);
                        *reinterpret_cast<float2*>(lo + q * pl + c) = f2(nl[0][q], nl[1][q]);
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < 2; ++k) {
                        if (!(k == 0 ? ownA : ownB)) continue;
#pragma unroll
                        for (int q = 0; q < 3; ++q) {
                            Y[q * pl + c + k] = nf[k][q];
                            lo[q * pl + c + k] = nl[k][q];
                        }
                    }
                }
            }
        }
        gb0 = ft.l0; gb1 = ft.l1; gb2 = ft.l2;
        top = hi_1;
        w0 = w1; w1 = w2; w2 = w3; w3 = w4;
    }
    (void)w0;
    if (double(m_f) > m_loc) m_loc = double(m_f);
}

// Whether a paired strip's stencil lies inside the domain (columns x0-2 ..
// x0+61, rows y0-2 .. y0+rows+1).
template <int NW, int CPT>
__device__ __forceinline__ bool strip_interior2(const Params& L, int x0, int y0) {
    return (x0 - 2 >= 0) && (x0 + 61 <= L.nx - 1) && (y0 - 2 >= 0) && (y0 + NW * CPT + 1 <= L.ny - 1);
}

}  // namespace pk
}  // namespace zfv32
