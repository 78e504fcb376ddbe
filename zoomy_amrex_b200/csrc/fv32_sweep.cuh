// FP32 chosen form: the warp column-sweep stage.
//
// Work unit ("strip") = 30 owned columns x (NW * CPT) rows, one warp per
// 30 x CPT sub-strip. Lane L holds column x0 - 1 + L (lanes 1..30 own their
// column; lane 0 and lane 31 hold the neighbour columns x0 - 1 and x0 + 30).
// Each lane walks its CPT rows upward and, per row j,
//   * reconstructs its cell once in x (MUSCL/minmod slopes of b, h, hu, hv,
//     make_rhs.H:57-75, with the slope of h taken as d(eta) - d(b)) and once in
//     y (for row j+1, from a register window of its column),
//   * evaluates the x-face on its left from its left neighbour's right-face
//     state (one shuffle) and its own left-face state, and the y-face above
//     its cell from the carried top-face state of row j and the bottom-face
//     state of row j+1,
//   * receives the face on its right from lane+1 (one shuffle) and the face
//     below from the previous row (registers), and assembles its cell.
// Every face and every slope is evaluated once (plus 1/16 of the x work for
// the two neighbour columns). No shared memory and no barriers in the sweep.
//
// Ghost cells are produced by fetch(): the mirror index of
// ZoomyAmr::FillPhysicalBC_mf (ZoomyAmr.cpp:399-406) with the side's boundary
// condition (extrapolation copies; a wall reverses the normal momentum), x side
// first; strips whose stencil lies inside the domain skip that logic.
#pragma once
#include <cuda_pipeline.h>

namespace zfv32 {

// Reconstructed state of a cell at one of its faces.
struct RS { float b, h, e, u, v; };

__device__ __forceinline__ C4 shfl_up_c4(const C4& v, int d) {
    return C4{__shfl_up_sync(0xffffffffu, v.b, d), __shfl_up_sync(0xffffffffu, v.e, d),
              __shfl_up_sync(0xffffffffu, v.u, d), __shfl_up_sync(0xffffffffu, v.v, d)};
}
__device__ __forceinline__ C4 shfl_down_c4(const C4& v, int d) {
    return C4{__shfl_down_sync(0xffffffffu, v.b, d), __shfl_down_sync(0xffffffffu, v.e, d),
              __shfl_down_sync(0xffffffffu, v.u, d), __shfl_down_sync(0xffffffffu, v.v, d)};
}
__device__ __forceinline__ RS shfl_up_rs(const RS& v, int d) {
    return RS{__shfl_up_sync(0xffffffffu, v.b, d), __shfl_up_sync(0xffffffffu, v.h, d),
              __shfl_up_sync(0xffffffffu, v.e, d), __shfl_up_sync(0xffffffffu, v.u, d),
              __shfl_up_sync(0xffffffffu, v.v, d)};
}

// Per-cell MUSCL reconstruction from (minus, centre, plus) neighbours along one
// axis: lo = state at the cell's lower face, hi = at its upper face.
__device__ __forceinline__ void reconstruct(const C4& m, const C4& c, const C4& p, RS& lo, RS& hi) {
    const float dbm = c.b - m.b, dbp = p.b - c.b;
    const float dem = c.e - m.e, dep = p.e - c.e;
    const float gb = mm(dbm, dbp);
    const float gh = mm(dem - dbm, dep - dbp);
    const float gu = mm(c.u - m.u, p.u - c.u);
    const float gv = mm(c.v - m.v, p.v - c.v);
    const float h = c.e - c.b;
    const float hb = 0.5f * gb, hh = 0.5f * gh, he = 0.5f * (gh + gb);
    const float hu = 0.5f * gu, hv = 0.5f * gv;
    hi = RS{c.b + hb, h + hh, c.e + he, c.u + hu, c.v + hv};
    lo = RS{c.b - hb, h - hh, c.e - he, c.u - hu, c.v - hv};
}

// What a face contributes to the balance of its two cells (make_rhs.H:346-399):
// the cell on its high side gets  l = f - D+ (- P(h*_R) in the momentum
// normal to the face, the WB bed source), the cell on its low side loses
// r = f + D- (- P(h*_L)); a cell's balance is l(low face) - r(high face).
// D+ and D- differ only in the sign of the Rusanov term for h (so l0 = r0)
// and in the bed term of the normal momentum, so 5 values describe a face.
struct FaceR {
    float l0, l1, l2;
    float r1, r2;
};

// One face from its reconstructed left/right states (make_rhs.H:77-131 from
// the Audusse step on, with the model's flux and D+/- fluctuations).
template <int DIR, bool WB>
__device__ __forceinline__ FaceR face_rs(RS a, RS c, const Params& L) {
    float db = 0.0f;
    if constexpr (WB) {
        const float bf = fmaxf(a.b, c.b);
        const float hsL = fmaxf(0.0f, a.e - bf), hsR = fmaxf(0.0f, c.e - bf);
        const float sL = (a.h > 0.0f) ? __fdividef(hsL, a.h) : 0.0f;
        const float sR = (c.h > 0.0f) ? __fdividef(hsR, c.h) : 0.0f;
        a.u *= sL; a.v *= sL; c.u *= sR; c.v *= sR;
        a.h = hsL; c.h = hsR;
    } else {
        db = c.b - a.b;
    }
    const float g = L.g, hg = 0.5f * L.g;
    const float hiL = kp_hinv_w(a.h, L.eps, L.hwet), hiR = kp_hinv_w(c.h, L.eps, L.hwet);
    const float unL = (DIR == 0) ? a.u : a.v, unR = (DIR == 0) ? c.u : c.v;
    const float pL = hg * a.h * a.h, pR = hg * c.h * c.h;
    const float qL = unL * hiL, qR = unR * hiR;          // normal velocities
    float fuL, fvL, fuR, fvR;
    if constexpr (DIR == 0) {
        fuL = a.u * qL + pL;  fvL = a.v * qL;
        fuR = c.u * qR + pR;  fvR = c.v * qR;
    } else {
        fuL = a.u * qL;  fvL = a.v * qL + pL;
        fuR = c.u * qR;  fvR = c.v * qR + pR;
    }
    const float f0 = 0.5f * (unL + unR);
    const float f1 = 0.5f * (fuL + fuR);
    const float f2 = 0.5f * (fvL + fvR);
    const float evL = fabsf(qL) + sqrtf(g * fmaxf(a.h, 0.0f));
    const float evR = fabsf(qR) + sqrtf(g * fmaxf(c.h, 0.0f));
    const float hs = 0.5f * fmaxf(evL, evR);
    const float dh = c.h - a.h, du = c.u - a.u, dv = c.v - a.v;
    FaceR F;
    F.l0 = f0 - hs * dh;
    const float b1 = f1 - hs * du, b2 = f2 - hs * dv;
    F.l1 = F.r1 = b1;
    F.l2 = F.r2 = b2;
    // the normal momentum: WB pressure terms P(h*_R) / P(h*_L), else the
    // path-conservative bed product g (hL + hR)/2 (bR - bL) in D+ and D-
    const float kl = WB ? pR : 0.5f * g * (0.5f * (a.h + c.h)) * db;
    const float kr = WB ? pL : -kl;
    if constexpr (DIR == 0) { F.l1 = b1 - kl; F.r1 = b1 - kr; }
    else                    { F.l2 = b2 - kl; F.r2 = b2 - kr; }
    return F;
}

// Stage input of cell (i, j). S2 reads the stage-2 state X + inc1.
template <int MODE, bool INTERIOR>
__device__ __forceinline__ C4 fetch(const float* __restrict__ bed, const float* __restrict__ X,
                                    const float* __restrict__ inc, const Params& L, int i, int j) {
    const long long pl = L.plane;
    int ii = i, jj = j, side = -1;
    if constexpr (!INTERIOR) {
        const int nx = L.nx, ny = L.ny;
        if (L.frame && (i < 0 || i > nx - 1 || j < 0 || j > ny - 1)) {
            // AMR box: the ghost frame holds the stage input (corner cells,
            // which no face reads, are clamped into the frame)
            const int fi = min(max(i, -2), nx + 1) + 2, fj = min(max(j, -2), ny + 1) + 2;
            const long long fp = (long long)(nx + 4) * (ny + 4);
            const long long f = (long long)fj * (nx + 4) + fi;
            return C4{__ldg(L.frame + f), __ldg(L.frame + fp + f), __ldg(L.frame + 2 * fp + f),
                      __ldg(L.frame + 3 * fp + f)};
        }
        if (i < 0) { ii = -1 - i; side = 0; }
        else if (i > nx - 1) { ii = 2 * (nx - 1) + 1 - i; side = 1; }
        if (j < 0) { jj = -1 - j; if (side < 0) side = 2; }
        else if (j > ny - 1) { jj = 2 * (ny - 1) + 1 - j; if (side < 0) side = 3; }
        ii = min(max(ii, 0), nx - 1);      // beyond the ghost frame: unused, keep in bounds
        jj = min(max(jj, 0), ny - 1);
    }
    const long long c = (long long)jj * L.nx + ii;
    C4 q;
    q.b = __ldg(bed + c);
    q.e = __ldg(X + c);
    q.u = __ldg(X + pl + c);
    q.v = __ldg(X + 2 * pl + c);
    if constexpr (MODE == S2) {
        q.e += __ldg(inc + c);
        q.u += __ldg(inc + pl + c);
        q.v += __ldg(inc + 2 * pl + c);
    }
    if constexpr (!INTERIOR) {
        if (side >= 0 && L.bc_tag[side] == 1) {   // wall: reverse the normal momentum
            if (side < 2) q.u = -q.u;
            else q.v = -q.v;
        }
    }
    return q;
}

// One warp's sub-strip: columns x0-1 .. x0+30 (owned x0 .. x0+29), rows j0 .. j0+CPT-1.
// Accumulates this lane's CFL max and mass into m_loc / s_loc (stage 2).
template <int MODE, bool WB, bool IMPL, int CPT, bool INTERIOR, bool PF>
__device__ __forceinline__ void sweep_strip(const float* __restrict__ bed, const float* __restrict__ X,
                                            const float* __restrict__ inc_in, float* __restrict__ inc_out,
                                            float* __restrict__ Y, float* __restrict__ lo, const Params& L,
                                            int x0, int j0, float dt, double dtd, double& m_loc,
                                            double& s_loc, float* __restrict__ cstage) {
    const int lane = threadIdx.x & 31;
    const int nx = L.nx, ny = L.ny;
    const long long pl = L.plane;
    const int i = x0 - 1 + lane;
    const bool owns = (lane >= 1) && (lane <= 30) && (i < nx);
    // extra x-neighbour of the edge lanes: lane 0 needs x0-2, lane 31 needs x0+31
    const bool has_e = (lane == 0) || (lane == 31);
    const int xe = (lane == 0) ? x0 - 2 : x0 + 31;

    // y window of this lane's column: rows j0-1, j0, j0+1 (raw) and the
    // y-reconstruction of row j0 (its face states below and above)
    C4 wm = fetch<MODE, INTERIOR>(bed, X, inc_in, L, i, j0 - 2);
    C4 w0 = fetch<MODE, INTERIOR>(bed, X, inc_in, L, i, j0 - 1);
    C4 w1 = fetch<MODE, INTERIOR>(bed, X, inc_in, L, i, j0);
    C4 w2 = fetch<MODE, INTERIOR>(bed, X, inc_in, L, i, j0 + 1);
    RS lo_m, hi_m, lo_0, hi_0;
    reconstruct(wm, w0, w1, lo_m, hi_m);     // row j0-1
    reconstruct(w0, w1, w2, lo_0, hi_0);     // row j0
    // l of the face below the current row, carried from row to row
    float gb0, gb1, gb2;
    {
        const FaceR fb = face_rs<1, WB>(hi_m, lo_0, L);   // face below row j0
        gb0 = fb.l0; gb1 = fb.l1; gb2 = fb.l2;
    }
    float m_f = 0.0f;    // CFL max of this sweep (>= 0, never NaN), merged into m_loc at the end
    RS top = hi_0;                           // row j0's state at its upper face
    C4 w3 = fetch<MODE, INTERIOR>(bed, X, inc_in, L, i, j0 + 2);

#pragma unroll 1
    for (int r = 0; r < CPT; ++r) {
        const int j = j0 + r;
        if (j >= ny) break;                  // uniform across the warp
        // row j: w1; rows j-1, j+1, j+2: w0, w2, w3. Row j+3 is loaded one
        // iteration ahead so its latency overlaps this row's arithmetic.
        const C4 w4 = (r + 1 < CPT) ? fetch<MODE, INTERIOR>(bed, X, inc_in, L, i, j + 3) : w3;
        // stage 2: this cell's FP32 state, stage-1 increment and remainder for
        // the compensated update. PF: copied asynchronously into this warp's
        // shared staging area (cp.async, no registers held) at the top of the
        // row so that they arrive during the face work; otherwise loaded where
        // they are used.
        float cx[3] = {0.0f, 0.0f, 0.0f}, ci[3] = {0.0f, 0.0f, 0.0f}, cl[3] = {0.0f, 0.0f, 0.0f};
        auto load_comp = [&]() {
            if (owns) {
                const long long c = (long long)j * nx + i;
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    cx[q] = __ldg(X + q * pl + c);
                    ci[q] = __ldg(inc_in + q * pl + c);
                    cl[q] = lo[q * pl + c];
                }
            }
        };
        if constexpr (MODE == S2 && PF) {
            if (owns) {
                const long long c = (long long)j * nx + i;
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    __pipeline_memcpy_async(cstage + q * 32 + lane, X + q * pl + c, 4);
                    __pipeline_memcpy_async(cstage + (3 + q) * 32 + lane, inc_in + q * pl + c, 4);
                    __pipeline_memcpy_async(cstage + (6 + q) * 32 + lane, lo + q * pl + c, 4);
                }
                __pipeline_commit();
            }
        }
        RS lo_1, hi_1;
        reconstruct(w1, w2, w3, lo_1, hi_1);  // row j+1 in y
        const FaceR ft = face_rs<1, WB>(top, lo_1, L);   // face above row j

        // x reconstruction of row j
        C4 ex{};
        if (has_e) ex = fetch<MODE, INTERIOR>(bed, X, inc_in, L, xe, j);
        // every lane takes part in both shuffles (full-mask shuffles), then selects
        const C4 up = shfl_up_c4(w1, 1);
        const C4 dn = shfl_down_c4(w1, 1);
        const C4 left = (lane == 0) ? ex : up;
        const C4 right = (lane == 31) ? ex : dn;
        RS xlo, xhi;
        reconstruct(left, w1, right, xlo, xhi);
        const RS lhi = shfl_up_rs(xhi, 1);              // left neighbour's state at our left face
        const FaceR fl = face_rs<0, WB>(lhi, xlo, L);   // face on the left of column i (lanes >= 1)
        // r of the face on the right: lane+1's left face
        const float fr0 = __shfl_down_sync(0xffffffffu, fl.l0, 1);
        const float fr1 = __shfl_down_sync(0xffffffffu, fl.r1, 1);
        const float fr2 = __shfl_down_sync(0xffffffffu, fl.r2, 1);

        if (owns) {
            // make_rhs.H:346-399 (WB bed source folded into l / r before the 1/dx scaling)
            const float Ax0 = fl.l0 - fr0, Ax1 = fl.l1 - fr1, Ax2 = fl.l2 - fr2;
            const float Ay0 = gb0 - ft.l0, Ay1 = gb1 - ft.r1, Ay2 = gb2 - ft.r2;
            const float r0 = Ax0 * L.rdx + Ay0 * L.rdy;
            const float r1 = Ax1 * L.rdx + Ay1 * L.rdy;
            const float r2 = Ax2 * L.rdx + Ay2 * L.rdy;
            const float h = w1.e - w1.b;
            const float hinv = kp_hinv_w(h, L.eps, L.hwet);
            float inc_e = dt * r0, inc_u = dt * r1, inc_v = dt * r2;
            if constexpr (!IMPL) {
                const float mh = fmaxf(h, L.hfloor);
                const float k = L.g * L.nm * L.nm * zb::inv_cbrt_pos(mh);
                const float ux = w1.u * hinv, uy = w1.v * hinv;
                const float sp = sqrtf(ux * ux + uy * uy);
                inc_u += dt * (L.g * L.ex * h - k * ux * sp);
                inc_v += dt * (L.g * L.ey * h - k * uy * sp);
            } else {
                const float he = h + inc_e, ue = w1.u + inc_u, ve = w1.v + inc_v;
                if (he < kNearDry) {
                    double du = 0.0, dv = 0.0;
                    if (!rest_without_source(he, ue, ve, L))
                        manning_implicit<double>(double(he), double(ue), double(ve), double(hinv), dtd,
                                                 L.gd, L.exd, L.eyd, L.nmd, L.hfloord, du, dv);
                    inc_u += float(du); inc_v += float(dv);
                } else {
                    float du, dv;
                    manning_implicit<float>(he, ue, ve, hinv, dt, L.g, L.ex, L.ey, L.nm, L.hfloor, du, dv);
                    inc_u += du; inc_v += dv;
                }
            }
            const long long c = (long long)j * nx + i;
            if constexpr (MODE == S1) {
                inc_out[c] = inc_e; inc_out[pl + c] = inc_u; inc_out[2 * pl + c] = inc_v;
            } else {
                // compensated Heun update Q^{n+1} = (hi + lo) + (inc1 + inc2) / 2: the
                // small part t = lo + (inc1 + inc2) / 2 in FP32, then an exact
                // two-sum hi + t -> (hi', lo')
                if constexpr (PF) {
                    __pipeline_wait_prior(0);
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        cx[q] = cstage[q * 32 + lane];
                        ci[q] = cstage[(3 + q) * 32 + lane];
                        cl[q] = cstage[(6 + q) * 32 + lane];
                    }
                } else {
                    load_comp();
                }
                float he, hu, hv, le, lu, lv;
                two_sum(cx[0], __fadd_rn(cl[0], 0.5f * __fadd_rn(ci[0], inc_e)), he, le);
                two_sum(cx[1], __fadd_rn(cl[1], 0.5f * __fadd_rn(ci[1], inc_u)), hu, lu);
                two_sum(cx[2], __fadd_rn(cl[2], 0.5f * __fadd_rn(ci[2], inc_v)), hv, lv);
                Y[c] = he; Y[pl + c] = hu; Y[2 * pl + c] = hv;
                lo[c] = le; lo[pl + c] = lu; lo[2 * pl + c] = lv;
                // CFL terms of the new state (ZoomyAmr.cpp:472-487) and its FP64 mass
                const float hn = he - w1.b;
                const float hin = kp_hinv_w(hn, L.eps, L.hwet);
                const float c0 = sqrtf(L.g * fmaxf(hn, 0.0f));
                const float evx = (fabsf(hu * hin) + c0) * L.rfdx;
                const float evy = (fabsf(hv * hin) + c0) * L.rfdy;
                float mm_ = 0.0f;
                if (evx > mm_) mm_ = evx;
                if (evy > mm_) mm_ = evy;
                m_f = fmaxf(m_f, mm_);
                s_loc = s_loc + ((double(he) - double(w1.b)) + double(le));
            }
        }
        // advance: row j+1 becomes the current row
        gb0 = ft.l0; gb1 = ft.l1; gb2 = ft.l2;
        top = hi_1;
        w0 = w1; w1 = w2; w2 = w3; w3 = w4;
    }
    if (double(m_f) > m_loc) m_loc = double(m_f);
}

// Whether a strip's stencil (two ghost layers around its cells and its two
// neighbour columns) lies inside the domain, so fetch needs no mirroring.
template <int NW, int CPT>
__device__ __forceinline__ bool strip_interior(const Params& L, int x0, int y0) {
    return (x0 - 2 >= 0) && (x0 + 31 <= L.nx - 1) && (y0 - 2 >= 0) && (y0 + NW * CPT + 1 <= L.ny - 1);
}

}  // namespace zfv32
