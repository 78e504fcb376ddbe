// FP32 chosen form: the warp column-sweep stage kernel.
//
// Work unit = a strip of 31 owned columns x (NW * CPT) rows. One warp per
// 31 x CPT sub-strip; lane L holds column x0 + L (lane 31 holds the first
// column of the next strip, needed only as stencil input and for the right
// face of lane 30's cell). Each lane walks its CPT rows upward keeping a
// four-row register window of its column (the y-stencil of MUSCL needs rows
// j-2..j+1), takes the x-stencil of row j from its neighbours by warp
// shuffles, and evaluates
//   * the x-face on its left (the right face of its left neighbour arrives
//     by a shuffle, so every x-face is evaluated once, 1/32 redundant), and
//   * the y-face above its cell (the face below is carried over from the
//     previous row in registers),
// then assembles its cell. No shared memory and no barriers in the sweep.
//
// Ghost cells (outside the domain) are produced by `fetch`: the mirror index
// of ZoomyAmr::FillPhysicalBC_mf (ZoomyAmr.cpp:399-406) with the side's
// boundary condition (extrapolation copies; a wall reverses the normal
// momentum), x side first.
#pragma once

namespace zfv32 {

struct Strip {            // one work unit (a level may be an element of a batch)
    int x0, y0;           // first owned column / row
};

// State of one cell for the stencil: bed, surface, momenta.
__device__ __forceinline__ C4 shfl_c4(unsigned mask, const C4& v, int src) {
    return C4{__shfl_sync(mask, v.b, src), __shfl_sync(mask, v.e, src),
              __shfl_sync(mask, v.u, src), __shfl_sync(mask, v.v, src)};
}
__device__ __forceinline__ C4 shfl_up_c4(const C4& v, int d) {
    return C4{__shfl_up_sync(0xffffffffu, v.b, d), __shfl_up_sync(0xffffffffu, v.e, d),
              __shfl_up_sync(0xffffffffu, v.u, d), __shfl_up_sync(0xffffffffu, v.v, d)};
}
__device__ __forceinline__ C4 shfl_down_c4(const C4& v, int d) {
    return C4{__shfl_down_sync(0xffffffffu, v.b, d), __shfl_down_sync(0xffffffffu, v.e, d),
              __shfl_down_sync(0xffffffffu, v.u, d), __shfl_down_sync(0xffffffffu, v.v, d)};
}

// Stage input of cell (i, j) with ghost handling. S2 reads the stage-2 state
// X + inc1. Rows/columns more than 2 cells outside the domain are never
// consumed; they are clamped to a valid address.
template <int MODE>
__device__ __forceinline__ C4 fetch(const float* __restrict__ bed, const float* __restrict__ X,
                                    const float* __restrict__ inc, const Params& L, int i, int j) {
    const int nx = L.nx, ny = L.ny;
    int ii = i, jj = j;
    int side = -1;
    if (i < 0) { ii = -1 - i; side = 0; }
    else if (i > nx - 1) { ii = 2 * (nx - 1) + 1 - i; side = 1; }
    if (j < 0) { jj = -1 - j; if (side < 0) side = 2; }
    else if (j > ny - 1) { jj = 2 * (ny - 1) + 1 - j; if (side < 0) side = 3; }
    ii = min(max(ii, 0), nx - 1);
    jj = min(max(jj, 0), ny - 1);
    const long long c = (long long)jj * nx + ii;
    const long long pl = L.plane;
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
    if (side >= 0 && L.bc_tag[side] == 1) {   // wall: reverse the normal momentum
        if (side < 2) q.u = -q.u;
        else q.v = -q.v;
    }
    return q;
}

// Face outputs kept in registers.
struct FaceR {
    float f0, f1, f2;      // central flux (h, hu, hv)
    float dp0, dp1, dp2;   // D+
    float dm0, dm1, dm2;   // D-
    float pl, pr;          // P(h*_L), P(h*_R)
};
template <int ORDER, int DIR, bool WB>
__device__ __forceinline__ FaceR face_r(const C4& LL, const C4& Lc, const C4& Rc, const C4& RR,
                                        const Params& L) {
    float F[NFC];
    face<ORDER, DIR, WB>(LL, Lc, Rc, RR, L, F);
    return FaceR{F[0], F[1], F[2], F[3], F[4], F[5], F[6], F[7], F[8], F[9], F[10]};
}

template <int ORDER, int MODE, bool WB, bool IMPL, int NW, int CPT>
__global__ void __launch_bounds__(32 * NW)
k32s_stage(const float* __restrict__ bed, const float* __restrict__ X, const float* __restrict__ inc_in,
           float* __restrict__ inc_out, float* __restrict__ Y, float* __restrict__ lo, Params L,
           zfv::DevState* st, double* __restrict__ partials, double* __restrict__ log3, int log_cap)
{
    static_assert(ORDER == 2, "the sweep kernel implements the order-2 (SSP-RK2) path");
    constexpr int NT = 32 * NW;
    __shared__ double red[2 * NW];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nx = L.nx, ny = L.ny;
    const long long pl = L.plane;
    const int x0 = blockIdx.x * 31;
    const int i = x0 + lane;
    const int j0 = blockIdx.y * (NW * CPT) + w * CPT;

    if (*(volatile unsigned*)&st->flags & zfv::kFlagDone) {
        if constexpr (MODE == S2) {   // keep the state in this step's output buffer
            if (lane < 31 && i < nx)
                for (int r = 0; r < CPT; ++r) {
                    const int j = j0 + r;
                    if (j < ny) {
                        const long long c = (long long)j * nx + i;
                        Y[c] = X[c]; Y[pl + c] = X[pl + c]; Y[2 * pl + c] = X[2 * pl + c];
                    }
                }
        }
        return;
    }
    const double dtd = *(volatile double*)&st->dt;
    const double time = *(volatile double*)&st->time;
    const float dt = float(dtd);

    // column of the extra x-stencil value of this lane: lanes 0/1 hold x0-2 / x0-1,
    // lane 31 holds x0+32 (the right neighbour of lane 31's column)
    const int xe = (lane == 0) ? x0 - 2 : (lane == 1) ? x0 - 1 : x0 + 32;
    const bool has_e = (lane <= 1) || (lane == 31);
    // a lane whose column lies beyond the ghost frame only feeds unused values
    const bool col_ok = (i <= nx + 1);
    const bool owns = (lane < 31) && (i < nx);

    // y window of this lane's column: rows j-2, j-1, j, j+1
    C4 w0 = fetch<MODE>(bed, X, inc_in, L, i, j0 - 2);
    C4 w1 = fetch<MODE>(bed, X, inc_in, L, i, j0 - 1);
    C4 w2 = fetch<MODE>(bed, X, inc_in, L, i, j0);
    C4 w3 = fetch<MODE>(bed, X, inc_in, L, i, j0 + 1);
    // face below the first row (between rows j0-1 and j0)
    FaceR fb = face_r<ORDER, 1, WB>(w0, w1, w2, w3, L);

    double m_loc = 0.0, s_loc = 0.0;
#pragma unroll 1
    for (int r = 0; r < CPT; ++r) {
        const int j = j0 + r;
        if (j >= ny) break;                          // uniform across the warp
        // slide the window: rows j-1 .. j+2
        w0 = w1; w1 = w2; w2 = w3;
        w3 = fetch<MODE>(bed, X, inc_in, L, i, j + 2);
        // face above row j (between rows j and j+1): stencil rows j-1 .. j+2
        const FaceR ft = face_r<ORDER, 1, WB>(w0, w1, w2, w3, L);

        // x-stencil of row j: own = w1 (row j of column i)
        const C4 own = w1;
        C4 ex{};
        if (has_e) ex = fetch<MODE>(bed, X, inc_in, L, xe, j);
        const C4 up1 = shfl_up_c4(own, 1), up2 = shfl_up_c4(own, 2), dn1 = shfl_down_c4(own, 1);
        const C4 e1 = shfl_c4(0xffffffffu, ex, 1);   // x0-1, held by lane 1
        const C4 cm1 = (lane == 0) ? e1 : up1;       // column i-1
        const C4 cm2 = (lane <= 1) ? ex : up2;       // column i-2 (lane 0: x0-2, lane 1: x0-1)
        const C4 cp1 = (lane == 31) ? ex : dn1;      // column i+1
        // x-face on the left of column i: cells i-2, i-1 | i, i+1
        const FaceR fl = face_r<ORDER, 0, WB>(cm2, cm1, own, cp1, L);
        // the face on the right of column i is lane+1's left face
        FaceR fr;
        fr.f0 = __shfl_down_sync(0xffffffffu, fl.f0, 1);
        fr.f1 = __shfl_down_sync(0xffffffffu, fl.f1, 1);
        fr.f2 = __shfl_down_sync(0xffffffffu, fl.f2, 1);
        fr.dm0 = __shfl_down_sync(0xffffffffu, fl.dm0, 1);
        fr.dm1 = __shfl_down_sync(0xffffffffu, fl.dm1, 1);
        fr.dm2 = __shfl_down_sync(0xffffffffu, fl.dm2, 1);
        fr.pl = __shfl_down_sync(0xffffffffu, fl.pl, 1);

        if (owns && col_ok) {
            // make_rhs.H:346-399 with the WB source folded before the 1/dx scaling
            float Ax0 = -(fr.f0 - fl.f0) - fr.dm0 - fl.dp0;
            float Ax1 = -(fr.f1 - fl.f1) - fr.dm1 - fl.dp1;
            float Ax2 = -(fr.f2 - fl.f2) - fr.dm2 - fl.dp2;
            float Ay0 = -(ft.f0 - fb.f0) - ft.dm0 - fb.dp0;
            float Ay1 = -(ft.f1 - fb.f1) - ft.dm1 - fb.dp1;
            float Ay2 = -(ft.f2 - fb.f2) - ft.dm2 - fb.dp2;
            if constexpr (WB) {
                Ax1 += fr.pl - fl.pr;
                Ay2 += ft.pl - fb.pr;
            }
            const float r0 = Ax0 * L.rdx + Ay0 * L.rdy;
            const float r1 = Ax1 * L.rdx + Ay1 * L.rdy;
            const float r2 = Ax2 * L.rdx + Ay2 * L.rdy;
            const float h = own.e - own.b;
            const float hinv = kp_hinv(h, L.eps);
            float inc_e = dt * r0, inc_u = dt * r1, inc_v = dt * r2;
            if constexpr (!IMPL) {
                const float mh = fmaxf(h, L.hfloor);
                const float k = L.g * L.nm * L.nm * zb::inv_cbrt_pos(mh);
                const float ux = own.u * hinv, uy = own.v * hinv;
                const float sp = sqrtf(ux * ux + uy * uy);
                inc_u += dt * (L.g * L.ex * h - k * ux * sp);
                inc_v += dt * (L.g * L.ey * h - k * uy * sp);
            } else {
                const float he = h + inc_e, ue = own.u + inc_u, ve = own.v + inc_v;
                if (he < kNearDry) {
                    double du, dv;
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
                const float i1e = __ldg(inc_in + c), i1u = __ldg(inc_in + pl + c), i1v = __ldg(inc_in + 2 * pl + c);
                const float xe_ = __ldg(X + c), xu = __ldg(X + pl + c), xv = __ldg(X + 2 * pl + c);
                const double ne = (double(xe_) + double(lo[c])) + 0.5 * (double(i1e) + double(inc_e));
                const double nu = (double(xu) + double(lo[pl + c])) + 0.5 * (double(i1u) + double(inc_u));
                const double nv = (double(xv) + double(lo[2 * pl + c])) + 0.5 * (double(i1v) + double(inc_v));
                const float he = float(ne), hu = float(nu), hv = float(nv);
                Y[c] = he; Y[pl + c] = hu; Y[2 * pl + c] = hv;
                lo[c] = float(ne - double(he));
                lo[pl + c] = float(nu - double(hu));
                lo[2 * pl + c] = float(nv - double(hv));
                const float hn = he - own.b;
                const float hin = kp_hinv(hn, L.eps);
                const float c0 = sqrtf(L.g * fmaxf(hn, 0.0f));
                const float evx = (fabsf(hu * hin) + c0) / L.fdx;
                const float evy = (fabsf(hv * hin) + c0) / L.fdy;
                float mm_ = 0.0f;
                if (evx > mm_) mm_ = evx;
                if (evy > mm_) mm_ = evy;
                if (double(mm_) > m_loc) m_loc = double(mm_);
                s_loc = s_loc + (ne - double(own.b));
            }
        }
        fb = ft;   // the face above row j is the face below row j+1
    }
    if constexpr (MODE == S2)
        zfv::finish_step<NT>(m_loc, s_loc, red, partials, log3, log_cap, st, L, dtd, time);
}

}  // namespace zfv32
