// Reverse-mode kernels of the FP64 SSP-RK2 step of the 2-D shallow-water
// scheme (the adjoint of zfv::k_stage in modes S1 / S2 for SWE2D, order 2).
//
// Forward step n (ZoomyAmr::Advance, ZoomyAmr.cpp:538-731; one stage is
// do_stage, :561-662):
//   stage s on input X:  q* = X + dt RHS(X)            (faces: make_rhs.H:31-399)
//                         Y  = q* + dq(q*, hinv(X.h))   (implicit: make_rhs.H:429-509)
//   Y1 = stage(Q^n), Y2 = stage(Y1), Q^{n+1} = (Q^n + Y2) / 2
//   dt_n = cfl / (d (2k+1) max_inv(Q^n))                (ComputeDt, ZoomyAmr.cpp:448-515)
// The tape of a step holds Q^n, Y1 and the q* of both stages; the reverse of
// one stage is two kernels:
//   k_adj_cell   per cell: lam_q* from lam_Y through the implicit update (IFT),
//                the hinv(X.h) term, and per-block partial sums of dL/dn_m and
//                dL/ddt;
//   k_adj_face   per tile: lam_X = lam_q* + dt (dRHS/dX)^T lam_q* (+ the hinv
//                term, + the Heun term for stage 1), the face reverses of
//                swe_adjoint.H gathered per cell in a fixed order (no atomics);
// and k_adj_dt, once per step, reduces the partials, finds the CFL argmax cell
// of Q^n and adds the dt_n term there (zero when dt was clamped).
#pragma once
#include "fv_device.cuh"
#include "swe_adjoint.H"

namespace zfv {
namespace adj {

using P6 = LevelParams<double, 6>;

__device__ __forceinline__ zadj::SweP<double> swe_params(P6 const& L) {
    return zadj::SweP<double>{L.p[0], L.p[1], L.p[2], L.p[3], L.p[4], L.p[5]};
}

// Sum of two doubles over the block (thread 0 holds the result).
template <int NT>
__device__ __forceinline__ void block_sum2(double& a, double& b, double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, off);
        b += __shfl_down_sync(0xffffffffu, b, off);
    }
    constexpr int NW = NT / 32;
    __syncthreads();
    if (lane == 0) { red[2 * warp] = a; red[2 * warp + 1] = b; }
    __syncthreads();
    if (threadIdx.x == 0) {
        a = red[0]; b = red[1];
        for (int w = 1; w < NW; ++w) { a += red[2 * w]; b += red[2 * w + 1]; }
    }
}

// Pass A. lamY = scale * lam_in (the Heun factor 1/2 for stage 2). X: stage
// input (planes 1..3 read), qs: q* (3 planes h, hu, hv). Writes lamq (4
// planes) and loc (the hinv(X.h) term of lam_X.h), partials[2 * block] =
// (dL/dn_m, dL/ddt) of this block's cells.
template <bool IMPL, int NT>
__global__ void __launch_bounds__(NT, 1024 / NT)
k_adj_cell(const double* __restrict__ lam_in, double scale, const double* __restrict__ X,
           const double* __restrict__ qs, P6 L, const double* __restrict__ meta,
           double* __restrict__ lamq, double* __restrict__ loc, double* __restrict__ partials) {
    __shared__ double red[2 * (NT / 32)];
    const long long pl = L.plane;
    const double dt = meta[1];
    const long long c = (long long)blockIdx.x * NT + threadIdx.x;
    double pnm = 0.0, pdt = 0.0;
    if (c < pl) {
        const zadj::SweP<double> p = swe_params(L);
        double lq[4];
#pragma unroll
        for (int n = 0; n < 4; ++n) lq[n] = scale * lam_in[n * pl + c];
        const double h = qs[c], mx = qs[pl + c], my = qs[2 * pl + c];
        double lhv = 0.0, dhv = 0.0;
        if constexpr (IMPL) {
            const double hv = zadj::hinv(X[pl + c], p.eps);
            dhv = zadj::dhinv_r(X[pl + c], p.eps);
            double lqi[4] = {0.0, 0.0, 0.0, 0.0};
            const double lam[2] = {lq[2], lq[3]};
            zadj::implicit_rev(h, mx, my, hv, dt, p, lam, lqi, lhv, pnm, pdt);
            lq[1] += lqi[1]; lq[2] += lqi[2]; lq[3] += lqi[3];
        }
        // q* = X + dt RHS(X): dL/ddt += lam_q* . RHS
        pdt += (lq[1] * (h - X[pl + c]) + lq[2] * (mx - X[2 * pl + c]) + lq[3] * (my - X[3 * pl + c])) / dt;
#pragma unroll
        for (int n = 0; n < 4; ++n) lamq[n * pl + c] = lq[n];
        loc[c] = IMPL ? lhv * dhv : 0.0;
    }
    block_sum2<NT>(pnm, pdt, red);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = pnm;
        partials[2 * blockIdx.x + 1] = pdt;
    }
}

// Mirror a possibly-outside index into [0, n) (ZoomyAmr.cpp:399-406; indices
// no real face reads are clamped, their values unused).
__device__ __forceinline__ int mirror(int i, int n, bool& out) {
    out = false;
    if (i < 0) { out = true; i = -1 - i; }
    else if (i >= n) { out = true; i = 2 * n - 1 - i; }
    return i < 0 ? 0 : (i >= n ? n - 1 : i);
}

// A TX x TY tile reversed by NT >= TX * TY threads: the face pass spreads
// the tile's NF faces (more than 2 per cell with the halo) over all NT
// threads; the first TX * TY threads then own one cell each.
template <int TX, int TY, int NT_ = TX * TY>
struct AdjTile {
    static constexpr int NT = NT_;
    static_assert(NT_ >= TX * TY, "one thread per cell at least");
    static constexpr int XW = TX + 6, XH = TY + 6;      // X with 3 halo cells
    static constexpr int LW = TX + 4, LH = TY + 4;      // lam_q* with 2 halo cells
    static constexpr int NFX = (TX + 3) * TY;           // x-faces x0-1 .. x0+TX+1 (right cell index)
    static constexpr int NFY = TX * (TY + 3);
    static constexpr int NF = NFX + NFY;                // both directions in one pass
    static constexpr size_t x_elems = size_t(4) * XH * XW;
    static constexpr size_t l_elems = size_t(3) * LH * LW;
    static constexpr size_t f_elems = size_t(NF) * 16;  // [16][NF]: face f's output q at q * NF + f
    static constexpr size_t smem_bytes = (x_elems + l_elems + f_elems) * sizeof(double);
};

// Pass B. X: stage input (bed from qbed, planes 1..3 from X). lamq, loc from
// pass A; addend (NULL or 4 planes) * addscale is added (the Heun term
// lam_{n+1}/2 of stage 1). lamX may alias addend.
template <bool WB, int TX, int TY, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB)
k_adj_face(const double* __restrict__ X, const double* __restrict__ qbed, const double* __restrict__ lamq,
           const double* __restrict__ loc, const double* addend, double addscale, P6 L,
           const double* __restrict__ meta, double* lamX) {
    using T = AdjTile<TX, TY, NT>;
    const double dt = meta[1];
    extern __shared__ __align__(16) double smem[];
    double* sX = smem;                       // [4][XH][XW]
    double* sL = sX + T::x_elems;            // [3][LH][LW]
    double* sF = sL + T::l_elems;            // [16][NF]
    const int nx = L.nx, ny = L.ny;
    const long long pl = L.plane;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int tid = threadIdx.x;
    const zadj::SweP<double> p = swe_params(L);
    // bit s set: side s (x_lo, x_hi, y_lo, y_hi) is a wall
    const unsigned wall = (L.bc_tag[0] == 1 ? 1u : 0u) | (L.bc_tag[1] == 1 ? 2u : 0u) |
                          (L.bc_tag[2] == 1 ? 4u : 0u) | (L.bc_tag[3] == 1 ? 8u : 0u);

    // 1. X tile with mirrored ghosts (walls flip the normal momentum)
    for (int k = tid; k < T::XH * T::XW; k += T::NT) {
        const int ly = k / T::XW, lx = k % T::XW;
        bool ox, oy;
        const int gi = x0 - 3 + lx, gj = y0 - 3 + ly;
        const int ii = mirror(gi, nx, ox), jj = mirror(gj, ny, oy);
        const long long c = (long long)jj * nx + ii;
        double v[4] = {qbed[c], X[pl + c], X[2 * pl + c], X[3 * pl + c]};
        if (ox && ((wall >> (gi < 0 ? 0 : 1)) & 1u)) v[2] = -v[2];
        else if (!ox && oy && ((wall >> (gj < 0 ? 2 : 3)) & 1u)) v[3] = -v[3];
#pragma unroll
        for (int n = 0; n < 4; ++n) sX[(n * T::XH + ly) * T::XW + lx] = v[n];
    }
    // 2. lam_q* rows 1..3 with zero outside the domain
    for (int k = tid; k < T::LH * T::LW; k += T::NT) {
        const int ly = k / T::LW, lx = k % T::LW;
        const int gi = x0 - 2 + lx, gj = y0 - 2 + ly;
        const bool in = gi >= 0 && gi < nx && gj >= 0 && gj < ny;
        const long long c = (long long)gj * nx + gi;
#pragma unroll
        for (int n = 0; n < 3; ++n) sL[(n * T::LH + ly) * T::LW + lx] = in ? lamq[(n + 1) * pl + c] : 0.0;
    }
    __syncthreads();

    const bool owner = tid < TX * TY;       // this thread owns cell (i, j) of the tile
    const int tx = tid % TX, ty = tid / TX;
    const int i = x0 + tx, j = y0 + ty;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    auto sx = [&](int n, int gi, int gj) { return sX[(n * T::XH + (gj - y0 + 3)) * T::XW + (gi - x0 + 3)]; };
    auto sl = [&](int n, int gi, int gj) { return sL[(n * T::LH + (gj - y0 + 2)) * T::LW + (gi - x0 + 2)]; };

    // 3. face reverses of all this tile's faces, x then y in one pass. The
    // outputs are stored component-major ([16][NF]) so that neighbouring
    // threads write and read neighbouring words.
    for (int f = tid; f < T::NF; f += T::NT) {
        const int D = f < T::NFX ? 0 : 1;
        const int ff = D == 0 ? f : f - T::NFX;
        const int fw = D == 0 ? TX + 3 : TX;
        // face a between cells A = a-1 and B = a along D (stencil a-2 .. a+1);
        // a = 0 and a = n are the domain's boundary faces
        const int fa = ff % fw, fb = ff / fw;
        const int gi = D == 0 ? x0 - 1 + fa : x0 + fa;   // cell B
        const int gj = D == 0 ? y0 + fb : y0 - 1 + fb;
        const int a = D == 0 ? gi : gj, na = D == 0 ? nx : ny;
        const bool real = a >= 0 && a <= na && (D == 0 ? gj < ny : gi < nx);
        if (!real) {
#pragma unroll
            for (int k = 0; k < 16; ++k) sF[k * T::NF + f] = 0.0;
            continue;
        }
        const double sc = dt / (D == 0 ? L.dx : L.dy);
        double c[4][4], lo[11], lA[3], lB[3];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int ci = D == 0 ? gi - 2 + k : gi, cj = D == 0 ? gj : gj - 2 + k;
#pragma unroll
            for (int n = 0; n < 4; ++n) c[k][n] = sx(n, ci, cj);
        }
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            lA[n] = sl(n, D == 0 ? gi - 1 : gi, D == 0 ? gj : gj - 1);
            lB[n] = sl(n, gi, gj);
            lo[n] = sc * (lB[n] - lA[n]);
            lo[3 + n] = -sc * lB[n];
            lo[6 + n] = -sc * lA[n];
        }
        lo[9] = 0.0; lo[10] = 0.0;
        const double wA = WB ? sc * p.g * (D == 0 ? lA[1] : lA[2]) : 0.0;
        const double wB = WB ? -sc * p.g * (D == 0 ? lB[1] : lB[2]) : 0.0;
        double lc[4][4];
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int n = 0; n < 4; ++n) lc[k][n] = 0.0;
        if (D == 0) zadj::face_rev<0, WB>(c, p, lo, wA, wB, lc);
        else zadj::face_rev<1, WB>(c, p, lo, wA, wB, lc);
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int n = 0; n < 4; ++n) sF[(4 * k + n) * T::NF + f] = lc[k][n];
    }
    __syncthreads();
    // 4. gather per owned cell, fixed order: direct stencil entries, then
    // entries of ghost cells that mirror onto this cell
    if (owner && i < nx && j < ny) {
#pragma unroll 1
        for (int D = 0; D < 2; ++D) {
            const int ci = D == 0 ? i : j, n_d = D == 0 ? nx : ny;
            const int lo_f = D == 0 ? x0 - 1 : y0 - 1;        // first face index of the tile
            auto face_at = [&](int a) -> int {
                return D == 0 ? (j - y0) * (TX + 3) + (a - lo_f)
                              : T::NFX + (a - lo_f) * TX + (i - x0);
            };
            // face a touches cells a-2 .. a+1 (stencil position k = cell - a + 2)
            for (int a = ci - 1; a <= ci + 2; ++a) {
                if (a < 0 || a > n_d) continue;
                const int fidx = face_at(a);
                const int k = ci - a + 2;
#pragma unroll
                for (int n = 0; n < 4; ++n) acc[n] += sF[(4 * k + n) * T::NF + fidx];
            }
            const int flip = 2 + D;
            const bool wl = (wall >> (2 * D)) & 1u, wh = (wall >> (2 * D + 1)) & 1u;
            if (ci <= 1) {             // ghost g = -1 - ci mirrors onto this cell
                const int g = -1 - ci;
                for (int a = g - 1; a <= g + 2; ++a) {
                    if (a < 0 || a > n_d) continue;
                    const int fidx = face_at(a);
                    const int k = g - a + 2;
#pragma unroll
                    for (int n = 0; n < 4; ++n) {
                        const double v = sF[(4 * k + n) * T::NF + fidx];
                        acc[n] += (n == flip && wl) ? -v : v;
                    }
                }
            }
            if (ci >= n_d - 2) {       // ghost g = 2 n - 1 - ci
                const int g = 2 * n_d - 1 - ci;
                for (int a = g - 1; a <= g + 2; ++a) {
                    if (a < 0 || a > n_d) continue;
                    const int fidx = face_at(a);
                    const int k = g - a + 2;
#pragma unroll
                    for (int n = 0; n < 4; ++n) {
                        const double v = sF[(4 * k + n) * T::NF + fidx];
                        acc[n] += (n == flip && wh) ? -v : v;
                    }
                }
            }
        }
    }
    // 5. lam_X = lam_q* + loc + faces (+ addend)
    if (owner && i < nx && j < ny) {
        const long long c = (long long)j * nx + i;
        double add[4] = {0.0, 0.0, 0.0, 0.0};
        if (addend) {
#pragma unroll
            for (int n = 0; n < 4; ++n) add[n] = addscale * addend[n * pl + c];
        }
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            double v = lamq[n * pl + c] + acc[n];
            if (n == 1) v += loc[c];
            lamX[n * pl + c] = v + add[n];
        }
    }
}

// Per step: reduce the pass-A partials of both stages (dL/dn_m accumulated
// into grad[0]; dL/ddt_n), find the CFL argmax of Q^n and add
// dL/ddt_n * ddt_n/dQ^n there. aux0 (NULL unless this is the run's first
// step): the stored aux whose hinv the first ComputeDt used; otherwise hinv is
// the state's own (the final UpdateState of the previous step).
template <int NT>
__global__ void __launch_bounds__(NT)
k_adj_dt(const double* __restrict__ Q, const double* __restrict__ aux0, int n_aux, P6 L,
         const double* __restrict__ meta, const double* __restrict__ partials, int n_part,
         double* __restrict__ amax_part, unsigned* __restrict__ counter, double* __restrict__ lam,
         double* __restrict__ grad) {
    __shared__ double sv[NT];
    __shared__ long long si[NT];
    __shared__ unsigned s_last;
    const long long pl = L.plane;
    const double g = L.p[0], eps = L.p[5];
    double best = -1.0;
    long long bi = -1;   // cell * 2 + direction
    for (long long c = (long long)blockIdx.x * NT + threadIdx.x; c < pl; c += (long long)gridDim.x * NT) {
        const double h = Q[pl + c];
        const double hv = aux0 ? aux0[(n_aux - 1) * pl + c] : zadj::hinv(h, eps);
        const double cw = sqrt(g * amrex::max(h, 0.0));
#pragma unroll
        for (int d = 0; d < 2; ++d) {
            const double v = (fabs(Q[(2 + d) * pl + c] * hv) + cw) / (d == 0 ? L.dx : L.dy);
            if (v > best) { best = v; bi = 2 * c + d; }
        }
    }
    sv[threadIdx.x] = best;
    si[threadIdx.x] = bi;
    __syncthreads();
    for (int s = NT / 2; s > 0; s >>= 1) {   // max, lowest index on ties
        if (threadIdx.x < s) {
            const double v2 = sv[threadIdx.x + s];
            const long long i2 = si[threadIdx.x + s];
            if (v2 > sv[threadIdx.x] || (v2 == sv[threadIdx.x] && i2 >= 0 && (si[threadIdx.x] < 0 || i2 < si[threadIdx.x]))) {
                sv[threadIdx.x] = v2; si[threadIdx.x] = i2;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        amax_part[2 * blockIdx.x] = sv[0];
        amax_part[2 * blockIdx.x + 1] = double(si[0]);
        __threadfence();
        s_last = (atomicAdd(counter, 1u) == gridDim.x - 1) ? 1u : 0u;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // the argmax over block results (max, lowest index on ties) and the
    // partial sums, all in a fixed order
    best = -1.0; bi = -1;
    double snm = 0.0, sdt = 0.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += NT) {
        const double v = __ldcg(&amax_part[2 * b]);
        const long long ib = (long long)__ldcg(&amax_part[2 * b + 1]);
        if (v > best || (v == best && ib >= 0 && (bi < 0 || ib < bi))) { best = v; bi = ib; }
    }
    for (int b = threadIdx.x; b < n_part; b += NT) {
        snm += __ldcg(&partials[2 * b]);
        sdt += __ldcg(&partials[2 * b + 1]);
    }
    __syncthreads();
    sv[threadIdx.x] = best;
    si[threadIdx.x] = bi;
    __shared__ double s1[NT], s2[NT];
    s1[threadIdx.x] = snm;
    s2[threadIdx.x] = sdt;
    __syncthreads();
    for (int s = NT / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            const double v2 = sv[threadIdx.x + s];
            const long long i2 = si[threadIdx.x + s];
            if (v2 > sv[threadIdx.x] || (v2 == sv[threadIdx.x] && i2 >= 0 && (si[threadIdx.x] < 0 || i2 < si[threadIdx.x]))) {
                sv[threadIdx.x] = v2; si[threadIdx.x] = i2;
            }
            s1[threadIdx.x] += s1[threadIdx.x + s];
            s2[threadIdx.x] += s2[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    const double time_taped = meta[0], dt_taped = meta[1];
    const double M = sv[0];
    const long long idx = si[0];
    snm = s1[0];
    sdt = s2[0];
    grad[0] += snm;
    grad[1] += sdt;            // dL/ddt of the steps so far (diagnostic)
    *counter = 0u;
    // dt = cfl / (div M), unless clamped (dtmin / dtmax / time_end / dry)
    if (M < 1e-14 || idx < 0) return;
    const double div = double(L.cfl_dimension) * double(L.cfl_degree_factor);
    const double dt_free = L.cfl / (div * M);
    double dt = amrex::max(amrex::min(dt_free, L.dtmax), L.dtmin);
    const double remaining = L.time_end - time_taped;
    if (remaining > 0.0 && dt > remaining) dt = remaining;
    if (!(dt == dt_free) || !(dt == dt_taped)) return;
    const double lM = -sdt * dt / M;
    const long long c = idx / 2;
    const int d = int(idx % 2);
    const double h = Q[pl + c], m = Q[(2 + d) * pl + c];
    const double hv = aux0 ? aux0[(n_aux - 1) * pl + c] : zadj::hinv(h, eps);
    const double rd = 1.0 / (d == 0 ? L.dx : L.dy);
    const double u = m * hv;
    const double su = zadj::sgn(u);
    lam[(2 + d) * pl + c] += lM * rd * su * hv;
    double lh = 0.0;
    if (h > 0.0) lh += lM * rd * g / (2.0 * sqrt(g * h));
    if (!aux0) lh += lM * rd * su * m * zadj::dhinv(h, eps);
    lam[pl + c] += lh;
}

}  // namespace adj
}  // namespace zfv
