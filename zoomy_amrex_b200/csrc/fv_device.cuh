// Per-cell and per-face device arithmetic of the finite-volume step, shared by
// every kernel in libzoomyfv.so. Each function restates one piece of the
// reference's Source/make_rhs.H or Source/ZoomyAmr.cpp with the same IEEE
// operation order, so that with --fmad=false the FP64 results are bitwise
// those of the CPU build (which uses -ffp-contract=off).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "AMReX_SmallMatrix.H"
#include "fv_model_traits.H"

namespace zfv {

constexpr int kIdxB = 0;   // constants.H:7
constexpr int kIdxH = 1;   // constants.H:6

// Geometry and run constants of one level, passed to every kernel by value.
template <class R, int NP>
struct LevelParams {
    int nx, ny;
    long long plane;        // elements per component plane (= nx * ny)
    R dx, dy, plox, ploy;
    R p[NP];                // p_mat
    int bc_tag[4];          // x_lo, x_hi, y_lo, y_hi -> Model tag index
    int clamp;              // clamp_positivity && positivity != "mood"
    int well_balanced;
    int implicit_source;
    double cfl, dtmin, dtmax, time_end;
    int max_step;
    int cfl_dimension, cfl_degree_factor;
};

// Device-side run state; the first 64 bytes are zfv_status.
struct alignas(128) DevState {
    double time, dt, mass, max_inv;
    long long step;
    unsigned flags, mood_redos;
    unsigned pad0[4];
    unsigned counter;       // last-block-done counter of the grid reductions
    unsigned troubled;      // MOOD: some cell of this step's order-2 candidate has h < 0 or non-finite
    unsigned parity;        // FP32 form: which ping-pong buffer holds the state (0 = Q, 1 = alt)
    unsigned pad1[13];
};
static_assert(sizeof(DevState) == 128, "DevState layout");

constexpr unsigned kFlagNonfiniteDt = 1u;
constexpr unsigned kFlagMoodRedo = 2u;
constexpr unsigned kFlagDone = 4u;
constexpr unsigned kFlagDeviceWait = 8u;   // a bounded device-side wait gave up: the step is invalid

// ZoomyAmr::UpdateState's per-cell body (ZoomyAmr.cpp:310-331).
template <class Model, class R, class PL>
__device__ __forceinline__ void update_state_cell(typename ModelTypes<Model>::VQ& q,
                                                  typename ModelTypes<Model>::VA& a,
                                                  typename ModelTypes<Model>::VP const& p,
                                                  PL const& L, R time,
                                                  typename ModelTypes<Model>::VX const& X) {
    q = Model::update_variables(q, a, p);
    if (L.clamp && q(kIdxH, 0) < R(0.0)) q(kIdxH, 0) = R(0.0);
    a = Model::update_aux_variables(q, a, p, time, X);
}

template <class Model, class R, class PL>
__device__ __forceinline__ typename ModelTypes<Model>::VX cell_centre(PL const& L, int i, int j) {
    typename ModelTypes<Model>::VX X{};
    X(0, 0) = L.plox + (i + R(0.5)) * L.dx;
    X(1, 0) = (Model::dimension == 2) ? L.ploy + (j + R(0.5)) * L.dy : R(0.0);
    X(2, 0) = R(0.0);
    return X;
}

// Mirror a ghost index about the domain face (ZoomyAmr.cpp:399-406) and pick
// the side whose BC applies, x sides first (ZoomyAmr.cpp:414-422).
template <int DIM>
struct GhostMap {
    int ii, jj, bc_side;    // mirrored interior cell, side 0..3 or -1
    int normal_dir;         // 0 or 1
    int normal_sign;        // -1 or +1
};

template <int DIM>
__device__ __forceinline__ GhostMap<DIM> ghost_map(int i, int j, int nx, int ny) {
    GhostMap<DIM> g;
    g.ii = i; g.jj = j; g.bc_side = -1; g.normal_dir = 0; g.normal_sign = 0;
    if (i < 0) g.ii = -1 - i;
    else if (i > nx - 1) g.ii = 2 * (nx - 1) + 1 - i;
    if (DIM == 2) {
        if (j < 0) g.jj = -1 - j;
        else if (j > ny - 1) g.jj = 2 * (ny - 1) + 1 - j;
    }
    if (i < 0) { g.bc_side = 0; g.normal_dir = 0; g.normal_sign = -1; }
    else if (i > nx - 1) { g.bc_side = 1; g.normal_dir = 0; g.normal_sign = 1; }
    else if (DIM == 2 && j < 0) { g.bc_side = 2; g.normal_dir = 1; g.normal_sign = -1; }
    else if (DIM == 2 && j > ny - 1) { g.bc_side = 3; g.normal_dir = 1; g.normal_sign = 1; }
    return g;
}

// make_rhs.H:9-13
template <class R>
__device__ __forceinline__ R minmod(R a, R b) {
    if (a * b <= R(0.0)) return R(0.0);
    return (fabs(a) < fabs(b)) ? a : b;
}

// One face's numerical flux, fluctuations and Audusse depths
// (make_rhs.H:31-131). qLL, qL, qR, qRR are the (updated) cell states
// iL-1, iL, iR, iR+1 along the face normal DIR.
template <class Model, class Numerics, int ORDER, int DIR, bool WB, class R, class PL>
__device__ __forceinline__ void eval_face(typename ModelTypes<Model>::VQ const& cLL,
                                          typename ModelTypes<Model>::VQ const& cL,
                                          typename ModelTypes<Model>::VQ const& cR,
                                          typename ModelTypes<Model>::VQ const& cRR,
                                          typename ModelTypes<Model>::VA const& aLc,
                                          typename ModelTypes<Model>::VA const& aRc,
                                          typename ModelTypes<Model>::VP const& p, PL const& L,
                                          R time, int iL, int jL, int iR, int jR,
                                          typename ModelTypes<Model>::VQ& flux,
                                          typename ModelTypes<Model>::V2Q& fluct, R& hLs,
                                          R& hRs) {
    using T = ModelTypes<Model>;
    constexpr int nq = Model::n_dof_q;
    typename T::VQ qL, qR;
#pragma unroll
    for (int n = 0; n < nq; ++n) {
        if constexpr (ORDER == 1) {
            qL(n, 0) = cL(n, 0);
            qR(n, 0) = cR(n, 0);
        } else {
            const R gL = minmod(cL(n, 0) - cLL(n, 0), cR(n, 0) - cL(n, 0));
            const R gR = minmod(cR(n, 0) - cL(n, 0), cRR(n, 0) - cR(n, 0));
            qL(n, 0) = cL(n, 0) + R(0.5) * gL;
            qR(n, 0) = cR(n, 0) - R(0.5) * gR;
        }
    }
    hLs = qL(kIdxH, 0);
    hRs = qR(kIdxH, 0);
    if constexpr (WB) {
        const R bL = qL(kIdxB, 0), bR = qR(kIdxB, 0);
        const R bf = amrex::max(bL, bR);
        hLs = amrex::max(R(0.0), qL(kIdxH, 0) + bL - bf);
        hRs = amrex::max(R(0.0), qR(kIdxH, 0) + bR - bf);
        const R sL = (qL(kIdxH, 0) > R(0)) ? hLs / qL(kIdxH, 0) : R(0.0);
        const R sR = (qR(kIdxH, 0) > R(0)) ? hRs / qR(kIdxH, 0) : R(0.0);
#pragma unroll
        for (int d = 0; d < Model::dimension; ++d) {
            qL(kIdxH + 1 + d, 0) *= sL;
            qR(kIdxH + 1 + d, 0) *= sR;
        }
        qL(kIdxH, 0) = hLs; qR(kIdxH, 0) = hRs;
        qL(kIdxB, 0) = bf; qR(kIdxB, 0) = bf;
    }
    const auto XL = cell_centre<Model, R>(L, iL, jL);
    const auto XR = cell_centre<Model, R>(L, iR, jR);
    const typename T::VA aL = Model::update_aux_variables(qL, aLc, p, time, XL);
    const typename T::VA aR = Model::update_aux_variables(qR, aRc, p, time, XR);
    typename T::VN nh{};
    nh(DIR, 0) = R(1.0);
    flux = Numerics::numerical_flux(qL, qR, aL, aR, p, nh);
    fluct = Numerics::numerical_fluctuations(qL, qR, aL, aR, p, nh);
}

// make_rhs.H:429-509 on one cell: q0 (post-explicit-update state, in/out),
// a (stage aux). The dense elimination, register-resident.
template <class Model, class R>
__device__ __forceinline__ void implicit_source_dense(typename ModelTypes<Model>::VQ& q,
                                                     typename ModelTypes<Model>::VA const& a,
                                                     R dt, typename ModelTypes<Model>::VP const& p,
                                                     R time,
                                                     typename ModelTypes<Model>::VX const& X) {
    constexpr int nq = Model::n_dof_q;
    constexpr int na = Model::n_dof_qaux;
    const typename ModelTypes<Model>::VQ q0 = q;
    const auto S = Model::source(q0, a, p, time, X);
    const auto JQ = Model::source_jacobian_wrt_variables(q0, a, p);
    const auto JA = Model::source_jacobian_wrt_aux_variables(q0, a, p);
    const auto AQ = Model::update_aux_variables_jacobian_wrt_variables(q0, a, p, time, X);
    R M[nq][nq], b[nq];
#pragma unroll
    for (int r = 0; r < nq; ++r) {
        b[r] = dt * S(r, 0);
#pragma unroll
        for (int c = 0; c < nq; ++c) {
            R t = JQ(r * nq + c, 0);
#pragma unroll
            for (int k = 0; k < na; ++k) t += JA(r * na + k, 0) * AQ(k * nq + c, 0);
            M[r][c] = (r == c ? R(1.0) : R(0.0)) - dt * t;
        }
    }
    // Register-resident elimination: every loop has a constant trip count
    // (inner ranges such as c >= k are guards, not bounds, so the compiler
    // unrolls inner loops before outer ones and every index is a constant),
    // rows are swapped by selecting through the unrolled rows, and there is
    // no early exit: once a pivot fails, the remaining arithmetic runs on
    // values that are then discarded for the explicit fallback, as the
    // reference's early exit discards them. The operations on the kept
    // values are the reference's, in its order.
    bool ok = true;
#pragma unroll
    for (int k = 0; k < nq; ++k) {
        int piv = k;
        R best = fabs(M[k][k]);
#pragma unroll
        for (int r = 0; r < nq; ++r)
            if (r > k && fabs(M[r][k]) > best) { best = fabs(M[r][k]); piv = r; }
        ok = ok && (best > R(0.0)) && isfinite(best);
#pragma unroll
        for (int r = 0; r < nq; ++r) {
            if (r > k && r == piv) {
#pragma unroll
                for (int c = 0; c < nq; ++c)
                    if (c >= k) { R t = M[k][c]; M[k][c] = M[r][c]; M[r][c] = t; }
                R t = b[k]; b[k] = b[r]; b[r] = t;
            }
        }
#pragma unroll
        for (int r = 0; r < nq; ++r) {
            if (r <= k) continue;
            const R f = M[r][k] / M[k][k];
#pragma unroll
            for (int c = 0; c < nq; ++c)
                if (c >= k) M[r][c] -= f * M[k][c];
            b[r] -= f * b[k];
        }
    }
    if (ok) {
        R dq[nq];
#pragma unroll
        for (int r = nq - 1; r >= 0; --r) {
            R s = R(0.0);
#pragma unroll
            for (int c = 0; c < nq; ++c)
                if (c > r) s += M[r][c] * dq[c];
            dq[r] = (b[r] - s) / M[r][r];
            ok = ok && isfinite(dq[r]);
        }
        if (ok) {
#pragma unroll
            for (int n = 0; n < nq; ++n) q(n, 0) = q0(n, 0) + dq[n];
            return;
        }
    }
#pragma unroll
    for (int n = 0; n < nq; ++n) {
        const R v = q0(n, 0) + dt * S(n, 0);
        q(n, 0) = isfinite(v) ? v : q0(n, 0);
    }
}

// The same elimination out of line, its matrix in local memory (runtime
// loops): the structured path below falls back to it for the rare cells
// whose system does not have the declared structure, without raising the
// calling kernel's register count. The operations are the reference's, in
// its order.
template <class Model, class R>
__device__ __noinline__ void implicit_source_outline(typename ModelTypes<Model>::VQ& q,
                                                     typename ModelTypes<Model>::VA const& a,
                                                     R dt, typename ModelTypes<Model>::VP const& p,
                                                     R time,
                                                     typename ModelTypes<Model>::VX const& X) {
    constexpr int nq = Model::n_dof_q;
    constexpr int na = Model::n_dof_qaux;
    const typename ModelTypes<Model>::VQ q0 = q;
    const auto S = Model::source(q0, a, p, time, X);
    const auto JQ = Model::source_jacobian_wrt_variables(q0, a, p);
    const auto JA = Model::source_jacobian_wrt_aux_variables(q0, a, p);
    const auto AQ = Model::update_aux_variables_jacobian_wrt_variables(q0, a, p, time, X);
    R M[nq][nq], b[nq], dq[nq];
#pragma unroll 1
    for (int r = 0; r < nq; ++r) {
        b[r] = dt * S(r, 0);
#pragma unroll 1
        for (int c = 0; c < nq; ++c) {
            R t = JQ(r * nq + c, 0);
#pragma unroll 1
            for (int k = 0; k < na; ++k) t += JA(r * na + k, 0) * AQ(k * nq + c, 0);
            M[r][c] = (r == c ? R(1.0) : R(0.0)) - dt * t;
        }
    }
    bool ok = true;
#pragma unroll 1
    for (int k = 0; k < nq && ok; ++k) {
        int piv = k;
        R best = fabs(M[k][k]);
#pragma unroll 1
        for (int r = k + 1; r < nq; ++r)
            if (fabs(M[r][k]) > best) { best = fabs(M[r][k]); piv = r; }
        if (!(best > R(0.0)) || !isfinite(best)) { ok = false; break; }
        if (piv != k) {
#pragma unroll 1
            for (int c = k; c < nq; ++c) { const R t = M[k][c]; M[k][c] = M[piv][c]; M[piv][c] = t; }
            const R t = b[k]; b[k] = b[piv]; b[piv] = t;
        }
#pragma unroll 1
        for (int r = k + 1; r < nq; ++r) {
            const R f = M[r][k] / M[k][k];
#pragma unroll 1
            for (int c = k; c < nq; ++c) M[r][c] -= f * M[k][c];
            b[r] -= f * b[k];
        }
    }
#pragma unroll 1
    for (int r = nq - 1; r >= 0 && ok; --r) {
        R s = R(0.0);
#pragma unroll 1
        for (int c = r + 1; c < nq; ++c) s += M[r][c] * dq[c];
        dq[r] = (b[r] - s) / M[r][r];
        if (!isfinite(dq[r])) ok = false;
    }
    if (ok) {
#pragma unroll 1
        for (int n = 0; n < nq; ++n) q(n, 0) = q0(n, 0) + dq[n];
        return;
    }
#pragma unroll 1
    for (int n = 0; n < nq; ++n) {
        const R v = q0(n, 0) + dt * S(n, 0);
        q(n, 0) = isfinite(v) ? v : q0(n, 0);
    }
}

// The same system solved block by block, for models that declare the
// structure (zb_implicit_blocks, fv_model_traits.H). With rows 0 and 1 of
// the system the identity (zero source, zero off-diagonal entries in their
// rows and in column 0, no pivot in column 1), the reference's first two
// elimination steps change no nonzero value; with no entry coupling two
// blocks, every later step's pivot search, row swaps, eliminations and the
// back substitution touch other blocks' rows only through products with
// zeros. So solving each block with the reference's operations in the
// reference's order gives the reference's result (up to the sign of zero
// entries), with n_b small matrices in registers instead of one n x n. A
// cell whose system breaks the preconditions takes the full elimination.
template <class Model, class R>
__device__ __forceinline__ void implicit_source_blocks(typename ModelTypes<Model>::VQ& q,
                                                       typename ModelTypes<Model>::VA const& a,
                                                       R dt, typename ModelTypes<Model>::VP const& p,
                                                       R time,
                                                       typename ModelTypes<Model>::VX const& X) {
    constexpr int nq = Model::n_dof_q;
    constexpr int na = Model::n_dof_qaux;
    constexpr int NB = Model::zb_implicit_blocks, BS = Model::zb_implicit_block_size;
    static_assert(2 + NB * BS == nq, "the blocks and rows 0, 1 cover the state");
    const typename ModelTypes<Model>::VQ q0 = q;
    const auto S = Model::source(q0, a, p, time, X);
    const auto JQ = Model::source_jacobian_wrt_variables(q0, a, p);
    const auto JA = Model::source_jacobian_wrt_aux_variables(q0, a, p);
    const auto AQ = Model::update_aux_variables_jacobian_wrt_variables(q0, a, p, time, X);
    // an entry of I - dt J, formed as the reference forms it
    auto m = [&](int r, int c) -> R {
        R t = JQ(r * nq + c, 0);
#pragma unroll
        for (int k = 0; k < na; ++k) t += JA(r * na + k, 0) * AQ(k * nq + c, 0);
        return (r == c ? R(1.0) : R(0.0)) - dt * t;
    };
    const R m00 = m(0, 0), m11 = m(1, 1);
    bool pre = (m00 > R(0.0)) && isfinite(m00) && (m11 > R(0.0)) && isfinite(m11) &&
               (dt * S(0, 0) == R(0.0)) && (dt * S(1, 0) == R(0.0));
#pragma unroll
    for (int c = 1; c < nq; ++c) pre = pre && (m(c, 0) == R(0.0)) && (m(0, c) == R(0.0));
#pragma unroll
    for (int c = 2; c < nq; ++c) pre = pre && (m(1, c) == R(0.0)) && !(fabs(m(c, 1)) > m11);
    if (!pre) {
        implicit_source_outline<Model, R>(q, a, dt, p, time, X);
        return;
    }
    R dq[NB][BS];
    bool ok = true;
#pragma unroll
    for (int bi = 0; bi < NB; ++bi) {
        R A[BS][BS], b[BS];
#pragma unroll
        for (int r = 0; r < BS; ++r) {
            const int rr = Model::zb_implicit_row(bi, r);
            b[r] = dt * S(rr, 0);
#pragma unroll
            for (int c = 0; c < BS; ++c) A[r][c] = m(rr, Model::zb_implicit_row(bi, c));
        }
#pragma unroll
        for (int k = 0; k < BS; ++k) {
            int piv = k;
            R best = fabs(A[k][k]);
#pragma unroll
            for (int r = 0; r < BS; ++r)
                if (r > k && fabs(A[r][k]) > best) { best = fabs(A[r][k]); piv = r; }
            ok = ok && (best > R(0.0)) && isfinite(best);
#pragma unroll
            for (int r = 0; r < BS; ++r) {
                if (r > k && r == piv) {
#pragma unroll
                    for (int c = 0; c < BS; ++c)
                        if (c >= k) { const R t = A[k][c]; A[k][c] = A[r][c]; A[r][c] = t; }
                    const R t = b[k]; b[k] = b[r]; b[r] = t;
                }
            }
#pragma unroll
            for (int r = 0; r < BS; ++r) {
                if (r <= k) continue;
                const R f = A[r][k] / A[k][k];
#pragma unroll
                for (int c = 0; c < BS; ++c)
                    if (c >= k) A[r][c] -= f * A[k][c];
                b[r] -= f * b[k];
            }
        }
#pragma unroll
        for (int r = BS - 1; r >= 0; --r) {
            R s = R(0.0);
#pragma unroll
            for (int c = 0; c < BS; ++c)
                if (c > r) s += A[r][c] * dq[bi][c];
            dq[bi][r] = (b[r] - s) / A[r][r];
            ok = ok && isfinite(dq[bi][r]);
        }
    }
    if (ok) {
        // rows 0 and 1: (0 - 0) / 1 = +0 in the reference
        q(0, 0) = q0(0, 0) + R(0.0);
        q(1, 0) = q0(1, 0) + R(0.0);
#pragma unroll
        for (int bi = 0; bi < NB; ++bi)
#pragma unroll
            for (int r = 0; r < BS; ++r) {
                const int rr = Model::zb_implicit_row(bi, r);
                q(rr, 0) = q0(rr, 0) + dq[bi][r];
            }
        return;
    }
#pragma unroll
    for (int n = 0; n < nq; ++n) {
        const R v = q0(n, 0) + dt * S(n, 0);
        q(n, 0) = isfinite(v) ? v : q0(n, 0);
    }
}

// make_rhs.H:429-509 on one cell: the structured elimination where the model
// declares its blocks, the dense one otherwise.
template <class Model, class R>
__device__ __forceinline__ void implicit_source_cell(typename ModelTypes<Model>::VQ& q,
                                                     typename ModelTypes<Model>::VA const& a,
                                                     R dt, typename ModelTypes<Model>::VP const& p,
                                                     R time,
                                                     typename ModelTypes<Model>::VX const& X) {
    if constexpr (implicit_blocks<Model>::value) implicit_source_blocks<Model, R>(q, a, dt, p, time, X);
    else implicit_source_dense<Model, R>(q, a, dt, p, time, X);
}

// Per-cell CFL quantity of ZoomyAmr::ComputeDt (ZoomyAmr.cpp:472-487).
template <class Model, class Numerics, class R, class PL>
__device__ __forceinline__ R cell_max_inv(typename ModelTypes<Model>::VQ const& q,
                                          typename ModelTypes<Model>::VA const& a,
                                          typename ModelTypes<Model>::VP const& p, PL const& L) {
    R m = R(0.0);
#pragma unroll
    for (int d = 0; d < Model::dimension; ++d) {
        typename ModelTypes<Model>::VN nh{};
        nh(d, 0) = R(1.0);
        const auto ev = Numerics::local_max_abs_eigenvalue(q, a, p, nh);
        const R inv = ev(0, 0) / (d == 0 ? L.dx : L.dy);
        if (inv > m) m = inv;
    }
    return m;
}

// dt from the global max (ZoomyAmr.cpp:499-514) and TimeStep's clamp to
// time_end (ZoomyAmr.cpp:746-749).
template <class PL>
__device__ __forceinline__ double dt_from_max(double gmax, double time, PL const& L) {
    double dt;
    if (gmax < 1e-14) {
        dt = L.dtmax;
    } else {
        const double div = double(L.cfl_dimension) * double(L.cfl_degree_factor);
        dt = L.cfl / (div * gmax);
        dt = amrex::max(amrex::min(dt, L.dtmax), L.dtmin);
    }
    const double remaining = L.time_end - time;
    if (remaining > 0.0 && dt > remaining) dt = remaining;
    return dt;
}

template <class PL>
__device__ __forceinline__ bool run_done(double time, long long step, PL const& L) {
    return !(time < L.time_end && (L.max_step < 0 || step < (long long)L.max_step));
}

}  // namespace zfv
