// CPU oracle for the zoomy-amrex hot path — TEST INFRASTRUCTURE ONLY.
//
// This is a plain C++ restatement of the reference's per-level finite-volume
// step, used to check the sm_100a kernels: Source/make_rhs.H (face
// reconstruction, fluxes, cell RHS, point-implicit source) and the
// single-level driver in Source/ZoomyAmr.cpp (UpdateState, FillPhysicalBC_mf,
// ComputeDt, ComputeTotalMass, Advance with MOOD, TimeStep, Evolve), plus
// init_solution (Source/init_solution.cpp:78-116). Nothing in the product
// links or calls it; only tests/, the smoke check and the benchmark's CPU
// baseline do.
//
// The level is one grown array per field (valid cells plus ng ghost layers
// on every side, ng = 2 at order 2, 1 at order 1: ZoomyAmr.H:152), laid out
// like an AMReX FArrayBox: component-major, x fastest. The reference splits a
// level into boxes of at most amr.max_grid_size cells; its results are
// decomposition-invariant (tests/test_parallel_two_ranks.py:56-57 asserts
// bit-identity), so one box is the same computation.
//
// The per-cell arithmetic is reached through a Kernels policy so the same
// driver runs either this file's restatement of make_rhs.H (OracleKernels) or
// the reference's own make_rhs.H compiled against the AMReX API shim
// (oracle/ref_*.cpp, built into oracle/_ref/).
//
// Build with -ffp-contract=off: the reference's CUDA build disables FMA
// contraction (build.py:33-41) and the sm_100a kernels are built with
// --fmad=false, so all three evaluate the same IEEE operations.
#pragma once
#include <vector>
#include <cmath>
#include <cstring>
#include <cstdint>
#include <algorithm>
#include "AMReX_Array4.H"
#include "AMReX_SmallMatrix.H"
#include "zoomy_fv.h"

namespace zoracle {

using Real = double;
constexpr int kIdxB = 0;   // constants.H:7
constexpr int kIdxH = 1;   // constants.H:6

// ---------------------------------------------------------------------------
// Restatement of Source/make_rhs.H (per-face and per-cell arithmetic).
// ---------------------------------------------------------------------------
template <class Model, class Numerics>
struct OracleKernels {
    static constexpr int nq = Model::n_dof_q;
    static constexpr int na = Model::n_dof_qaux;
    static constexpr int np = Model::n_parameters;
    static constexpr int dim = Model::dimension;
    using VQ = amrex::SmallMatrix<Real, nq, 1>;
    using VA = amrex::SmallMatrix<Real, na, 1>;
    using VP = amrex::SmallMatrix<Real, np, 1>;
    using VX = amrex::SmallMatrix<Real, 3, 1>;
    using A4c = amrex::Array4<const Real>;
    using A4 = amrex::Array4<Real>;

    // make_rhs.H:9-13: zero on a sign change, else the smaller magnitude
    static Real limiter(Real a, Real b) {
        if (a * b <= 0.0) return 0.0;
        return (std::abs(a) < std::abs(b)) ? a : b;
    }

    // make_rhs.H:17-26
    static VX centre(int i, int j, Real dx, Real dy, Real plox, Real ploy) {
        VX X{};
        X(0, 0) = plox + (i + 0.5) * dx;
        X(1, 0) = (dim == 2) ? ploy + (j + 0.5) * dy : Real(0.0);
        X(2, 0) = Real(0.0);
        return X;
    }

    struct Face {
        VQ flux;
        amrex::SmallMatrix<Real, 2 * nq, 1> fluct;   // D+ at [n], D- at [nq + n]
        Real hstar_l, hstar_r;
    };

    // make_rhs.H:31-131 (eval_face): left state from cell (iL,jL), right from (iR,jR)
    static Face face(int iL, int jL, int iR, int jR, int dir, int order, A4c const& Q,
                     A4c const& Qa, VP const& p, Real time, Real dx, Real dy, Real plox,
                     Real ploy, bool wb) {
        VQ qL, qR;
        const int si = (dir == 0) ? 1 : 0, sj = (dir == 0) ? 0 : 1;
        for (int n = 0; n < nq; ++n) {
            const Real cL = Q(iL, jL, 0, n), cR = Q(iR, jR, 0, n);
            if (order == 1) {
                qL(n, 0) = cL;
                qR(n, 0) = cR;
            } else {
                const Real sL = limiter(cL - Q(iL - si, jL - sj, 0, n), Q(iL + si, jL + sj, 0, n) - cL);
                const Real sR = limiter(cR - Q(iR - si, jR - sj, 0, n), Q(iR + si, jR + sj, 0, n) - cR);
                qL(n, 0) = cL + 0.5 * sL;
                qR(n, 0) = cR - 0.5 * sR;
            }
        }
        // make_rhs.H:84-98: Audusse hydrostatic reconstruction about b_face = max(bL, bR)
        Real hl = qL(kIdxH, 0), hr = qR(kIdxH, 0);
        if (wb) {
            const Real bL = qL(kIdxB, 0), bR = qR(kIdxB, 0);
            const Real bf = amrex::max(bL, bR);
            hl = amrex::max(Real(0.0), qL(kIdxH, 0) + bL - bf);
            hr = amrex::max(Real(0.0), qR(kIdxH, 0) + bR - bf);
            const Real fl = (qL(kIdxH, 0) > Real(0)) ? hl / qL(kIdxH, 0) : Real(0.0);
            const Real fr = (qR(kIdxH, 0) > Real(0)) ? hr / qR(kIdxH, 0) : Real(0.0);
            for (int d = 0; d < dim; ++d) {
                qL(kIdxH + 1 + d, 0) *= fl;
                qR(kIdxH + 1 + d, 0) *= fr;
            }
            qL(kIdxH, 0) = hl; qR(kIdxH, 0) = hr;
            qL(kIdxB, 0) = bf; qR(kIdxB, 0) = bf;
        }
        VA aL, aR;
        for (int n = 0; n < na; ++n) { aL(n, 0) = Qa(iL, jL, 0, n); aR(n, 0) = Qa(iR, jR, 0, n); }
        aL = Model::update_aux_variables(qL, aL, p, time, centre(iL, jL, dx, dy, plox, ploy));
        aR = Model::update_aux_variables(qR, aR, p, time, centre(iR, jR, dx, dy, plox, ploy));
        amrex::SmallMatrix<Real, dim, 1> nh{};
        nh(dir, 0) = 1.0;
        Face f;
        f.flux = Numerics::numerical_flux(qL, qR, aL, aR, p, nh);
        f.fluct = Numerics::numerical_fluctuations(qL, qR, aL, aR, p, nh);
        f.hstar_l = hl;
        f.hstar_r = hr;
        return f;
    }

    // make_rhs.H:142-147
    static Real divergence(Real f_r, Real f_l, Real dm_r, Real dp_l) { return -(f_r - f_l) - dm_r - dp_l; }

    // make_rhs.H:234-290 (cell-centric RHS: each face evaluated from the cell's side)
    static void cell_rhs(int i, int j, A4c const& Q, A4c const& Qa, A4 const& RHS, Real dx, Real dy,
                         int order, bool implicit_source, VP const& p, Real time, Real plox,
                         Real ploy, bool wb) {
        const Face xr = face(i, j, i + 1, j, 0, order, Q, Qa, p, time, dx, dy, plox, ploy, wb);
        const Face xl = face(i - 1, j, i, j, 0, order, Q, Qa, p, time, dx, dy, plox, ploy, wb);
        Face yr{}, yl{};
        if constexpr (dim == 2) {
            yr = face(i, j, i, j + 1, 1, order, Q, Qa, p, time, dx, dy, plox, ploy, wb);
            yl = face(i, j - 1, i, j, 1, order, Q, Qa, p, time, dx, dy, plox, ploy, wb);
        }
        assemble_from(i, j, Q, Qa, RHS, dx, dy, implicit_source, p, time, plox, ploy, wb, xr, xl, yr, yl);
    }

    static void assemble_from(int i, int j, A4c const& Q, A4c const& Qa, A4 const& RHS, Real dx,
                              Real dy, bool implicit_source, VP const& p, Real time, Real plox,
                              Real ploy, bool wb, Face const& xr, Face const& xl, Face const& yr,
                              Face const& yl) {
        VQ q, S;
        VA a;
        for (int n = 0; n < nq; ++n) q(n, 0) = Q(i, j, 0, n);
        for (int n = 0; n < na; ++n) a(n, 0) = Qa(i, j, 0, n);
        for (int n = 0; n < nq; ++n) S(n, 0) = 0.0;
        if (!implicit_source) S = Model::source(q, a, p, time, centre(i, j, dx, dy, plox, ploy));
        for (int n = 0; n < nq; ++n) {
            const Real Fx = divergence(xr.flux(n, 0), xl.flux(n, 0), xr.fluct(nq + n, 0), xl.fluct(n, 0));
            Real Fy = 0.0;
            if constexpr (dim == 2)
                Fy = divergence(yr.flux(n, 0), yl.flux(n, 0), yr.fluct(nq + n, 0), yl.fluct(n, 0));
            RHS(i, j, 0, n) = Fx / dx + Fy / dy;
            if (!implicit_source) RHS(i, j, 0, n) += S(n, 0);
        }
        if (wb) {   // make_rhs.H:154-163 with g = p(0)
            const Real g = p(0, 0);
            RHS(i, j, 0, kIdxH + 1) += 0.5 * g * (xr.hstar_l * xr.hstar_l - xl.hstar_r * xl.hstar_r) / dx;
            if constexpr (dim == 2)
                RHS(i, j, 0, kIdxH + 2) += 0.5 * g * (yr.hstar_l * yr.hstar_l - yl.hstar_r * yl.hstar_r) / dy;
        }
        static_assert(!Model::has_diffusion, "diffusive models are not restated");
    }

    // make_rhs.H:315-342: face (i,j) in direction dir sits between cell
    // (i-1,j)|(i,j-1) and (i,j). Stored as flux[nq], fluct[2nq], h*_L, h*_R.
    static constexpr int n_face_comp = 3 * nq + 2;
    static void face_data(int i, int j, int dir, int order, A4c const& Q, A4c const& Qa,
                          A4 const& F, VP const& p, Real time, Real dx, Real dy, Real plox,
                          Real ploy, bool wb) {
        const int iL = (dir == 0) ? i - 1 : i, jL = (dir == 1) ? j - 1 : j;
        const Face f = face(iL, jL, i, j, dir, order, Q, Qa, p, time, dx, dy, plox, ploy, wb);
        for (int n = 0; n < nq; ++n) F(i, j, 0, n) = f.flux(n, 0);
        for (int n = 0; n < 2 * nq; ++n) F(i, j, 0, nq + n) = f.fluct(n, 0);
        F(i, j, 0, 3 * nq) = f.hstar_l;
        F(i, j, 0, 3 * nq + 1) = f.hstar_r;
    }

    static Face load_face(A4c const& F, int i, int j) {
        Face f;
        for (int n = 0; n < nq; ++n) f.flux(n, 0) = F(i, j, 0, n);
        for (int n = 0; n < 2 * nq; ++n) f.fluct(n, 0) = F(i, j, 0, nq + n);
        f.hstar_l = F(i, j, 0, 3 * nq);
        f.hstar_r = F(i, j, 0, 3 * nq + 1);
        return f;
    }

    // make_rhs.H:346-399
    static void assemble(int i, int j, A4c const& Q, A4c const& Qa, A4c const& Fx, A4c const& Fy,
                         A4 const& RHS, Real dx, Real dy, bool implicit_source, VP const& p,
                         Real time, Real plox, Real ploy, bool wb) {
        const Face xr = load_face(Fx, i + 1, j), xl = load_face(Fx, i, j);
        Face yr{}, yl{};
        if constexpr (dim == 2) { yr = load_face(Fy, i, j + 1); yl = load_face(Fy, i, j); }
        assemble_from(i, j, Q, Qa, RHS, dx, dy, implicit_source, p, time, plox, ploy, wb, xr, xl, yr, yl);
    }

    // make_rhs.H:429-509: one linearised backward-Euler source step,
    // (I - dt J) dq = dt S, J = dS/dQ + dS/dA dA/dQ, solved by Gaussian
    // elimination with partial pivoting; explicit fallback if singular.
    static void implicit_source(int i, int j, A4 const& Q, A4c const& Qa, Real dt, VP const& p,
                                Real time, VX const& X) {
        VQ q0;
        VA a;
        for (int n = 0; n < nq; ++n) q0(n, 0) = Q(i, j, 0, n);
        for (int n = 0; n < na; ++n) a(n, 0) = Qa(i, j, 0, n);
        const auto S = Model::source(q0, a, p, time, X);
        const auto JQ = Model::source_jacobian_wrt_variables(q0, a, p);
        const auto JA = Model::source_jacobian_wrt_aux_variables(q0, a, p);
        const auto AQ = Model::update_aux_variables_jacobian_wrt_variables(q0, a, p, time, X);
        Real M[nq][nq], b[nq];
        for (int r = 0; r < nq; ++r) {
            b[r] = dt * S(r, 0);
            for (int c = 0; c < nq; ++c) {
                Real t = JQ(r * nq + c, 0);
                for (int k = 0; k < na; ++k) t += JA(r * na + k, 0) * AQ(k * nq + c, 0);
                M[r][c] = (r == c ? 1.0 : 0.0) - dt * t;
            }
        }
        bool ok = true;
        for (int k = 0; k < nq && ok; ++k) {
            int piv = k;
            Real best = std::abs(M[k][k]);
            for (int r = k + 1; r < nq; ++r)
                if (std::abs(M[r][k]) > best) { best = std::abs(M[r][k]); piv = r; }
            if (!(best > 0.0) || !std::isfinite(best)) { ok = false; break; }
            if (piv != k) {
                for (int c = k; c < nq; ++c) std::swap(M[k][c], M[piv][c]);
                std::swap(b[k], b[piv]);
            }
            for (int r = k + 1; r < nq; ++r) {
                const Real f = M[r][k] / M[k][k];
                for (int c = k; c < nq; ++c) M[r][c] -= f * M[k][c];
                b[r] -= f * b[k];
            }
        }
        if (ok) {
            Real dq[nq];
            for (int r = nq - 1; r >= 0; --r) {
                Real s = 0.0;
                for (int c = r + 1; c < nq; ++c) s += M[r][c] * dq[c];
                dq[r] = (b[r] - s) / M[r][r];
                if (!std::isfinite(dq[r])) { ok = false; break; }
            }
            if (ok) {
                for (int n = 0; n < nq; ++n) Q(i, j, 0, n) = q0(n, 0) + dq[n];
                return;
            }
        }
        for (int n = 0; n < nq; ++n) {
            const Real v = q0(n, 0) + dt * S(n, 0);
            Q(i, j, 0, n) = std::isfinite(v) ? v : q0(n, 0);
        }
    }
};

// ---------------------------------------------------------------------------
// Restatement of the single-level driver in Source/ZoomyAmr.cpp.
// ---------------------------------------------------------------------------
// solver.implicit_global (imex_solver.H:102-160) solves
// F(Q) = Q - Qexp - dt S(Q) = 0 for the whole field by Jacobian-free
// Newton-Krylov, with S evaluated on aux refreshed from the state
// (ComputeSourceField, :21-58). For a cell-local source that system is one
// small system per cell; this solves each one exactly (Newton with the
// model's analytic source Jacobian, to round-off): the answer the field solve
// approaches within its stopping rule (|F| < 1e-9 |F_0|).
template <class Model, class A4, class VP, class VX>
void implicit_source_exact(int i, int j, A4 const& Q, Real dt, VP const& p, Real time, VX const& X) {
    constexpr int nq = Model::n_dof_q;
    using VQ = amrex::SmallMatrix<Real, nq, 1>;
    using VA = amrex::SmallMatrix<Real, Model::n_dof_qaux, 1>;
    VQ qe, q;
    for (int n = 0; n < nq; ++n) qe(n, 0) = q(n, 0) = Q(i, j, 0, n);
    for (int it = 0; it < 50; ++it) {
        VA a;
        for (int n = 0; n < Model::n_dof_qaux; ++n) a(n, 0) = 0.0;
        a = Model::update_aux_variables(q, a, p, time, X);
        const auto S = Model::source(q, a, p, time, X);
        const auto JQ = Model::source_jacobian_wrt_variables(q, a, p);
        Real M[nq][nq], b[nq], fmax = 0.0, qmax = 0.0;
        for (int r = 0; r < nq; ++r) {
            b[r] = -((q(r, 0) - qe(r, 0)) - dt * S(r, 0));
            fmax = std::max(fmax, std::abs(b[r]));
            qmax = std::max(qmax, std::abs(q(r, 0)));
            for (int c = 0; c < nq; ++c) M[r][c] = (r == c ? 1.0 : 0.0) - dt * JQ(r * nq + c, 0);
        }
        if (!(fmax > 1e-16 * (1.0 + qmax))) break;
        for (int k = 0; k < nq; ++k) {      // Gaussian elimination, partial pivoting
            int piv = k;
            for (int r = k + 1; r < nq; ++r)
                if (std::abs(M[r][k]) > std::abs(M[piv][k])) piv = r;
            if (!(std::abs(M[piv][k]) > 0.0)) return;
            if (piv != k) {
                for (int c = k; c < nq; ++c) std::swap(M[k][c], M[piv][c]);
                std::swap(b[k], b[piv]);
            }
            for (int r = k + 1; r < nq; ++r) {
                const Real f = M[r][k] / M[k][k];
                for (int c = k; c < nq; ++c) M[r][c] -= f * M[k][c];
                b[r] -= f * b[k];
            }
        }
        for (int r = nq - 1; r >= 0; --r) {
            Real t = b[r];
            for (int c = r + 1; c < nq; ++c) t -= M[r][c] * b[c];
            b[r] = t / M[r][r];
        }
        for (int n = 0; n < nq; ++n) q(n, 0) += b[n];
    }
    for (int n = 0; n < nq; ++n) Q(i, j, 0, n) = q(n, 0);
}

struct StepLog { Real dt, time, mass; };

template <class Model, class Numerics, class K>
struct Level {
    static constexpr int nq = Model::n_dof_q;
    static constexpr int na = Model::n_dof_qaux;
    static constexpr int np = Model::n_parameters;
    static constexpr int dim = Model::dimension;
    using VQ = amrex::SmallMatrix<Real, nq, 1>;
    using VA = amrex::SmallMatrix<Real, na, 1>;
    using VP = amrex::SmallMatrix<Real, np, 1>;
    using VX = amrex::SmallMatrix<Real, 3, 1>;

    zfv_config cfg;
    int nx, ny, ng, gx, gy;
    Real dx, dy, plox, ploy;
    VP p;
    std::vector<Real> Q, Qa, Rhs, Qold, Fx, Fy;
    Real time = 0.0;
    int64_t step = 0;
    int mood_redos = 0;
    std::vector<StepLog> log;

    explicit Level(const zfv_config& c) : cfg(c) {
        nx = c.nx; ny = c.ny;
        ng = (c.spatial_order == 2) ? 2 : 1;            // ZoomyAmr.H:152
        gx = nx + 2 * ng; gy = ny + 2 * ng;
        dx = (c.prob_hi[0] - c.prob_lo[0]) / nx;
        dy = (c.prob_hi[1] - c.prob_lo[1]) / ny;
        plox = c.prob_lo[0]; ploy = c.prob_lo[1];
        for (int k = 0; k < np; ++k) p(k, 0) = c.params[k];
        Q.assign(size_t(gx) * gy * nq, 0.0);
        Qa.assign(size_t(gx) * gy * na, 0.0);
        Rhs.assign(size_t(gx) * gy * nq, 0.0);
        Qold.assign(size_t(gx) * gy * nq, 0.0);
    }

    amrex::Array4<Real> arr(std::vector<Real>& v, int ncomp, int bx = -1, int by = -1) {
        if (bx < 0) { bx = gx; by = gy; }
        return amrex::Array4<Real>(v.data(), {-ng, -ng, 0}, {-ng + bx, -ng + by, 1}, ncomp);
    }
    amrex::Array4<Real> aQ() { return arr(Q, nq); }
    amrex::Array4<Real> aA() { return arr(Qa, na); }

    VX centre(int i, int j) const {
        VX X{};
        X(0, 0) = plox + (i + 0.5) * dx;
        X(1, 0) = (dim == 2) ? ploy + (j + 0.5) * dy : Real(0.0);
        X(2, 0) = Real(0.0);
        return X;
    }

    // valid arrays (n, ny, nx) <-> grown storage
    void load(const Real* Qv, const Real* Av) {
        auto q = aQ(); auto a = aA();
        for (int n = 0; n < nq; ++n)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) q(i, j, 0, n) = Qv[(size_t(n) * ny + j) * nx + i];
        for (int n = 0; n < na; ++n)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) a(i, j, 0, n) = Av[(size_t(n) * ny + j) * nx + i];
    }
    void store(Real* Qv, Real* Av) {
        auto q = aQ(); auto a = aA();
        if (Qv)
            for (int n = 0; n < nq; ++n)
                for (int j = 0; j < ny; ++j)
                    for (int i = 0; i < nx; ++i) Qv[(size_t(n) * ny + j) * nx + i] = q(i, j, 0, n);
        if (Av)
            for (int n = 0; n < na; ++n)
                for (int j = 0; j < ny; ++j)
                    for (int i = 0; i < nx; ++i) Av[(size_t(n) * ny + j) * nx + i] = a(i, j, 0, n);
    }

    // ZoomyAmr.cpp:293-334, over the grown box
    void update_state(Real t) {
        const bool clamp = cfg.clamp_positivity && !cfg.positivity_mood;   // :303
        auto q4 = aQ(); auto a4 = aA();
#pragma omp parallel for schedule(static)
        for (int j = -ng; j < ny + ng; ++j)
            for (int i = -ng; i < nx + ng; ++i) {
                VQ q; VA a;
                for (int n = 0; n < nq; ++n) q(n, 0) = q4(i, j, 0, n);
                for (int n = 0; n < na; ++n) a(n, 0) = a4(i, j, 0, n);
                q = Model::update_variables(q, a, p);
                if (clamp && q(kIdxH, 0) < 0.0) q(kIdxH, 0) = 0.0;
                a = Model::update_aux_variables(q, a, p, t, centre(i, j));
                for (int n = 0; n < nq; ++n) q4(i, j, 0, n) = q(n, 0);
                for (int n = 0; n < na; ++n) a4(i, j, 0, n) = a(n, 0);
            }
    }

    // ZoomyAmr.cpp:342-443: reflect the ghost index about the domain face and
    // apply Model::boundary_conditions; x sides take precedence at corners.
    void fill_physical_bc(Real t) {
        auto q4 = aQ(); auto a4 = aA();
        const int lo_x = 0, hi_x = nx - 1, lo_y = 0, hi_y = ny - 1;
#pragma omp parallel for schedule(static)
        for (int j = -ng; j < ny + ng; ++j)
            for (int i = -ng; i < nx + ng; ++i) {
                const bool out_x = (i < lo_x || i > hi_x);
                const bool out_y = (dim == 2) && (j < lo_y || j > hi_y);
                if (!out_x && !out_y) continue;
                int ii = i, jj = j;
                if (i < lo_x) ii = 2 * lo_x - 1 - i;
                else if (i > hi_x) ii = 2 * hi_x + 1 - i;
                if (dim == 2) {
                    if (j < lo_y) jj = 2 * lo_y - 1 - j;
                    else if (j > hi_y) jj = 2 * hi_y + 1 - j;
                }
                int bc = -1;
                amrex::SmallMatrix<Real, dim, 1> nh{};
                if (i < lo_x) { bc = cfg.bc_tag[0]; nh(0, 0) = -1.0; }
                else if (i > hi_x) { bc = cfg.bc_tag[1]; nh(0, 0) = 1.0; }
                else if (dim == 2 && j < lo_y) { bc = cfg.bc_tag[2]; nh(dim - 1, 0) = -1.0; }
                else if (dim == 2 && j > hi_y) { bc = cfg.bc_tag[3]; nh(dim - 1, 0) = 1.0; }
                if (bc == -1) continue;
                VQ qi; VA ai;
                for (int n = 0; n < nq; ++n) qi(n, 0) = q4(ii, jj, 0, n);
                for (int n = 0; n < na; ++n) ai(n, 0) = a4(ii, jj, 0, n);
                const VX X = centre(i, j);
                const VQ qg = Model::boundary_conditions(bc, qi, ai, nh, X, t, dx);
                const VA ag = Model::aux_boundary_conditions(bc, qi, ai, nh, X, t, dx);
                for (int n = 0; n < nq; ++n) q4(i, j, 0, n) = qg(n, 0);
                for (int n = 0; n < na; ++n) a4(i, j, 0, n) = ag(n, 0);
            }
    }

    // ZoomyAmr.cpp:448-515
    Real compute_dt(Real* max_inv_out = nullptr) {
        auto q4 = aQ(); auto a4 = aA();
        const Real dxs[2] = {dx, dy};
        Real gmax = 0.0;
#pragma omp parallel for reduction(max : gmax) schedule(static)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                VQ q; VA a;
                for (int n = 0; n < nq; ++n) q(n, 0) = q4(i, j, 0, n);
                for (int n = 0; n < na; ++n) a(n, 0) = a4(i, j, 0, n);
                Real m = 0.0;
                for (int d = 0; d < dim; ++d) {
                    amrex::SmallMatrix<Real, dim, 1> nh{};
                    nh(d, 0) = 1.0;
                    const auto ev = Numerics::local_max_abs_eigenvalue(q, a, p, nh);
                    const Real inv = ev(0, 0) / dxs[d];
                    if (inv > m) m = inv;
                }
                gmax = (gmax < m) ? m : gmax;
            }
        if (max_inv_out) *max_inv_out = gmax;
        if (gmax < 1e-14) return cfg.dtmax;                               // :499
        const Real div = Real(cfg.cfl_dimension) * Real(cfg.cfl_degree_factor);
        const Real dt = cfg.cfl / (div * gmax);
        return amrex::max(amrex::min(dt, cfg.dtmax), cfg.dtmin);
    }

    // ZoomyAmr.cpp:517-536 (single level): sum(h) * dx * dy, summed row by row
    Real total_mass() {
        auto q4 = aQ();
        Real s = 0.0;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) s += q4(i, j, 0, kIdxH);
        return s * (dx * dy);
    }

    void ensure_faces() {
        if (Fx.empty()) {
            Fx.assign(size_t(gx + 1) * gy * K::n_face_comp, 0.0);
            Fy.assign(size_t(gx) * (gy + 1) * K::n_face_comp, 0.0);
        }
    }

    // The RHS of one stage (ZoomyAmr.cpp:575-626) into Rhs.
    void rhs(int order, Real t, bool face_based) {
        auto q4 = aQ(); auto a4 = aA();
        amrex::Array4<const Real> qc(q4), ac(a4);
        auto r4 = arr(Rhs, nq);
        const bool impl = cfg.implicit_source, wb = cfg.well_balanced;
        if (!face_based) {
#pragma omp parallel for schedule(static)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i)
                    K::cell_rhs(i, j, qc, ac, r4, dx, dy, order, impl, p, t, plox, ploy, wb);
            return;
        }
        ensure_faces();
        auto fx = arr(Fx, K::n_face_comp, gx + 1, gy);
        auto fy = arr(Fy, K::n_face_comp, gx, gy + 1);
#pragma omp parallel for schedule(static)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i <= nx; ++i)
                K::face_data(i, j, 0, order, qc, ac, fx, p, t, dx, dy, plox, ploy, wb);
        if constexpr (dim == 2) {
#pragma omp parallel for schedule(static)
            for (int j = 0; j <= ny; ++j)
                for (int i = 0; i < nx; ++i)
                    K::face_data(i, j, 1, order, qc, ac, fy, p, t, dx, dy, plox, ploy, wb);
        }
        amrex::Array4<const Real> fxc(fx), fyc(dim == 2 ? fy : fx);
#pragma omp parallel for schedule(static)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                K::assemble(i, j, qc, ac, fxc, fyc, r4, dx, dy, impl, p, t, plox, ploy, wb);
    }

    // One stage of ZoomyAmr::Advance (do_stage, ZoomyAmr.cpp:561-662)
    // set by a multi-level driver that fills this box's ghost cells itself
    // (from its neighbours and the coarser level) before each stage
    bool own_ghosts = false;

    void stage(int order, Real t, Real dt, bool face_based) {
        update_state(t);
        if (!own_ghosts) fill_physical_bc(t);   // FillPatch + FillBoundary for one box
        rhs(order, t, face_based);
        auto q4 = aQ(); auto a4 = aA(); auto r4 = arr(Rhs, nq);
#pragma omp parallel for schedule(static)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                for (int n = 0; n < nq; ++n) q4(i, j, 0, n) += dt * r4(i, j, 0, n);
        if (cfg.implicit_source && cfg.implicit_global) {
#pragma omp parallel for schedule(static)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) implicit_source_exact<Model>(i, j, q4, dt, p, t, centre(i, j));
        } else if (cfg.implicit_source) {
            amrex::Array4<const Real> ac(a4);
#pragma omp parallel for schedule(static)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) K::implicit_source(i, j, q4, ac, dt, p, t, centre(i, j));
        }
    }

    void heun() {   // ZoomyAmr.cpp:665-675
        auto q4 = aQ(); auto o4 = arr(Qold, nq);
#pragma omp parallel for schedule(static)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                for (int n = 0; n < nq; ++n) q4(i, j, 0, n) = 0.5 * o4(i, j, 0, n) + 0.5 * q4(i, j, 0, n);
    }

    void copy_valid(std::vector<Real>& dst, std::vector<Real>& src) {
        auto d4 = arr(dst, nq); auto s4 = arr(src, nq);
        for (int n = 0; n < nq; ++n)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) d4(i, j, 0, n) = s4(i, j, 0, n);
    }

    // ZoomyAmr.cpp:538-731
    void advance(Real t, Real dt, bool face_based = true) {
        if (cfg.spatial_order == 1) {
            stage(1, t, dt, face_based);
        } else {
            copy_valid(Qold, Q);
            stage(cfg.spatial_order, t, dt, face_based);
            stage(cfg.spatial_order, t, dt, face_based);
            heun();
            if (cfg.positivity_mood) {   // :699-720
                auto q4 = aQ();
                bool troubled = false;
                for (int j = 0; j < ny && !troubled; ++j)
                    for (int i = 0; i < nx; ++i) {
                        const Real h = q4(i, j, 0, kIdxH);
                        if (!(h >= 0.0) || !(h < 1.0e300)) { troubled = true; break; }
                    }
                if (troubled) {
                    ++mood_redos;
                    copy_valid(Q, Qold);
                    stage(1, t, dt, face_based);
                    stage(1, t, dt, face_based);
                    heun();
                }
            }
        }
        update_state(t);   // :730
    }

    // ZoomyAmr.cpp:733-751 (level 0, no subcycling) + the Evolve loop body :789-809
    bool done() const {
        return !(time < cfg.time_end && (cfg.max_step < 0 || step < cfg.max_step));
    }
    void time_step(bool face_based = true) {
        Real dt = compute_dt();
        const Real remaining = cfg.time_end - time;
        if (remaining > 0.0 && dt > remaining) dt = remaining;
        advance(time, dt, face_based);
        time += dt;
        ++step;
        log.push_back({dt, time, total_mass()});
    }
};

// init_solution (Source/init_solution.cpp:78-116): dam break in x over a flat
// bed for any field with >= 2 components, applied to the state AND the aux
// (ZoomyAmr.cpp:174-175), valid cells only.
inline void init_solution(int ncomp, int nx, int ny, const double* prob_lo, const double* prob_hi,
                          double* v) {
    const double dxc = (prob_hi[0] - prob_lo[0]) / nx;
    const double x_mid = 0.5 * (prob_lo[0] + prob_hi[0]);
    for (int n = 0; n < ncomp; ++n)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) v[(size_t(n) * ny + j) * nx + i] = 0.0;
    if (ncomp >= 2)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const double x = prob_lo[0] + (i + 0.5) * dxc;
                v[(size_t(kIdxB) * ny + j) * nx + i] = 0.0;
                v[(size_t(kIdxH) * ny + j) * nx + i] = (x < x_mid) ? 2.0 : 1.0;
            }
}

}  // namespace zoracle
