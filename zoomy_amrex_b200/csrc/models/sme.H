// Shallow-moment equations (SME) of level L in 1-D or 2-D, written against the
// device-function interface that zoomy-amrex's printer emits into Model.H /
// Numerics.H (zoomy_amrex/transformation/to_amrex.py:326-498 for Model::, the
// make_rhs.H:129-130 / ZoomyAmr.cpp:483 call sites for Numerics::). The
// reference's SWE is this family at level 0 (tests/models.py:17-24 builds it
// as SME(level=0, ...)); the driver is generic in Model::n_dof_q (README.md).
// The generator that emits the reference's SME headers (zoomy_core) is not part
// of the reference, so the system is derived here from its published form:
//
//   J. Kowalski, M. Torrilhon, "Moment approximations and model cascades for
//   shallow flow", Commun. Comput. Phys. 25 (2019) 669-702:
//   velocity profiles u(z) = u_m + sum_j alpha_j phi_j(zeta),
//   v(z) = v_m + sum_j beta_j phi_j(zeta), zeta = (z - b)/h in [0, 1], with the
//   scaled Legendre polynomials phi_j(zeta) = (1/j!) d^j/dzeta^j (zeta - zeta^2)^j
//   (phi_j(0) = 1, int_0^1 phi_i phi_j = delta_ij / (2j + 1)); Galerkin
//   projection of the incompressible hydrostatic equations in the sigma
//   coordinate onto phi_0..phi_L; Newtonian viscosity nu, Navier slip at the
//   bed (slip length lambda), stress-free surface.
//
// The 2-D system (d = x, y; "normal" quantities of direction d are the mean
// velocity w and moments gamma_j along d, "transverse" ones t and tau_j):
//   d_t h + div(h u_m) = 0
//   d_t(h w) + d_d(h w^2 + g h^2/2 + h sum_j gamma_j^2/(2j+1)) + ... = -g h d_d b + S_w
//   d_t(h gamma_i) + d_d(h(2 w gamma_i + sum_jk A_ijk gamma_j gamma_k))
//                  = w D_i - sum_jk B_ijk gamma_k D_j + S_i
//   with D_j = d_x(h alpha_j) + d_y(h beta_j) (the vertical-velocity coupling),
//   transverse moments: flux h(w tau_i + t gamma_i + sum_jk A_ijk gamma_j tau_k),
//   non-conservative part t D_i - sum_jk B_ijk tau_k D_j,
//   A_ijk = (2i+1) int phi_i phi_j phi_k, B_ijk = (2i+1) int phi_i' (int_0^zeta phi_j) phi_k,
//   C_ij = int phi_i' phi_j',
//   S_w = g e_d h - (nu/lambda) u_b(d),  S_i = -(2i+1) [(nu/lambda) u_b(d) + (nu/h) sum_j C_ij gamma_j],
//   u_b = w + sum_j gamma_j the bed velocity (phi_j(0) = 1).
// tests/sme_sympy.py derives the same system symbolically from the velocity
// profiles (no coefficient tables) and tests/test_sme_model.py compares it with
// this header.
//
// State layout: Q = [b, h, hu, (hv), h alpha_1..h alpha_L, (h beta_1..h beta_L)],
// so the driver's bed and depth rows (constants.H:6-7) and its mean-momentum
// rows idx_h+1+d (make_rhs.H:91-94 Audusse rescaling, :159-162 WB source) are
// where the driver expects them. Aux = [hinv] (the desingularised 1/h of the
// shallow-water model, tests/refs/*.npz).
//
// Numerics: central flux 0.5 (F(qL) + F(qR)); fluctuations
// D+- = 0.5 Btilde (qR - qL) +- 0.5 s (qR - qL) with Btilde = int_0^1 B(psi(s)) ds
// along the straight path psi in the conserved variables: the bed product
// g h db exactly (g (hL + hR)/2 (bR - bL), as the shallow-water model), the
// moment products by 3-point Gauss-Legendre quadrature with hinv recomputed
// from the path depth; s = max over both sides of local_max_abs_eigenvalue.
// local_max_abs_eigenvalue is the Gershgorin row-sum bound of the quasilinear
// matrix dF/dQ + B in the face-normal direction over the evolved rows and
// columns (the bed row is zero, so the bed's eigenvalue is 0 and the others
// are those of the evolved block): the fallback the reference's numerics use
// when a model has no closed-form eigenvalues (README.md: "Gershgorin row-sum
// when eigenvalues=None"). With every moment zero the flux and the
// non-conservative products reduce bit for bit to the shallow-water model's.
#pragma once
#include <vector>
#include <string>
#include <cmath>
#include "AMReX_REAL.H"
#include "AMReX_SmallMatrix.H"
#include "AMReX_Algorithm.H"
#include "AMReX_Math.H"

#ifndef PORTABLE_FN
#  ifdef __CUDACC__
#    define PORTABLE_FN __host__ __device__
#  else
#    define PORTABLE_FN
#  endif
#endif

namespace zb {

// Parameter slots: p(0) = g is the gravity make_rhs.H:287 passes to the WB bed
// source; p(5) the hinv floor, as in the shallow-water model.
enum SMEParam : int {
    sme_g = 0,        // gravity
    sme_ex = 1,       // along-x gravity component of an inclined bed frame
    sme_ey = 2,       // along-y counterpart
    sme_nu = 3,       // kinematic viscosity
    sme_lambda = 4,   // Navier slip length at the bed
    sme_eps = 5,      // hinv desingularisation: h^4 floor
    sme_n_params = 6
};

// Projection coefficients of the scaled Legendre basis (exact rationals, from
// the integrals above), indices 1..3 (0 unused). Functions rather than
// arrays so that device code can use them; with the level a compile-time
// constant every index folds away.
struct SMECoef {
    static constexpr int kMaxLevel = 3;
    // A_ijk = (2i+1) int_0^1 phi_i phi_j phi_k
    static constexpr PORTABLE_FN double A(int i, int j, int k) {
        constexpr double t[4][4][4] = {
            {{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}},
            {{0, 0, 0, 0}, {0, 0, 2.0 / 5.0, 0}, {0, 2.0 / 5.0, 0, 9.0 / 35.0}, {0, 0, 9.0 / 35.0, 0}},
            {{0, 0, 0, 0}, {0, 2.0 / 3.0, 0, 3.0 / 7.0}, {0, 0, 2.0 / 7.0, 0}, {0, 3.0 / 7.0, 0, 4.0 / 21.0}},
            {{0, 0, 0, 0}, {0, 0, 3.0 / 5.0, 0}, {0, 3.0 / 5.0, 0, 4.0 / 15.0}, {0, 0, 4.0 / 15.0, 0}}};
        return t[i][j][k];
    }
    // B_ijk = (2i+1) int_0^1 phi_i' (int_0^zeta phi_j) phi_k
    static constexpr PORTABLE_FN double B(int i, int j, int k) {
        constexpr double t[4][4][4] = {
            {{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}},
            {{0, 0, 0, 0}, {0, 0, 1.0 / 5.0, 0}, {0, -1.0 / 5.0, 0, 3.0 / 35.0}, {0, 0, -3.0 / 35.0, 0}},
            {{0, 0, 0, 0}, {0, -1.0, 0, 3.0 / 7.0}, {0, 0, -1.0 / 7.0, 0}, {0, -2.0 / 7.0, 0, -1.0 / 21.0}},
            {{0, 0, 0, 0}, {0, 0, -6.0 / 5.0, 0}, {0, -4.0 / 5.0, 0, -2.0 / 15.0}, {0, 0, -1.0 / 5.0, 0}}};
        return t[i][j][k];
    }
    // C_ij = int_0^1 phi_i' phi_j'
    static constexpr PORTABLE_FN double C(int i, int j) {
        constexpr double t[4][4] = {{0, 0, 0, 0}, {0, 4, 0, 4}, {0, 0, 12, 0}, {0, 4, 0, 24}};
        return t[i][j];
    }
    // 1 / (2j + 1) = int_0^1 phi_j^2
    static constexpr PORTABLE_FN double N(int j) {
        constexpr double t[4] = {1.0, 1.0 / 3.0, 1.0 / 5.0, 1.0 / 7.0};
        return t[j];
    }
    // 3-point Gauss-Legendre on [0, 1]: nodes 1/2 -+ sqrt(15)/10, 1/2; weights 5/18, 8/18, 5/18
    static constexpr PORTABLE_FN double gl_s(int q) {
        constexpr double t[3] = {0.11270166537925831148, 0.5, 0.88729833462074168852};
        return t[q];
    }
    static constexpr PORTABLE_FN double gl_w(int q) {
        constexpr double t[3] = {5.0 / 18.0, 8.0 / 18.0, 5.0 / 18.0};
        return t[q];
    }
};

template <class R, int DIM, int LEVEL>
struct SME
{
    static_assert(DIM == 1 || DIM == 2, "SME is 1-D or 2-D");
    static_assert(LEVEL >= 0 && LEVEL <= SMECoef::kMaxLevel, "SME levels 0..3 are tabulated");
    using T = R;
    using K = SMECoef;
    static constexpr int level = LEVEL;
    static constexpr int n_dof_q = 2 + DIM * (1 + LEVEL);
    static constexpr int n_dof_eq = n_dof_q;
    static constexpr int n_dof_qaux = 1;
    static constexpr int n_parameters = sme_n_params;
    static constexpr int dimension = DIM;
    static constexpr int n_dof_gradQ = n_dof_q * DIM;
    static constexpr bool has_diffusion = false;
    static constexpr int n_boundary_tags = 2;
    static constexpr int i_hinv = 0;

    // Build-side traits (see fv_model_traits.H): aux is a function of Q, the
    // bed row never changes.
    static constexpr bool zb_aux_pure = true;
    static constexpr bool zb_static_bed = true;

    // Row of the mean momentum along direction d, and of moment j (1-based) along d.
    // The point-implicit system's blocks (see fv_model_traits.H): per
    // direction d the mean momentum and its LEVEL moments.
    static constexpr int zb_implicit_blocks = DIM;
    static constexpr int zb_implicit_block_size = 1 + LEVEL;
    static constexpr PORTABLE_FN int zb_implicit_row(int b, int i) { return i == 0 ? mom(b) : mnt(b, i); }

    static constexpr PORTABLE_FN int mom(int d) { return 2 + d; }
    static constexpr PORTABLE_FN int mnt(int d, int j) { return 2 + DIM + d * LEVEL + (j - 1); }

    using VQ = amrex::SmallMatrix<R, n_dof_q, 1>;
    using VA = amrex::SmallMatrix<R, n_dof_qaux, 1>;
    using VP = amrex::SmallMatrix<R, n_parameters, 1>;
    using VN = amrex::SmallMatrix<R, DIM, 1>;
    using VX = amrex::SmallMatrix<R, 3, 1>;

    static const std::vector<std::string> get_boundary_tags() { return {"extrapolation", "wall"}; }
    static const std::vector<std::string> parameter_names() {
        return {"g", "ex", "ey", "nu", "lambda", "eps"};
    }
    static const std::vector<R> default_parameters() {
        return {R(9.81), R(0.0), R(0.0), R(1.0e-3), R(0.1), R(1.0e-24)};
    }

    // Kurganov-Petrova desingularised 1/h (the shallow-water model's).
    static PORTABLE_FN AMREX_FORCE_INLINE R hinv_of(R h, R eps) {
        R x0 = amrex::Math::powi<4>(h);
        return std::sqrt(R(2)) * h / std::sqrt(x0 + amrex::max(x0, eps));
    }

    static PORTABLE_FN AMREX_FORCE_INLINE VQ update_variables(VQ const& Q, VA const&, VP const&) {
        return Q;
    }

    static PORTABLE_FN AMREX_FORCE_INLINE VA update_aux_variables(
        VQ const& Q, VA const& /*Qaux*/, VP const& p, R const /*time*/, VX const& /*X*/) {
        VA a;
        a(i_hinv, 0) = hinv_of(Q(1, 0), p(sme_eps, 0));
        return a;
    }

    static PORTABLE_FN AMREX_FORCE_INLINE amrex::SmallMatrix<R, n_dof_qaux * n_dof_q, 1>
    update_aux_variables_jacobian_wrt_variables(VQ const&, VA const&, VP const&, R const, VX const&) {
        amrex::SmallMatrix<R, n_dof_qaux * n_dof_q, 1> J{};
        return J;   // the printer emits all zeros here (to_amrex.py:475-480)
    }

    // h times the bed velocity along d: h u(zeta = 0) = h w + sum_j h gamma_j.
    static PORTABLE_FN AMREX_FORCE_INLINE R bed_flux(VQ const& Q, int d) {
        R ub = Q(mom(d), 0);
#pragma unroll
        for (int j = 1; j <= LEVEL; ++j) ub = ub + Q(mnt(d, j), 0);
        return ub;
    }

    static PORTABLE_FN AMREX_FORCE_INLINE VQ source(
        VQ const& Q, VA const& Qaux, VP const& p, R const /*time*/, VX const& /*X*/) {
        VQ S{};
        const R g = p(sme_g, 0), nu = p(sme_nu, 0);
        const R kb = nu / p(sme_lambda, 0);
        const R hinv = Qaux(i_hinv, 0);
        const R h = Q(1, 0);
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const R e = (d == 0) ? p(sme_ex, 0) : p(sme_ey, 0);
            const R fb = kb * (hinv * bed_flux(Q, d));
            S(mom(d), 0) = g * e * h - fb;
#pragma unroll
            for (int i = 1; i <= LEVEL; ++i) {
                R cs = R(0);
#pragma unroll
                for (int j = 1; j <= LEVEL; ++j)
                    if (K::C(i, j) != 0.0) cs = cs + R(K::C(i, j)) * Q(mnt(d, j), 0);
                S(mnt(d, i), 0) = -R(2 * i + 1) * (fb + nu * (hinv * hinv) * cs);
            }
        }
        return S;
    }

    // dS/dQ with the aux (hinv) held fixed, row-major (n_eq x n_q): constant
    // in Q for a given hinv (the friction is linear in the momenta).
    static PORTABLE_FN AMREX_FORCE_INLINE amrex::SmallMatrix<R, n_dof_q * n_dof_q, 1>
    source_jacobian_wrt_variables(VQ const& /*Q*/, VA const& Qaux, VP const& p) {
        constexpr int n = n_dof_q;
        amrex::SmallMatrix<R, n * n, 1> J{};
        const R g = p(sme_g, 0), nu = p(sme_nu, 0);
        const R kb = nu / p(sme_lambda, 0);
        const R hinv = Qaux(i_hinv, 0);
        const R kh = kb * hinv;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const R e = (d == 0) ? p(sme_ex, 0) : p(sme_ey, 0);
            const int w = mom(d);
            J(w * n + 1, 0) = g * e;
            J(w * n + w, 0) = -kh;
#pragma unroll
            for (int j = 1; j <= LEVEL; ++j) J(w * n + mnt(d, j), 0) = -kh;
#pragma unroll
            for (int i = 1; i <= LEVEL; ++i) {
                const int r = mnt(d, i);
                const R ci = R(2 * i + 1);
                J(r * n + w, 0) = -ci * kh;
#pragma unroll
                for (int j = 1; j <= LEVEL; ++j)
                    J(r * n + mnt(d, j), 0) = -ci * (kh + nu * (hinv * hinv) * R(K::C(i, j)));
            }
        }
        return J;
    }

    // dS/dQaux, row-major (n_eq x n_aux): the hinv column.
    static PORTABLE_FN AMREX_FORCE_INLINE amrex::SmallMatrix<R, n_dof_q * n_dof_qaux, 1>
    source_jacobian_wrt_aux_variables(VQ const& Q, VA const& Qaux, VP const& p) {
        constexpr int na = n_dof_qaux;
        amrex::SmallMatrix<R, n_dof_q * na, 1> J{};
        const R nu = p(sme_nu, 0);
        const R kb = nu / p(sme_lambda, 0);
        const R hinv = Qaux(i_hinv, 0);
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const R ub = bed_flux(Q, d);
            J(mom(d) * na + i_hinv, 0) = -kb * ub;
#pragma unroll
            for (int i = 1; i <= LEVEL; ++i) {
                R cs = R(0);
#pragma unroll
                for (int j = 1; j <= LEVEL; ++j)
                    if (K::C(i, j) != 0.0) cs = cs + R(K::C(i, j)) * Q(mnt(d, j), 0);
                J(mnt(d, i) * na + i_hinv, 0) = -R(2 * i + 1) * (kb * ub + R(2) * nu * hinv * cs);
            }
        }
        return J;
    }

    // Build-side shortcut (not part of the printer's interface): the
    // point-implicit step of make_rhs.H:429-509, (I - dt J) dq = dt S with
    // J = dS/dQ at fixed aux, solved block by block. The bed and depth rows of
    // J and S are zero (dq = 0 there) and the friction couples only the mean
    // momentum and the moments of one direction, so the system splits into
    // DIM blocks of 1 + LEVEL unknowns, each solved by elimination with
    // partial pivoting. Non-finite results fall back to the explicit step
    // dt S (or 0), as make_rhs.H:501-508. The FP32 kernels use it; the FP64
    // form keeps the reference's full elimination for bitwise parity.
    static PORTABLE_FN AMREX_FORCE_INLINE void zb_implicit_increment(VQ const& Q, VA const& Qaux, VP const& p,
                                                                    R dt, VQ& dq) {
        constexpr int nb = 1 + LEVEL;
        const auto S = source(Q, Qaux, p, R(0), VX{});
        const R nu = p(sme_nu, 0);
        const R kh = (nu / p(sme_lambda, 0)) * Qaux(i_hinv, 0);
        const R hh = Qaux(i_hinv, 0) * Qaux(i_hinv, 0);
        dq(0, 0) = R(0);
        dq(1, 0) = R(0);
        // Every loop has a constant trip count (ranges are guards) and no
        // early exit (after a failed pivot the values are discarded for the
        // fallback), and rows are swapped by selecting through the unrolled
        // rows, so the blocks stay in registers.
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            R A[nb][nb], b[nb];
#pragma unroll
            for (int r = 0; r < nb; ++r) {
                const int row = (r == 0) ? mom(d) : mnt(d, r);
                b[r] = dt * S(row, 0);
                const R cr = R(2 * r + 1);
#pragma unroll
                for (int c = 0; c < nb; ++c) {
                    R j = -kh;
                    if (r > 0 && c > 0 && K::C(r, c) != 0.0) j = j - nu * hh * R(K::C(r, c));
                    A[r][c] = (r == c ? R(1) : R(0)) - dt * (cr * j);
                }
            }
            bool ok = true;
#pragma unroll
            for (int k = 0; k < nb; ++k) {
                int piv = k;
                R best = std::abs(A[k][k]);
#pragma unroll
                for (int r = 0; r < nb; ++r)
                    if (r > k && std::abs(A[r][k]) > best) { best = std::abs(A[r][k]); piv = r; }
                ok = ok && (best > R(0));
#pragma unroll
                for (int r = 0; r < nb; ++r) {
                    if (r > k && r == piv) {
#pragma unroll
                        for (int c = 0; c < nb; ++c) { const R t = A[k][c]; A[k][c] = A[r][c]; A[r][c] = t; }
                        const R t = b[k]; b[k] = b[r]; b[r] = t;
                    }
                }
#pragma unroll
                for (int r = 0; r < nb; ++r) {
                    if (r <= k) continue;
                    const R f = A[r][k] / A[k][k];
#pragma unroll
                    for (int c = 0; c < nb; ++c)
                        if (c >= k) A[r][c] = A[r][c] - f * A[k][c];
                    b[r] = b[r] - f * b[k];
                }
            }
            R x[nb];
#pragma unroll
            for (int r = nb - 1; r >= 0; --r) {
                R s = b[r];
#pragma unroll
                for (int c = 0; c < nb; ++c)
                    if (c > r) s = s - A[r][c] * x[c];
                x[r] = s / A[r][r];
                ok = ok && std::isfinite(x[r]);
            }
#pragma unroll
            for (int r = 0; r < nb; ++r) {
                const int row = (r == 0) ? mom(d) : mnt(d, r);
                const R e = dt * S(row, 0);
                dq(row, 0) = ok ? x[r] : (std::isfinite(e) ? e : R(0));
            }
        }
    }

    static PORTABLE_FN AMREX_FORCE_INLINE amrex::SmallMatrix<R, n_dof_q * DIM, 1>
    diffusive_flux(VQ const&, VA const&, amrex::SmallMatrix<R, n_dof_gradQ, 1> const&, VP const&) {
        amrex::SmallMatrix<R, n_dof_q * DIM, 1> F{};
        return F;   // has_diffusion == false: never called
    }

    // Ghost state from the mirrored interior state (ZoomyAmr.cpp:435).
    // bc_idx 0: extrapolation; bc_idx 1: reflective wall, which mirrors the
    // whole velocity profile: the normal mean momentum and every normal moment
    // flip sign.
    static PORTABLE_FN AMREX_FORCE_INLINE VQ boundary_conditions(
        const int bc_idx, VQ const& Q, VA const& /*Qaux*/, VN const& n, VX const& /*X*/,
        R const /*time*/, R const /*dX*/) {
        VQ g = Q;
        if (bc_idx == 1) {
#pragma unroll
            for (int j = 0; j <= LEVEL; ++j) {
                R qn = Q(j == 0 ? mom(0) : mnt(0, j), 0) * n(0, 0);
                if constexpr (DIM == 2) qn = qn + Q(j == 0 ? mom(1) : mnt(1, j), 0) * n(1, 0);
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    const int r = (j == 0) ? mom(d) : mnt(d, j);
                    g(r, 0) = Q(r, 0) - R(2) * qn * n(d, 0);
                }
            }
        }
        return g;
    }
    static PORTABLE_FN AMREX_FORCE_INLINE VA aux_boundary_conditions(
        const int, VQ const&, VA const& Qaux, VN const&, VX const&, R const, R const) {
        return Qaux;   // identity (to_amrex.py:491-498)
    }

    // Physical flux projected on the face normal e_D.
    template <int D>
    static PORTABLE_FN AMREX_FORCE_INLINE VQ flux_dir(VQ const& Q, VA const& Qaux, VP const& p) {
        constexpr int E = (DIM == 2) ? 1 - D : D;   // the transverse direction (2-D)
        VQ F;
        const R g = p(sme_g, 0);
        const R hinv = Qaux(i_hinv, 0);
        const R h = Q(1, 0);
        const R qw = Q(mom(D), 0);
        F(0, 0) = R(0);
        F(1, 0) = qw;
        // mean momenta: the shallow-water terms, then the moments' share
        R sw = R(0);
#pragma unroll
        for (int j = 1; j <= LEVEL; ++j) sw = sw + R(K::N(j)) * (Q(mnt(D, j), 0) * Q(mnt(D, j), 0));
        F(mom(D), 0) = (qw * qw * hinv + R(0.5) * g * h * h) + hinv * sw;
        if constexpr (DIM == 2) {
            const R qt = Q(mom(E), 0);
            R st = R(0);
#pragma unroll
            for (int j = 1; j <= LEVEL; ++j) st = st + R(K::N(j)) * (Q(mnt(D, j), 0) * Q(mnt(E, j), 0));
            F(mom(E), 0) = qt * qw * hinv + hinv * st;
        }
        // moments along D (normal) and across it (transverse)
#pragma unroll
        for (int i = 1; i <= LEVEL; ++i) {
            R an = R(0), at = R(0);
#pragma unroll
            for (int j = 1; j <= LEVEL; ++j)
#pragma unroll
                for (int k = 1; k <= LEVEL; ++k) {
                    const R a = R(K::A(i, j, k));
                    if (a == R(0)) continue;
                    an = an + a * (Q(mnt(D, j), 0) * Q(mnt(D, k), 0));
                    if constexpr (DIM == 2) at = at + a * (Q(mnt(D, j), 0) * Q(mnt(E, k), 0));
                }
            F(mnt(D, i), 0) = hinv * (R(2) * qw * Q(mnt(D, i), 0) + an);
            if constexpr (DIM == 2) {
                const R qt = Q(mom(E), 0);
                F(mnt(E, i), 0) = hinv * (qw * Q(mnt(E, i), 0) + qt * Q(mnt(D, i), 0) + at);
            }
        }
        return F;
    }

    // The moment rows of B_D(Q) dq: the non-conservative products of the
    // vertical coupling along D (the bed product is handled by the numerics).
    template <int D>
    static PORTABLE_FN AMREX_FORCE_INLINE void ncp_moments(VQ const& Q, R hinv, VQ const& dq, VQ& out) {
        constexpr int E = (DIM == 2) ? 1 - D : D;
        const R wm = Q(mom(D), 0) * hinv;
        R tm = R(0);
        if constexpr (DIM == 2) tm = Q(mom(E), 0) * hinv;
#pragma unroll
        for (int i = 1; i <= LEVEL; ++i) {
            R rn = -wm * dq(mnt(D, i), 0), rt = -tm * dq(mnt(D, i), 0);
#pragma unroll
            for (int j = 1; j <= LEVEL; ++j) {
                R cn = R(0), ct = R(0);
#pragma unroll
                for (int k = 1; k <= LEVEL; ++k) {
                    const R bc = R(K::B(i, j, k));
                    if (bc == R(0)) continue;
                    cn = cn + bc * (Q(mnt(D, k), 0) * hinv);
                    if constexpr (DIM == 2) ct = ct + bc * (Q(mnt(E, k), 0) * hinv);
                }
                rn = rn + cn * dq(mnt(D, j), 0);
                rt = rt + ct * dq(mnt(D, j), 0);
            }
            out(mnt(D, i), 0) = rn;
            if constexpr (DIM == 2) out(mnt(E, i), 0) = rt;
        }
    }

    // Gershgorin row-sum bound of |eig(dF_D/dQ + B_D)| over the evolved rows
    // and columns (the derivatives taken with hinv = 1/h).
    template <int D>
    static PORTABLE_FN AMREX_FORCE_INLINE R max_abs_eig_dir(VQ const& Q, VA const& Qaux, VP const& p) {
        constexpr int E = (DIM == 2) ? 1 - D : D;
        const R hinv = Qaux(i_hinv, 0);
        const R g = p(sme_g, 0);
        const R h = Q(1, 0);
        const R w = Q(mom(D), 0) * hinv;
        R ga[LEVEL + 1], ta[LEVEL + 1];
        ga[0] = R(0); ta[0] = R(0);
#pragma unroll
        for (int j = 1; j <= LEVEL; ++j) ga[j] = Q(mnt(D, j), 0) * hinv;
        R t = R(0);
        if constexpr (DIM == 2) {
            t = Q(mom(E), 0) * hinv;
#pragma unroll
            for (int j = 1; j <= LEVEL; ++j) ta[j] = Q(mnt(E, j), 0) * hinv;
        } else {
#pragma unroll
            for (int j = 1; j <= LEVEL; ++j) ta[j] = R(0);
        }
        R best = R(1);   // the depth row: dF_h/dq_w = 1
        {   // normal mean momentum: columns h, q_w, h gamma_j
            R d0 = g * h - w * w;
            R r = std::abs(R(2) * w);
#pragma unroll
            for (int j = 1; j <= LEVEL; ++j) {
                d0 = d0 - R(K::N(j)) * (ga[j] * ga[j]);
                r = r + std::abs(R(2) * R(K::N(j)) * ga[j]);
            }
            r = r + std::abs(d0);
            best = amrex::max(best, r);
        }
        if constexpr (DIM == 2) {   // transverse mean momentum: h, q_w, q_t, h gamma_j, h tau_j
            R d0 = -w * t;
            R r = std::abs(t) + std::abs(w);
#pragma unroll
            for (int j = 1; j <= LEVEL; ++j) {
                d0 = d0 - R(K::N(j)) * (ga[j] * ta[j]);
                r = r + std::abs(R(K::N(j)) * ta[j]) + std::abs(R(K::N(j)) * ga[j]);
            }
            r = r + std::abs(d0);
            best = amrex::max(best, r);
        }
#pragma unroll
        for (int i = 1; i <= LEVEL; ++i) {
            // normal moment i: h, q_w, h gamma_j (flux + non-conservative)
            R d0 = R(-2) * w * ga[i];
            R r = std::abs(R(2) * ga[i]);
#pragma unroll
            for (int j = 1; j <= LEVEL; ++j) {
                R c = (i == j) ? w : R(0);
#pragma unroll
                for (int k = 1; k <= LEVEL; ++k) {
                    // (the tables are compile-time constants: zero terms fold away)
                    if (K::A(i, j, k) != 0.0) d0 = d0 - R(K::A(i, j, k)) * (ga[j] * ga[k]);
                    if (2.0 * K::A(i, j, k) + K::B(i, j, k) != 0.0)
                        c = c + R(2.0 * K::A(i, j, k) + K::B(i, j, k)) * ga[k];
                }
                r = r + std::abs(c);
            }
            r = r + std::abs(d0);
            best = amrex::max(best, r);
            if constexpr (DIM == 2) {
                // transverse moment i: h, q_w, q_t, h gamma_j, h tau_k
                R e0 = -w * ta[i] - t * ga[i];
                R s = std::abs(ta[i]) + std::abs(ga[i]);
#pragma unroll
                for (int j = 1; j <= LEVEL; ++j) {
                    R cg = R(0), ct = (i == j) ? w : R(0);
#pragma unroll
                    for (int k = 1; k <= LEVEL; ++k) {
                        if (K::A(i, j, k) != 0.0) e0 = e0 - R(K::A(i, j, k)) * (ga[j] * ta[k]);
                        if (K::A(i, j, k) + K::B(i, j, k) != 0.0)
                            cg = cg + R(K::A(i, j, k) + K::B(i, j, k)) * ta[k];
                        if (K::A(i, k, j) != 0.0) ct = ct + R(K::A(i, k, j)) * ga[k];
                    }
                    s = s + std::abs(cg) + std::abs(ct);
                }
                s = s + std::abs(e0);
                best = amrex::max(best, s);
            }
        }
        return best;
    }
};

// Numerics: central flux + path-conservative Rusanov fluctuations (see the
// header comment).
template <class R, int DIM, int LEVEL>
struct SMENumerics
{
    using M = SME<R, DIM, LEVEL>;
    using K = SMECoef;
    static constexpr int nq = M::n_dof_q;
    using VQ = typename M::VQ;
    using VA = typename M::VA;
    using VP = typename M::VP;
    using VN = typename M::VN;
    using V2Q = amrex::SmallMatrix<R, 2 * nq, 1>;

    static PORTABLE_FN AMREX_FORCE_INLINE int dir_of(VN const& n) {
        if constexpr (DIM == 2) return (n(1, 0) != R(0)) ? 1 : 0;
        else return 0;
    }

    template <int D>
    static PORTABLE_FN AMREX_FORCE_INLINE VQ flux_d(VQ const& qL, VQ const& qR, VA const& aL,
                                                    VA const& aR, VP const& p) {
        VQ fL = M::template flux_dir<D>(qL, aL, p);
        VQ fR = M::template flux_dir<D>(qR, aR, p);
        VQ F;
#pragma unroll
        for (int n = 0; n < nq; ++n) F(n, 0) = R(0.5) * (fL(n, 0) + fR(n, 0));
        return F;
    }

    // Btilde (qR - qL): the bed product exactly, the moment products by
    // Gauss-Legendre quadrature along the straight path.
    template <int D>
    static PORTABLE_FN AMREX_FORCE_INLINE VQ path_product(VQ const& qL, VQ const& qR, VP const& p) {
        VQ dq, bdq{};
#pragma unroll
        for (int n = 0; n < nq; ++n) dq(n, 0) = qR(n, 0) - qL(n, 0);
        bdq(M::mom(D), 0) = p(sme_g, 0) * (R(0.5) * (qL(1, 0) + qR(1, 0))) * dq(0, 0);
        if constexpr (LEVEL > 0) {
            const R eps = p(sme_eps, 0);
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const R s = R(K::gl_s(q));
                VQ ps, part;
#pragma unroll
                for (int n = 1; n < nq; ++n) ps(n, 0) = qL(n, 0) + s * dq(n, 0);
                M::template ncp_moments<D>(ps, M::hinv_of(ps(1, 0), eps), dq, part);
#pragma unroll
                for (int j = 1; j <= LEVEL; ++j) {
                    bdq(M::mnt(D, j), 0) = bdq(M::mnt(D, j), 0) + R(K::gl_w(q)) * part(M::mnt(D, j), 0);
                    if constexpr (DIM == 2) {
                        constexpr int E = 1 - D;
                        bdq(M::mnt(E, j), 0) = bdq(M::mnt(E, j), 0) + R(K::gl_w(q)) * part(M::mnt(E, j), 0);
                    }
                }
            }
        }
        return bdq;
    }

    template <int D>
    static PORTABLE_FN AMREX_FORCE_INLINE V2Q fluct_d(VQ const& qL, VQ const& qR, VA const& aL,
                                                      VA const& aR, VP const& p) {
        const R s = amrex::max(M::template max_abs_eig_dir<D>(qL, aL, p),
                               M::template max_abs_eig_dir<D>(qR, aR, p));
        const VQ bdq = path_product<D>(qL, qR, p);
        V2Q D2;
        D2(0, 0) = R(0);
        D2(nq, 0) = R(0);
#pragma unroll
        for (int n = 1; n < nq; ++n) {
            const R dq = qR(n, 0) - qL(n, 0);
            D2(n, 0) = R(0.5) * bdq(n, 0) + R(0.5) * s * dq;        // D+
            D2(nq + n, 0) = R(0.5) * bdq(n, 0) - R(0.5) * s * dq;   // D-
        }
        return D2;
    }

    static PORTABLE_FN AMREX_FORCE_INLINE VQ numerical_flux(VQ const& qL, VQ const& qR, VA const& aL,
                                                            VA const& aR, VP const& p, VN const& n) {
        if constexpr (DIM == 2) { if (dir_of(n) == 1) return flux_d<1>(qL, qR, aL, aR, p); }
        return flux_d<0>(qL, qR, aL, aR, p);
    }

    static PORTABLE_FN AMREX_FORCE_INLINE V2Q numerical_fluctuations(VQ const& qL, VQ const& qR,
                                                                     VA const& aL, VA const& aR,
                                                                     VP const& p, VN const& n) {
        if constexpr (DIM == 2) { if (dir_of(n) == 1) return fluct_d<1>(qL, qR, aL, aR, p); }
        return fluct_d<0>(qL, qR, aL, aR, p);
    }

    static PORTABLE_FN AMREX_FORCE_INLINE amrex::SmallMatrix<R, 1, 1>
    local_max_abs_eigenvalue(VQ const& q, VA const& a, VP const& p, VN const& n) {
        amrex::SmallMatrix<R, 1, 1> ev;
        if constexpr (DIM == 2) {
            if (dir_of(n) == 1) { ev(0, 0) = M::template max_abs_eig_dir<1>(q, a, p); return ev; }
        }
        ev(0, 0) = M::template max_abs_eig_dir<0>(q, a, p);
        return ev;
    }
};

}  // namespace zb
