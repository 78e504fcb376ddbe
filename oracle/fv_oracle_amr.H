// Two-level AMR driver of the CPU oracle — TEST INFRASTRUCTURE ONLY.
//
// The hierarchy the GPU builds (zoomy_amrex_b200/amr.py, csrc/fv32_amr.cuh),
// restated in FP64 on top of the oracle's single-box Level: a base level over
// the whole domain and a fixed set of rectangular fine patches (refinement
// ratio 2, properly nested, never regridded), stepped like the reference's
// subcycled TimeStep (ZoomyAmr.cpp:733-762): a base-level step of dt, then
// two fine steps of dt/2, then average_down. Before each fine stage every
// ghost cell of a patch takes
//   * the stage input of the fine cell there when a fine patch holds it
//     (FillBoundary), a cell outside the domain being mirrored into it first
//     with the wall's normal-momentum flip (FillPhysicalBC_mf),
//   * else a conservative linear interpolation of the base level's current
//     state with minmod-limited slopes of b, eta = h + b, hu, hv
//     (FillPatchTwoLevels with the single coarse time level the reference
//     passes, ZoomyAmr.cpp:258-277);
// average_down replaces each coarse cell under the fine level by the mean of
// its four fine cells (eta, hu, hv; the coarse bed is kept). A new fine
// patch starts as the same interpolation of the base level
// (MakeNewLevelFromCoarse). The step size is either given (both levels' CFL
// laws are then moot, which isolates the ghost fill, the subcycling and the
// averaging) or the reference's per-level law (ZoomyAmr.cpp:739-749): each
// level takes ComputeDt of its current state before each of its steps (the
// fine level's over all its patches), the base level's clamped to land on
// time_end.
#pragma once
#include <array>
#include <vector>
#include "fv_oracle.H"

namespace zoracle {

template <class Model, class Numerics, class K>
struct Hierarchy2 {
    using Lev = Level<Model, Numerics, K>;
    static constexpr int nq = Model::n_dof_q;
    static_assert(Model::dimension == 2 && nq == 4, "the two-level driver is written for 2-D shallow water");

    Lev L0;
    std::vector<Lev> P;
    std::vector<std::array<int, 4>> rect;     // fine cells: i0, j0, nx, ny
    int nxf, nyf;
    bool wall[4];

    Hierarchy2(const zfv_config& c0, const int* rects, int n_rects) : L0(c0) {
        nxf = 2 * c0.nx; nyf = 2 * c0.ny;
        for (int s = 0; s < 4; ++s) wall[s] = c0.bc_tag[s] == 1;
        const Real dxf = L0.dx * 0.5, dyf = L0.dy * 0.5;
        for (int k = 0; k < n_rects; ++k) {
            std::array<int, 4> r{rects[4 * k], rects[4 * k + 1], rects[4 * k + 2], rects[4 * k + 3]};
            zfv_config c = c0;
            c.nx = r[2]; c.ny = r[3];
            c.prob_lo[0] = c0.prob_lo[0] + r[0] * dxf;
            c.prob_lo[1] = c0.prob_lo[1] + r[1] * dyf;
            c.prob_hi[0] = c.prob_lo[0] + r[2] * dxf;
            c.prob_hi[1] = c.prob_lo[1] + r[3] * dyf;
            rect.push_back(r);
            P.emplace_back(c);
            P.back().own_ghosts = true;
        }
    }

    // base-level cell (i, j), mirrored into the domain with the wall flips: b, eta, hu, hv
    std::array<Real, 4> coarse_at(int i, int j) {
        bool fu = false, fv = false;
        const int nx = L0.nx, ny = L0.ny;
        if (i < 0) { i = -1 - i; fu = wall[0]; } else if (i >= nx) { i = 2 * nx - 1 - i; fu = wall[1]; }
        if (j < 0) { j = -1 - j; fv = wall[2]; } else if (j >= ny) { j = 2 * ny - 1 - j; fv = wall[3]; }
        auto q = L0.aQ();
        std::array<Real, 4> v{q(i, j, 0, 0), q(i, j, 0, 1) + q(i, j, 0, 0), q(i, j, 0, 2), q(i, j, 0, 3)};
        if (fu) v[2] = -v[2];
        if (fv) v[3] = -v[3];
        return v;
    }

    static Real mm(Real a, Real b) {   // make_rhs.H:9-13
        if (a * b <= 0.0) return 0.0;
        return (std::abs(a) < std::abs(b)) ? a : b;
    }

    // conservative linear interpolation of the base level at fine cell (I, J): b, h, hu, hv
    std::array<Real, 4> interp(int I, int J) {
        const int ic = I >> 1, jc = J >> 1;
        const auto c = coarse_at(ic, jc), xm = coarse_at(ic - 1, jc), xp = coarse_at(ic + 1, jc);
        const auto ym = coarse_at(ic, jc - 1), yp = coarse_at(ic, jc + 1);
        const Real ox = (I & 1) ? 0.25 : -0.25, oy = (J & 1) ? 0.25 : -0.25;
        std::array<Real, 4> r;
        for (int n = 0; n < 4; ++n)
            r[n] = c[n] + ox * mm(c[n] - xm[n], xp[n] - c[n]) + oy * mm(c[n] - ym[n], yp[n] - c[n]);
        return {r[0], r[1] - r[0], r[2], r[3]};
    }

    // the fine level's current value at (I, J) (mirrored into the domain),
    // false when no patch holds it
    bool fine_at(int I, int J, std::array<Real, 4>& v) {
        bool fu = false, fv = false;
        if (I < 0) { I = -1 - I; fu = wall[0]; } else if (I >= nxf) { I = 2 * nxf - 1 - I; fu = wall[1]; }
        if (J < 0) { J = -1 - J; fv = wall[2]; } else if (J >= nyf) { J = 2 * nyf - 1 - J; fv = wall[3]; }
        for (size_t k = 0; k < P.size(); ++k) {
            const auto& r = rect[k];
            if (I >= r[0] && I < r[0] + r[2] && J >= r[1] && J < r[1] + r[3]) {
                auto q = P[k].aQ();
                for (int n = 0; n < 4; ++n) v[n] = q(I - r[0], J - r[1], 0, n);
                if (fu) v[2] = -v[2];
                if (fv) v[3] = -v[3];
                return true;
            }
        }
        return false;
    }

    void fill_fine_ghosts() {
        for (size_t k = 0; k < P.size(); ++k) {
            Lev& L = P[k];
            const auto& r = rect[k];
            auto q = L.aQ();
            const int ng = L.ng;
            for (int j = -ng; j < L.ny + ng; ++j)
                for (int i = -ng; i < L.nx + ng; ++i) {
                    if (i >= 0 && i < L.nx && j >= 0 && j < L.ny) continue;
                    const int I = r[0] + i, J = r[1] + j;
                    std::array<Real, 4> v{0.0, 0.0, 0.0, 0.0};
                    const bool inside = I >= 0 && I < nxf && J >= 0 && J < nyf;
                    if (!fine_at(I, J, v) && inside) v = interp(I, J);
                    for (int n = 0; n < 4; ++n) q(i, j, 0, n) = v[n];
                }
        }
    }

    void init_fine_from_coarse() {
        for (size_t k = 0; k < P.size(); ++k) {
            auto q = P[k].aQ();
            const auto& r = rect[k];
            for (int j = 0; j < r[3]; ++j)
                for (int i = 0; i < r[2]; ++i) {
                    const auto v = interp(r[0] + i, r[1] + j);
                    for (int n = 0; n < 4; ++n) q(i, j, 0, n) = v[n];
                }
        }
    }

    void fine_step(Real t, Real dt) {
        for (auto& L : P) L.copy_valid(L.Qold, L.Q);
        for (int s = 0; s < 2; ++s) {
            fill_fine_ghosts();
            for (auto& L : P) L.stage(2, t, dt, true);
        }
        for (auto& L : P) L.heun();
        for (auto& L : P) L.update_state(t);
    }

    void average_down() {
        auto qc = L0.aQ();
        for (size_t k = 0; k < P.size(); ++k) {
            auto q = P[k].aQ();
            const auto& r = rect[k];
            for (int j = 0; j < r[3] / 2; ++j)
                for (int i = 0; i < r[2] / 2; ++i) {
                    const int ic = (r[0] >> 1) + i, jc = (r[1] >> 1) + j;
                    Real s[3] = {0.0, 0.0, 0.0};
                    for (int d = 0; d < 4; ++d) {
                        const int fi = 2 * i + (d & 1), fj = 2 * j + (d >> 1);
                        s[0] += q(fi, fj, 0, 1) + q(fi, fj, 0, 0);
                        s[1] += q(fi, fj, 0, 2);
                        s[2] += q(fi, fj, 0, 3);
                    }
                    qc(ic, jc, 0, 1) = 0.25 * s[0] - qc(ic, jc, 0, 0);
                    qc(ic, jc, 0, 2) = 0.25 * s[1];
                    qc(ic, jc, 0, 3) = 0.25 * s[2];
                }
        }
    }

    void coarse_step(Real t, Real dt) {
        L0.advance(t, dt, true);
        fine_step(t, 0.5 * dt);
        fine_step(t + 0.5 * dt, 0.5 * dt);
        average_down();
    }

    // ZoomyAmr::ComputeDt's law on the CFL maximum gm (ZoomyAmr.cpp:499-514)
    Real dt_of(Real gm) const {
        const zfv_config& c = L0.cfg;
        if (gm < 1e-14) return c.dtmax;
        const Real div = Real(c.cfl_dimension) * Real(c.cfl_degree_factor);
        return amrex::max(amrex::min(c.cfl / (div * gm), c.dtmax), c.dtmin);
    }

    // One coarse step under the per-level law; returns the base level's dt.
    Real coarse_step_per_level(Real t) {
        L0.update_state(t);
        Real m0 = 0.0;
        L0.compute_dt(&m0);
        Real dt0 = dt_of(m0);
        const Real remaining = L0.cfg.time_end - t;
        dt0 = remaining > 0.0 ? amrex::min(dt0, remaining) : 0.0;
        L0.advance(t, dt0, true);
        Real tf = t;
        for (int i = 0; i < 2; ++i) {
            Real gm = 0.0;
            for (auto& L : P) {
                L.update_state(tf);
                Real m = 0.0;
                L.compute_dt(&m);
                if (m > gm) gm = m;
            }
            const Real dtf = dt_of(gm);
            fine_step(tf, dtf);
            tf += dtf;
        }
        average_down();
        return dt0;
    }
};

}  // namespace zoracle
