// CPU oracle shared library (the restatement) — TEST INFRASTRUCTURE ONLY.
#define ZORACLE_PREFIX oracle_
#include "oracle_api.H"

ZORACLE_DEFINE_API(zoracle::OracleKernels)

extern "C" void oracle_init_solution(int ncomp, int nx, int ny, const double* lo, const double* hi,
                                     double* v) {
    zoracle::init_solution(ncomp, nx, ny, lo, hi, v);
}

#include "fv_oracle_amr.H"

// Two-level AMR run (fv_oracle_amr.H): base state (4, ny, nx) in/out, fine
// patches as rectangles {i0, j0, nx, ny} in fine cells; the fine patches
// start as the interpolation of the base state and are returned
// concatenated, patch after patch, each (4, ny_p, nx_p). per_level = 0:
// coarse steps of dt (fine dt / 2); 1: the reference's per-level CFL law
// (dt unused). *t_out: the base level's time at the end.
extern "C" int oracle_amr2_run(const zfv_config* cfg, double* Q0, const int* rects, int n_rects, int n_steps,
                               double dt, int per_level, double* fine_out, double* t_out) {
    if (cfg->model != ZFV_MODEL_SWE2D) return -1;
    using M = zb::SWE<double, 2>;
    using N = zb::SWENumerics<double, 2>;
    zoracle::Hierarchy2<M, N, zoracle::OracleKernels<M, N>> H(*cfg, rects, n_rects);
    std::vector<double> A(size_t(M::n_dof_qaux) * cfg->nx * cfg->ny, 0.0);
    H.L0.load(Q0, A.data());
    H.L0.update_state(0.0);
    H.init_fine_from_coarse();
    for (auto& L : H.P) L.update_state(0.0);
    double t = 0.0;
    for (int s = 0; s < n_steps; ++s) {
        if (per_level) {
            t += H.coarse_step_per_level(t);
        } else {
            H.coarse_step(t, dt);
            t += dt;
        }
    }
    if (t_out) *t_out = t;
    H.L0.store(Q0, nullptr);
    size_t off = 0;
    for (auto& L : H.P) {
        L.store(fine_out + off, nullptr);
        off += size_t(4) * L.nx * L.ny;
    }
    return 0;
}
