// C entry points of the CPU oracle — TEST INFRASTRUCTURE ONLY.
// One set of functions per kernel policy: PREFIX(run) etc. are defined by the
// translation unit that includes this file with ZORACLE_PREFIX set
// (oracle_* for the restatement, ref_* for the reference's make_rhs.H).
#pragma once
#include <cstdio>
#include <omp.h>
#include "fv_oracle.H"
#include "swe.H"
#include "sme.H"

#define ZO_CAT2(a, b) a##b
#define ZO_CAT(a, b) ZO_CAT2(a, b)
#define ZO_FN(name) ZO_CAT(ZORACLE_PREFIX, name)

namespace zoracle {

template <template <class, class> class Kern, class F>
int dispatch(const zfv_config* cfg, F&& f) {
    switch (cfg->model) {
    case ZFV_MODEL_SWE1D: {
        using M = zb::SWE<double, 1>; using N = zb::SWENumerics<double, 1>;
        Level<M, N, Kern<M, N>> L(*cfg);
        return f(L);
    }
    case ZFV_MODEL_SWE2D: {
        using M = zb::SWE<double, 2>; using N = zb::SWENumerics<double, 2>;
        Level<M, N, Kern<M, N>> L(*cfg);
        return f(L);
    }
    case ZFV_MODEL_SME2D_L2: {
        using M = zb::SME<double, 2, 2>; using N = zb::SMENumerics<double, 2, 2>;
        Level<M, N, Kern<M, N>> L(*cfg);
        return f(L);
    }
    case ZFV_MODEL_SME1D_L2: {
        using M = zb::SME<double, 1, 2>; using N = zb::SMENumerics<double, 1, 2>;
        Level<M, N, Kern<M, N>> L(*cfg);
        return f(L);
    }
    default: return -1;
    }
}

}  // namespace zoracle

#define ZORACLE_DEFINE_API(KERN)                                                                   \
extern "C" {                                                                                       \
/* Evolve (ZoomyAmr.cpp:767-816) from (Q, aux); writes the final state back. */                    \
int ZO_FN(run)(const zfv_config* cfg, double* Q, double* aux, int max_steps, int face_based,        \
               double* log3, int log_cap, int64_t* n_steps, double* t_out, int* mood_redos) {      \
    return zoracle::dispatch<KERN>(cfg, [&](auto& L) {                                             \
        L.load(Q, aux);                                                                            \
        while (!L.done() && (max_steps < 0 || L.step < max_steps)) L.time_step(face_based != 0);   \
        L.store(Q, aux);                                                                           \
        for (size_t s = 0; s < L.log.size() && (int)s < log_cap; ++s) {                            \
            log3[3 * s] = L.log[s].dt; log3[3 * s + 1] = L.log[s].time;                            \
            log3[3 * s + 2] = L.log[s].mass;                                                       \
        }                                                                                          \
        *n_steps = L.step; *t_out = L.time; *mood_redos = L.mood_redos;                            \
        return 0;                                                                                  \
    });                                                                                            \
}                                                                                                  \
/* UpdateState + FillPatch/FillPhysicalBC; grown arrays out. */                                    \
int ZO_FN(fill_ghosts)(const zfv_config* cfg, const double* Q, const double* aux, double time,     \
                       double* Qg, double* auxg) {                                                 \
    return zoracle::dispatch<KERN>(cfg, [&](auto& L) {                                             \
        L.load(Q, aux); L.update_state(time); L.fill_physical_bc(time);                            \
        std::memcpy(Qg, L.Q.data(), L.Q.size() * sizeof(double));                                 \
        std::memcpy(auxg, L.Qa.data(), L.Qa.size() * sizeof(double));                             \
        return 0;                                                                                  \
    });                                                                                            \
}                                                                                                  \
/* UpdateState + ghost fill + one RHS at the configured order; valid RHS out. */                   \
int ZO_FN(rhs)(const zfv_config* cfg, const double* Q, const double* aux, double time,             \
               int face_based, double* rhs) {                                                      \
    return zoracle::dispatch<KERN>(cfg, [&](auto& L) {                                             \
        L.load(Q, aux); L.update_state(time); L.fill_physical_bc(time);                            \
        L.rhs(cfg->spatial_order, time, face_based != 0);                                          \
        std::swap(L.Q, L.Rhs); L.store(rhs, nullptr); return 0;                                    \
    });                                                                                            \
}                                                                                                  \
/* ComputeDt on (Q, aux) as given. */                                                              \
int ZO_FN(compute_dt)(const zfv_config* cfg, const double* Q, const double* aux, double* dt,      \
                      double* max_inv) {                                                           \
    return zoracle::dispatch<KERN>(cfg, [&](auto& L) {                                             \
        L.load(Q, aux); *dt = L.compute_dt(max_inv); return 0;                                     \
    });                                                                                            \
}                                                                                                  \
/* UpdateState on the valid cells, in place. */                                                    \
int ZO_FN(update_state)(const zfv_config* cfg, double* Q, double* aux, double time) {              \
    return zoracle::dispatch<KERN>(cfg, [&](auto& L) {                                             \
        L.load(Q, aux); L.update_state(time); L.store(Q, aux); return 0;                           \
    });                                                                                            \
}                                                                                                  \
/* One Advance (SSP-RK2 step incl. final UpdateState) with a given dt. */                          \
int ZO_FN(advance)(const zfv_config* cfg, double* Q, double* aux, double time, double dt,         \
                   int face_based) {                                                               \
    return zoracle::dispatch<KERN>(cfg, [&](auto& L) {                                             \
        L.load(Q, aux); L.advance(time, dt, face_based != 0); L.store(Q, aux); return 0;           \
    });                                                                                            \
}                                                                                                  \
void ZO_FN(set_threads)(int n) { if (n > 0) omp_set_num_threads(n); }                              \
int ZO_FN(max_threads)(void) { return omp_get_max_threads(); }                                     \
}
