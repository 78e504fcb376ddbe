// Host build of the model headers (zoomy_amrex_b200/csrc/models/{swe,sme}.H)
// for CPU tests: plain C entry points that evaluate single Model::/Numerics::
// functions on given states, so tests can compare them with a symbolic
// derivation and with each other. Built by tests/test_sme_model.py with
// g++ -O2 -ffp-contract=off.
#include <cstring>
#include <type_traits>
#include "swe.H"
#include "sme.H"

namespace {

// Models with moment rows (the non-conservative products live there).
template <class M, class = void> struct requires_ncp : std::false_type {};
template <class M> struct requires_ncp<M, std::void_t<decltype(M::level)>> : std::true_type {};

template <class M>
typename M::VQ loadq(const double* q) {
    typename M::VQ v;
    for (int n = 0; n < M::n_dof_q; ++n) v(n, 0) = q[n];
    return v;
}
template <class M>
typename M::VP loadp(const double* p) {
    typename M::VP v;
    for (int n = 0; n < M::n_parameters; ++n) v(n, 0) = p[n];
    return v;
}
template <class M>
typename M::VA aux_of(typename M::VQ const& q, typename M::VP const& p) {
    typename M::VA a{};
    typename M::VX X{};
    return M::update_aux_variables(q, a, p, 0.0, X);
}

// what: 0 flux along D, 1 moment rows of B_D(q) dq, 2 source, 3 dS/dq (row-major),
//       4 dS/dhinv, 5 Gershgorin bound along D (out[0]), 6 numerical flux (qL = q, qR = dq),
//       7 numerical fluctuations (qL = q, qR = dq; 2 n values), 8 path product Btilde (qR - qL),
//       9 wall ghost state for the face normal e_D, 10 the block point-implicit increment (dt = dq[0])
template <class M, class N>
int eval(int what, int D, const double* q, const double* dq, const double* pp, double* out) {
    constexpr int n = M::n_dof_q;
    const auto Q = loadq<M>(q);
    const auto p = loadp<M>(pp);
    const auto a = aux_of<M>(Q, p);
    typename M::VX X{};
    typename M::VN nh{};
    nh(D, 0) = 1.0;
    switch (what) {
    case 0: {
        const auto F = (D == 0) ? M::template flux_dir<0>(Q, a, p) : M::template flux_dir<M::dimension - 1>(Q, a, p);
        for (int k = 0; k < n; ++k) out[k] = F(k, 0);
        return 0;
    }
    case 1: {
        if constexpr (requires_ncp<M>::value) {
            typename M::VQ o{};
            const auto dQ = loadq<M>(dq);
            if (D == 0) M::template ncp_moments<0>(Q, a(M::i_hinv, 0), dQ, o);
            else M::template ncp_moments<M::dimension - 1>(Q, a(M::i_hinv, 0), dQ, o);
            for (int k = 0; k < n; ++k) out[k] = o(k, 0);
            return 0;
        }
        return -1;
    }
    case 2: {
        const auto S = M::source(Q, a, p, 0.0, X);
        for (int k = 0; k < n; ++k) out[k] = S(k, 0);
        return 0;
    }
    case 3: {
        const auto J = M::source_jacobian_wrt_variables(Q, a, p);
        for (int k = 0; k < n * n; ++k) out[k] = J(k, 0);
        return 0;
    }
    case 4: {
        const auto J = M::source_jacobian_wrt_aux_variables(Q, a, p);
        for (int k = 0; k < n; ++k) out[k] = J(k * M::n_dof_qaux + M::i_hinv, 0);
        return 0;
    }
    case 5: {
        out[0] = N::local_max_abs_eigenvalue(Q, a, p, nh)(0, 0);
        return 0;
    }
    case 6: {
        const auto QR = loadq<M>(dq);
        const auto F = N::numerical_flux(Q, QR, a, aux_of<M>(QR, p), p, nh);
        for (int k = 0; k < n; ++k) out[k] = F(k, 0);
        return 0;
    }
    case 7: {
        const auto QR = loadq<M>(dq);
        const auto F = N::numerical_fluctuations(Q, QR, a, aux_of<M>(QR, p), p, nh);
        for (int k = 0; k < 2 * n; ++k) out[k] = F(k, 0);
        return 0;
    }
    case 10: {
        if constexpr (requires_ncp<M>::value) {   // the block point-implicit step, dt = dq[0]
            typename M::VQ d{};
            M::zb_implicit_increment(Q, a, p, dq[0], d);
            for (int k = 0; k < n; ++k) out[k] = d(k, 0);
            return 0;
        }
        return -1;
    }
    case 9: {
        const auto G = M::boundary_conditions(1, Q, a, nh, X, 0.0, 1.0);
        for (int k = 0; k < n; ++k) out[k] = G(k, 0);
        return 0;
    }
    case 8: {
        if constexpr (requires_ncp<M>::value) {
            const auto QR = loadq<M>(dq);
            const auto B = (D == 0) ? N::template path_product<0>(Q, QR, p)
                                    : N::template path_product<M::dimension - 1>(Q, QR, p);
            for (int k = 0; k < n; ++k) out[k] = B(k, 0);
            return 0;
        }
        return -1;
    }
    }
    return -1;
}

}  // namespace

extern "C" {

// model: 0 SWE, 1 SME; dim 1 or 2; level 0..3 (SME).
int model_eval(int model, int dim, int level, int what, int D, const double* q, const double* dq,
               const double* p, double* out) {
    using namespace zb;
    if (model == 0) {
        if (dim == 1) return eval<SWE<double, 1>, SWENumerics<double, 1>>(what, D, q, dq, p, out);
        return eval<SWE<double, 2>, SWENumerics<double, 2>>(what, D, q, dq, p, out);
    }
    if (dim == 1) {
        switch (level) {
        case 0: return eval<SME<double, 1, 0>, SMENumerics<double, 1, 0>>(what, D, q, dq, p, out);
        case 1: return eval<SME<double, 1, 1>, SMENumerics<double, 1, 1>>(what, D, q, dq, p, out);
        case 2: return eval<SME<double, 1, 2>, SMENumerics<double, 1, 2>>(what, D, q, dq, p, out);
        case 3: return eval<SME<double, 1, 3>, SMENumerics<double, 1, 3>>(what, D, q, dq, p, out);
        }
    } else {
        switch (level) {
        case 0: return eval<SME<double, 2, 0>, SMENumerics<double, 2, 0>>(what, D, q, dq, p, out);
        case 1: return eval<SME<double, 2, 1>, SMENumerics<double, 2, 1>>(what, D, q, dq, p, out);
        case 2: return eval<SME<double, 2, 2>, SMENumerics<double, 2, 2>>(what, D, q, dq, p, out);
        case 3: return eval<SME<double, 2, 3>, SMENumerics<double, 2, 3>>(what, D, q, dq, p, out);
        }
    }
    return -1;
}

}  // extern "C"
