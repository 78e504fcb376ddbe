// Kernel policy that routes the oracle driver's per-cell work through the
// reference's own Source/make_rhs.H — TEST INFRASTRUCTURE ONLY.
//
// make_rhs.H is header-only C++ against AMReX's Array4/SmallMatrix and the
// generated Model::/Numerics:: functions. It is compiled here unmodified,
// from where it lies in the reference tree, against the AMReX API shim in
// zoomy_amrex_b200/csrc/amrex_compat and the model headers (csrc/models),
// once per model in its own namespace (ref_swe1d.cpp, ref_swe2d.cpp,
// ref_sme1d.cpp, ref_sme2d.cpp). The
// reference's driver (ZoomyAmr.cpp) needs AMReX, MPI and generated headers and
// is not buildable here; the oracle's restated driver stands in for it.
#pragma once
#include "fv_oracle.H"
#include "swe.H"
#include "sme.H"

namespace zoracle {

template <class M, class N> struct RefKernels;

#define ZREF_DECLARE_KERNELS(NAME, M)                                                             \
struct NAME {                                                                                     \
    using Real = double;                                                                          \
    static constexpr int n_face_comp = 3 * M::n_dof_q + 2;                                        \
    using A4c = amrex::Array4<const Real>;                                                        \
    using A4 = amrex::Array4<Real>;                                                               \
    using VP = amrex::SmallMatrix<Real, M::n_parameters, 1>;                                      \
    using VX = amrex::SmallMatrix<Real, 3, 1>;                                                    \
    static void cell_rhs(int i, int j, A4c const& Q, A4c const& Qa, A4 const& RHS, Real dx,       \
                         Real dy, int order, bool impl, VP const& p, Real time, Real plox,        \
                         Real ploy, bool wb);                                                     \
    static void face_data(int i, int j, int dir, int order, A4c const& Q, A4c const& Qa,          \
                          A4 const& F, VP const& p, Real time, Real dx, Real dy, Real plox,       \
                          Real ploy, bool wb);                                                    \
    static void assemble(int i, int j, A4c const& Q, A4c const& Qa, A4c const& Fx,                \
                         A4c const& Fy, A4 const& RHS, Real dx, Real dy, bool impl, VP const& p,  \
                         Real time, Real plox, Real ploy, bool wb);                               \
    static void implicit_source(int i, int j, A4 const& Q, A4c const& Qa, Real dt, VP const& p,   \
                                Real time, VX const& X);                                          \
};

using RefModelSWE1D = zb::SWE<double, 1>;
using RefModelSWE2D = zb::SWE<double, 2>;
using RefModelSME2D = zb::SME<double, 2, 2>;
using RefModelSME1D = zb::SME<double, 1, 2>;
ZREF_DECLARE_KERNELS(RefSWE1D, RefModelSWE1D)
ZREF_DECLARE_KERNELS(RefSWE2D, RefModelSWE2D)
ZREF_DECLARE_KERNELS(RefSME2D, RefModelSME2D)
ZREF_DECLARE_KERNELS(RefSME1D, RefModelSME1D)

template <> struct RefKernels<zb::SWE<double, 1>, zb::SWENumerics<double, 1>> : RefSWE1D {};
template <> struct RefKernels<zb::SWE<double, 2>, zb::SWENumerics<double, 2>> : RefSWE2D {};
template <> struct RefKernels<zb::SME<double, 2, 2>, zb::SMENumerics<double, 2, 2>> : RefSME2D {};
template <> struct RefKernels<zb::SME<double, 1, 2>, zb::SMENumerics<double, 1, 2>> : RefSME1D {};

}  // namespace zoracle

// Defines NAME's members by forwarding to the make_rhs.H functions in namespace NS.
#define ZREF_DEFINE_KERNELS(NAME, NS)                                                             \
namespace zoracle {                                                                               \
void NAME::cell_rhs(int i, int j, A4c const& Q, A4c const& Qa, A4 const& RHS, Real dx, Real dy,   \
                    int order, bool impl, VP const& p, Real time, Real plox, Real ploy, bool wb) {\
    NS::compute_cell_rhs(i, j, Q, Qa, RHS, dx, dy, order, impl, p, time, plox, ploy, wb);         \
}                                                                                                 \
void NAME::face_data(int i, int j, int dir, int order, A4c const& Q, A4c const& Qa, A4 const& F,  \
                     VP const& p, Real time, Real dx, Real dy, Real plox, Real ploy, bool wb) {   \
    NS::compute_face_data(i, j, dir, order, Q, Qa, F, p, time, dx, dy, plox, ploy, wb);           \
}                                                                                                 \
void NAME::assemble(int i, int j, A4c const& Q, A4c const& Qa, A4c const& Fx, A4c const& Fy,      \
                    A4 const& RHS, Real dx, Real dy, bool impl, VP const& p, Real time, Real plox, \
                    Real ploy, bool wb) {                                                         \
    NS::assemble_cell_rhs(i, j, Q, Qa, Fx, Fy, RHS, dx, dy, impl, p, time, plox, ploy, wb);       \
}                                                                                                 \
void NAME::implicit_source(int i, int j, A4 const& Q, A4c const& Qa, Real dt, VP const& p,        \
                           Real time, VX const& X) {                                              \
    NS::apply_implicit_source(i, j, Q, Qa, dt, p, time, X);                                       \
}                                                                                                 \
}
