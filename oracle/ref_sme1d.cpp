// Reference make_rhs.H instantiated for the 1-D shallow-moment model at level 2 — TEST INFRASTRUCTURE ONLY.
#include "ref_kernels.H"
namespace ref_sme1d {
using Model = zb::SME<double, 1, 2>;
using Numerics = zb::SMENumerics<double, 1, 2>;
#include "make_rhs.H"
}
ZREF_DEFINE_KERNELS(RefSME1D, ref_sme1d)
