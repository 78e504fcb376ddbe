// Reference make_rhs.H instantiated for the 2-D shallow-moment model at level 2 — TEST INFRASTRUCTURE ONLY.
#include "ref_kernels.H"
namespace ref_sme2d {
using Model = zb::SME<double, 2, 2>;
using Numerics = zb::SMENumerics<double, 2, 2>;
#include "make_rhs.H"
}
ZREF_DEFINE_KERNELS(RefSME2D, ref_sme2d)
