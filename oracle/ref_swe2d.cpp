// Reference make_rhs.H instantiated for the 2-D SWE model — TEST INFRASTRUCTURE ONLY.
#include "ref_kernels.H"
namespace ref_swe2d {
using Model = zb::SWE<double, 2>;
using Numerics = zb::SWENumerics<double, 2>;
#include "make_rhs.H"
}
ZREF_DEFINE_KERNELS(RefSWE2D, ref_swe2d)
