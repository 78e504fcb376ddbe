// Reference make_rhs.H instantiated for the 1-D SWE model — TEST INFRASTRUCTURE ONLY.
#include "ref_kernels.H"
namespace ref_swe1d {
using Model = zb::SWE<double, 1>;
using Numerics = zb::SWENumerics<double, 1>;
#include "make_rhs.H"
}
ZREF_DEFINE_KERNELS(RefSWE1D, ref_swe1d)
