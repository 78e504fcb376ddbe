// C entry points of the reference-make_rhs.H build — TEST INFRASTRUCTURE ONLY.
#define ZORACLE_PREFIX ref_
#include "ref_kernels.H"
#include "oracle_api.H"

ZORACLE_DEFINE_API(zoracle::RefKernels)
