// FP64 plain-form runners of the shallow-water family (ZFV_MODEL_SWE1D,
// ZFV_MODEL_SWE2D). Built with --fmad=false like zoomy_fv.cu.
#include "fv_runner64.cuh"

namespace zfvi {
Runner* make_runner_fp64_swe1d(zfv_handle* h) {
    return new zfv64::RunnerT<zb::SWE<double, 1>, zb::SWENumerics<double, 1>, 128, 1>(h);
}
Runner* make_runner_fp64_swe2d(zfv_handle* h) {
    return new zfv64::RunnerT<zb::SWE<double, 2>, zb::SWENumerics<double, 2>, 32, 8>(h);
}
}  // namespace zfvi
