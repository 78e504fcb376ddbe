// FP64 plain-form runners of the shallow-moment family at level 2
// (ZFV_MODEL_SME2D_L2, ZFV_MODEL_SME1D_L2). Built with --fmad=false like
// zoomy_fv.cu. The 2-D tile is 16 x 8 cells: with 8 state rows and 23 face
// components per face (make_rhs.H:315) a 16 x 8 tile holds 67 KB of shared
// memory, so three blocks fit an SM.
#include "fv_runner64.cuh"
#include "sme.H"

namespace zfvi {
Runner* make_runner_fp64_sme2d_l2(zfv_handle* h) {
    return new zfv64::RunnerT<zb::SME<double, 2, 2>, zb::SMENumerics<double, 2, 2>, 16, 8>(h);
}
Runner* make_runner_fp64_sme1d_l2(zfv_handle* h) {
    return new zfv64::RunnerT<zb::SME<double, 1, 2>, zb::SMENumerics<double, 1, 2>, 128, 1>(h);
}
}  // namespace zfvi
