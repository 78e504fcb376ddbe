// The FP32 chosen form's kernels for ONE strip shape (fv32_shapes.H), chosen
// at compile time by -DZFV32_SHAPE=<index>; the build compiles this file once
// per shape, with the same flags as zoomy_fv32.cu (FMA contraction, the
// hardware's approximate FP32 division and square root).
#include "zfv_internal.H"
#include "fv32_common.cuh"
#include "fv32_batch.cuh"
#include "fv32_shapes.H"

#ifndef ZFV32_SHAPE
#error "compile with -DZFV32_SHAPE=<strip shape index>"
#endif

#define ZFV32_CAT2(a, b) a##b
#define ZFV32_CAT(a, b) ZFV32_CAT2(a, b)

namespace zfv32 {
namespace {

constexpr int V = ZFV32_SHAPE;
static_assert(V >= 0 && V < kNumVariants, "strip shape index out of range");
constexpr int NW = kVarNW[V], CPT = kVarCPT[V], PK = kVarPK[V], PF = kVarPF[V];

void convert(int nu, cudaStream_t s, const BInst* d, const int2* u, int n_aux, bool exp) {
    if (exp) k32b_export<NW, CPT, PK><<<nu, 256, 0, s>>>(d, u, n_aux);
    else k32b_import<NW, CPT, PK><<<nu, 256, 0, s>>>(d, u);
}

void reduce(int nu, cudaStream_t s, const BInst* d, const int2* u, int n_aux, int what) {
    if (what == 0) k32b_reduce<NW, CPT, PK, 0><<<nu, 32 * NW, 0, s>>>(d, u, n_aux);
    else if (what == 2) k32b_reduce<NW, CPT, PK, 2><<<nu, 32 * NW, 0, s>>>(d, u, n_aux);
    else k32b_reduce<NW, CPT, PK, 1><<<nu, 32 * NW, 0, s>>>(d, u, n_aux);
}

template <bool W, bool I>
void step_t(int nu, cudaStream_t s, const BInst* d, const int2* u, int n_steps, int stages) {
    if (stages == 1) {
        launch_stage<S1, W, I, NW, CPT, PK, PF>(nu, s, d, u);
    } else if (stages == 2) {
        launch_stage<S2, W, I, NW, CPT, PK, PF>(nu, s, d, u);
    } else {
        for (int k = 0; k < n_steps; ++k) {
            launch_stage<S1, W, I, NW, CPT, PK, PF>(nu, s, d, u);
            launch_stage<S2, W, I, NW, CPT, PK, PF>(nu, s, d, u);
        }
    }
}

void step(int nu, cudaStream_t s, const BInst* d, const int2* u, bool wb, bool impl, int n_steps,
          int stages) {
    if (wb) {
        if (impl) step_t<true, true>(nu, s, d, u, n_steps, stages);
        else step_t<true, false>(nu, s, d, u, n_steps, stages);
    } else {
        if (impl) step_t<false, true>(nu, s, d, u, n_steps, stages);
        else step_t<false, false>(nu, s, d, u, n_steps, stages);
    }
}

}  // namespace

extern const ShapeOps ZFV32_CAT(kShapeOps, ZFV32_SHAPE) = {convert, reduce, step};

}  // namespace zfv32
