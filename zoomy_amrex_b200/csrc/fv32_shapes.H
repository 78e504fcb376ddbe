// Compiled strip shapes of the FP32 chosen form and the table of their
// launchers. Each shape's kernels are instantiated in a translation unit of
// their own (zoomy_fv32_shape.cu compiled once per shape with
// -DZFV32_SHAPE=<index>), so the shapes build in parallel; zoomy_fv32.cu
// reaches them through kShapeTable.
//
// A shape is (warps per block NW, rows per warp CPT = cells per thread,
// columns per lane PK, flags PF). A strip is 30 * PK columns x (NW * CPT)
// rows; PK = 2 is the packed-FP32 paired-column sweep. PF bits:
//   1  stage 2 stages its update's own inputs in shared memory with
//      asynchronous copies issued at the top of each row;
//   2  the stage-2 kernel is capped at 128 registers (4 blocks of 128
//      threads per SM instead of 3, at the cost of some spilling).
// (Holding both stages to 5 or 6 blocks per SM, at most 102 / 85
// registers, and unrolling the paired row loop by 4 were measured slower at
// 4096^2 -- spilling and instruction-cache misses -- and are not compiled.)
// Short strips (4 or 2 rows per warp) spend more on the y halo but finish a
// unit sooner: levels of a few million cells (AMR levels, ensemble boxes)
// fill the GPU for about one wave, so a launch there lasts about as long as
// one unit takes.
#pragma once
#include <cuda_runtime.h>

namespace zfv32 {

struct BInst;

constexpr int kNumVariants = 13;
constexpr int kVarNW[kNumVariants] = {4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4};
constexpr int kVarCPT[kNumVariants] = {16, 8, 16, 8, 16, 8, 16, 8, 16, 8, 4, 4, 2};
constexpr int kVarPK[kNumVariants] = {1, 1, 2, 2, 1, 1, 2, 2, 2, 2, 1, 2, 2};
constexpr int kVarPF[kNumVariants] = {0, 0, 0, 0, 1, 1, 1, 1, 3, 3, 1, 3, 3};
// Strip shape used until a caller picks one (zfv_set_variant /
// zfv_batch_set_variant): 4 warps x 8 rows, column pairs, stage-2 staging with
// the 128-register stage 2 -- the shape measured fastest on large levels.
constexpr int kDefaultVariant = 9;

// Launchers of one shape's kernels over a batch's unit table.
struct ShapeOps {
    // FP64 reference layout -> FP32 state (exp == false) or back (exp == true)
    void (*convert)(int n_units, cudaStream_t s, const BInst* d, const int2* u, int n_aux, bool exp);
    // grid reduction per instance: what 0 = ComputeDt from the stored aux, 1 = mass,
    // 2 = ComputeDt of the current state
    void (*reduce)(int n_units, cudaStream_t s, const BInst* d, const int2* u, int n_aux, int what);
    // stages 3 = both stages of n_steps steps; 1 or 2 = that stage alone, once
    void (*step)(int n_units, cudaStream_t s, const BInst* d, const int2* u, bool wb, bool impl,
                 int n_steps, int stages);
};

#define ZFV32_SHAPE_LIST(X) X(0) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12)
#define ZFV32_DECLARE_SHAPE(k) extern const ShapeOps kShapeOps##k;
ZFV32_SHAPE_LIST(ZFV32_DECLARE_SHAPE)

}  // namespace zfv32
