// FP32 chosen form of the families without a hand-tuned sweep
// (ZFV_PREC_FP32 with ZFV_MODEL_SME2D_L2, and ZFV_MODEL_SWE2D at spatial
// order 1 or with positivity "mood", which the shallow-water sweep does not
// implement): the generic tile kernels of fv32_tile.cuh behind the Runner
// interface. Order 2 runs the two SSP-RK2 stages, order 1 one forward-Euler
// stage per step; MOOD adds the candidate, commit and order-1 redo launches
// (the redo stages return at once for an untroubled step). Compiled with FMA contraction
// and the hardware's approximate FP32 division and square root, like
// zoomy_fv32.cu.
//
// Tile shapes (zfv_set_variant): 0 = 32 x 8 cells, 1 = 16 x 8, 2 = 32 x 4,
// staged by plain loads; 3, 4, 5 = the same shapes staged by TMA
// (cp.async.bulk.tensor boxes of the bed, state and increment planes, which
// needs nx a multiple of 4 and 16-byte aligned buffers). The shape and the
// staging change the launch grid and the copy engine only; every variant
// computes the same faces and updates in the same order, so results are
// identical.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <cuda.h>
#include <cuda_runtime.h>

#include "zfv_internal.H"
#include "sme.H"
#include "swe.H"
#include "fv32_tile.cuh"

using namespace zfvi;

namespace zfv32t {

constexpr int kTileShapes = 3;
constexpr int kTileVariants = 2 * kTileShapes;
constexpr int kTileTX[kTileShapes] = {32, 16, 32};
constexpr int kTileTY[kTileShapes] = {8, 8, 4};

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library links the CUDA runtime only).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<EncodeTiledFn>(f);
    }();
    return fn;
}

// A 3-D (nx, ny, planes) FP32 view with a (box_x, box_y, planes) box;
// cells outside the view read as zero.
int encode_planes(CUtensorMap* m, const float* base, int nx, int ny, int planes, int box_x, int box_y) {
    EncodeTiledFn enc = encode_tiled();
    if (!enc) return fail(-3, "zfv_set_variant: cuTensorMapEncodeTiled is not available");
    const cuuint64_t dims[3] = {cuuint64_t(nx), cuuint64_t(ny), cuuint64_t(planes)};
    const cuuint64_t strides[2] = {cuuint64_t(nx) * sizeof(float), cuuint64_t(nx) * ny * sizeof(float)};
    const cuuint32_t box[3] = {cuuint32_t(box_x), cuuint32_t(box_y), cuuint32_t(planes)};
    const cuuint32_t elem[3] = {1, 1, 1};
    const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, elem,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(-3, "cuTensorMapEncodeTiled failed (%d)", int(r));
    return 0;
}

template <class F>
struct RunnerTile final : Runner {
    static constexpr int NP = F::np, nq = F::nq, ne = F::ne;
    zfv_handle* h;
    TileParams<NP> L;
    int var = 0;
    bool order1 = false;
    bool mood = false;     // positivity "mood" at order 2

    explicit RunnerTile(zfv_handle* hh) : h(hh) {
        const zfv_config& c = h->cfg;
        std::memset(&L, 0, sizeof L);
        L.nx = c.nx; L.ny = c.ny;
        L.plane = (long long)c.nx * c.ny;
        L.dx = (c.prob_hi[0] - c.prob_lo[0]) / c.nx;
        L.dy = (c.prob_hi[1] - c.prob_lo[1]) / c.ny;
        L.plox = c.prob_lo[0]; L.ploy = c.prob_lo[1];
        L.fdx = float(L.dx); L.fdy = float(L.dy);
        L.rdx = float(1.0 / L.dx); L.rdy = float(1.0 / L.dy);
        for (int k = 0; k < NP; ++k) { L.p[k] = c.params[k]; L.pf[k] = float(c.params[k]); }
        for (int s = 0; s < 4; ++s) L.bc_tag[s] = c.bc_tag[s];
        L.cfl = c.cfl; L.dtmin = c.dtmin; L.dtmax = c.dtmax; L.time_end = c.time_end;
        L.max_step = c.max_step; L.cfl_dimension = c.cfl_dimension; L.cfl_degree_factor = c.cfl_degree_factor;
    }

    template <int V, bool TMA> using ShapeV = TShape<F, kTileTX[V], kTileTY[V], TMA>;

    // tensor maps of the last (Q, scratch) pair the TMA variants ran on
    TileMaps maps{};
    const void* maps_q = nullptr;
    const char* maps_scratch = nullptr;

    int max_blocks() const {
        int m = 0;
        for (int v = 0; v < kTileShapes; ++v)
            m = std::max(m, ((L.nx + kTileTX[v] - 1) / kTileTX[v]) * ((L.ny + kTileTY[v] - 1) / kTileTY[v]));
        return std::max(m, kReduceBlocksMax);
    }

    template <int V, int MODE, bool WB, bool IMPL, bool TMA>
    int set_smem1() {
        return cuda_check(cudaFuncSetAttribute(k32t_stage<F, MODE, WB, IMPL, kTileTX[V], kTileTY[V], TMA>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               int(ShapeV<V, TMA>::smem_bytes)),
                          "cudaFuncSetAttribute (FP32 tile)");
    }
    template <int V, bool WB, bool IMPL, bool TMA>
    int set_smem_modes() {
        return set_smem1<V, T_S1, WB, IMPL, TMA>() | set_smem1<V, T_S2, WB, IMPL, TMA>() |
               set_smem1<V, T_ONE, WB, IMPL, TMA>() | set_smem1<V, T_S2M, WB, IMPL, TMA>() |
               set_smem1<V, T_R1, WB, IMPL, TMA>() | set_smem1<V, T_R2, WB, IMPL, TMA>();
    }
    template <int V, bool WB, bool IMPL>
    int set_smem2() { return set_smem_modes<V, WB, IMPL, false>() | set_smem_modes<V, WB, IMPL, true>(); }
    template <int V>
    int set_smem_v() {
        return set_smem2<V, false, false>() | set_smem2<V, false, true>() | set_smem2<V, true, false>() |
               set_smem2<V, true, true>();
    }

    // TMA needs 16-byte row and plane strides and 16-byte aligned planes
    bool tma_ok(const void* Q) const {
        return L.nx % 4 == 0 && (reinterpret_cast<uintptr_t>(Q) & 15) == 0;
    }
    int ensure_maps(const void* Q, const char* scratch) {
        if (Q == maps_q && scratch == maps_scratch) return 0;
        if (!tma_ok(Q)) return fail(-1, "zfv: the TMA tile variants need nx %% 4 == 0 and a 16-byte aligned state");
        const int v = var - kTileShapes;
        const int bw = kTileTX[v] + 8, bh = kTileTY[v] + 4;
        const TileBufs B = bufs(Q, const_cast<char*>(scratch));
        int rc = encode_planes(&maps.bed, B.bed, L.nx, L.ny, 1, bw, bh);
        if (!rc) rc = encode_planes(&maps.qs, B.Qs, L.nx, L.ny, ne, bw, bh);
        if (!rc) rc = encode_planes(&maps.alt, B.alt, L.nx, L.ny, ne, bw, bh);
        if (!rc) rc = encode_planes(&maps.inc, B.inc, L.nx, L.ny, ne, bw, bh);
        if (rc) { maps_q = nullptr; maps_scratch = nullptr; return rc; }
        maps_q = Q;
        maps_scratch = scratch;
        return 0;
    }

    int setup() override {
        const zfv_config& c = h->cfg;
        if (c.spatial_order != 1 && c.spatial_order != 2)
            return fail(-2, "zfv_create: the FP32 form implements spatial_order 1 and 2");
        order1 = c.spatial_order == 1;
        if (c.clamp_positivity) return fail(-1, "zfv_create: the FP32 form does not implement clamp_positivity");
        mood = c.positivity_mood && c.spatial_order == 2;   // as the FP64 form: MOOD redoes order-2 steps
        if (c.implicit_global && c.implicit_source)
            return fail(-1, "zfv_create: implicit_global is built for the FP64 form");
        return set_smem_v<0>() | set_smem_v<1>() | set_smem_v<2>();
    }

    void layout(ScratchLayout& S) const override {
        const size_t pb = size_t(L.plane) * sizeof(float);
        S.state = 0;
        S.partials = align_up(sizeof(zfv::DevState));
        S.log = S.partials + align_up(sizeof(double) * 2 * size_t(max_blocks()));
        S.stage = S.log + align_up(sizeof(double) * 3 * kLogCap);   // inc1
        S.alt = S.stage + align_up(pb * ne);
        S.lo = S.alt + align_up(pb * ne);
        S.jfnk = 0;
        S.lo2 = mood ? S.lo + align_up(pb * ne) : 0;
        S.total = (mood ? S.lo2 : S.lo) + align_up(pb * ne);
    }

    TileBufs bufs(const void* Q, char* scratch) const {
        TileBufs B;
        const ScratchLayout& S = h->lay;
        float* q = static_cast<float*>(const_cast<void*>(Q));
        B.bed = q;
        B.Qs = q + L.plane;
        B.alt = reinterpret_cast<float*>(scratch + S.alt);
        B.inc = reinterpret_cast<float*>(scratch + S.stage);
        B.lo = reinterpret_cast<float*>(scratch + S.lo);
        B.lo2 = mood ? reinterpret_cast<float*>(scratch + S.lo2) : nullptr;
        B.st = reinterpret_cast<zfv::DevState*>(scratch + S.state);
        B.partials = reinterpret_cast<double*>(scratch + S.partials);
        B.log3 = reinterpret_cast<double*>(scratch + S.log);
        B.log_cap = kLogCap;
        return B;
    }

    int reduce_blocks() const {
        long long need = (L.plane + kReduceNT - 1) / kReduceNT;
        return int(need < kReduceBlocksMax ? (need > 0 ? need : 1) : kReduceBlocksMax);
    }

    int begin(const void* Q, const void* A, char* scratch, cudaStream_t s) override {
        aux_bound = static_cast<double*>(const_cast<void*>(A));
        const TileBufs B = bufs(Q, scratch);
        k32t_init<NP><<<1, 1, 0, s>>>(B.st, L);
        k32t_reduce<F, kReduceNT, 0><<<reduce_blocks(), kReduceNT, 0, s>>>(L, B, (const double*)A);
        return cuda_check(cudaGetLastError(), "zfv_begin launch (FP32 tile)");
    }

    int total_mass(const void* Q, char* scratch, cudaStream_t s) override {
        k32t_reduce<F, kReduceNT, 1><<<reduce_blocks(), kReduceNT, 0, s>>>(L, bufs(Q, scratch), nullptr);
        return cuda_check(cudaGetLastError(), "zfv_total_mass launch (FP32 tile)");
    }

    template <int V, bool WB, bool IMPL, bool TMA>
    void step_v(const TileBufs& B, int n, cudaStream_t s) {
        constexpr int TX = kTileTX[V], TY = kTileTY[V];
        const dim3 grid((L.nx + TX - 1) / TX, (L.ny + TY - 1) / TY, 1);
        const size_t sm = ShapeV<V, TMA>::smem_bytes;
        for (int k = 0; k < n; ++k) {
            if (order1) {
                k32t_stage<F, T_ONE, WB, IMPL, TX, TY, TMA><<<grid, TX * TY, sm, s>>>(L, B, 0, maps);
            } else if (mood) {
                // ZoomyAmr.cpp:699-730: candidate, then commit or whole-step order-1 redo
                k32t_stage<F, T_S1, WB, IMPL, TX, TY, TMA><<<grid, TX * TY, sm, s>>>(L, B, 1, maps);
                k32t_stage<F, T_S2M, WB, IMPL, TX, TY, TMA><<<grid, TX * TY, sm, s>>>(L, B, 1, maps);
                k32t_mood_commit<F, kReduceNT><<<reduce_blocks(), kReduceNT, 0, s>>>(L, B);
                k32t_stage<F, T_R1, WB, IMPL, TX, TY, TMA><<<grid, TX * TY, sm, s>>>(L, B, 0, maps);
                k32t_stage<F, T_R2, WB, IMPL, TX, TY, TMA><<<grid, TX * TY, sm, s>>>(L, B, 0, maps);
            } else {
                k32t_stage<F, T_S1, WB, IMPL, TX, TY, TMA><<<grid, TX * TY, sm, s>>>(L, B, 1, maps);
                k32t_stage<F, T_S2, WB, IMPL, TX, TY, TMA><<<grid, TX * TY, sm, s>>>(L, B, 1, maps);
            }
        }
    }
    template <int V, bool TMA>
    void step_flags(const TileBufs& B, int n, cudaStream_t s) {
        const bool wb = h->cfg.well_balanced != 0, im = h->cfg.implicit_source != 0;
        if (wb) { if (im) step_v<V, true, true, TMA>(B, n, s); else step_v<V, true, false, TMA>(B, n, s); }
        else { if (im) step_v<V, false, true, TMA>(B, n, s); else step_v<V, false, false, TMA>(B, n, s); }
    }

    int evolve(void* Q, void* A, char* scratch, int n, cudaStream_t s) override {
        if (A) aux_bound = static_cast<double*>(A);
        if (var >= kTileShapes) {
            const int rc = ensure_maps(Q, scratch);
            if (rc) return rc;
        }
        const TileBufs B = bufs(Q, scratch);
        switch (var) {
        case 0: step_flags<0, false>(B, n, s); break;
        case 1: step_flags<1, false>(B, n, s); break;
        case 2: step_flags<2, false>(B, n, s); break;
        case 3: step_flags<0, true>(B, n, s); break;
        case 4: step_flags<1, true>(B, n, s); break;
        default: step_flags<2, true>(B, n, s); break;
        }
        return cuda_check(cudaGetLastError(), "zfv_evolve launch (FP32 tile)");
    }

    int state_import(const double* Q64, void* Q, char* scratch, cudaStream_t s) override {
        const int nb = int(std::min<long long>((L.plane + 255) / 256, 148LL * 16));
        k32t_import<F><<<std::max(nb, 1), 256, 0, s>>>(Q64, static_cast<float*>(Q), bufs(Q, scratch).lo, L.plane);
        int rc = cuda_check(cudaGetLastError(), "zfv_state_import launch (FP32 tile)");
        if (rc) return rc;
        // the imported state is in Q: parity 0
        const TileBufs B = bufs(Q, scratch);
        return cuda_check(cudaMemsetAsync(&B.st->parity, 0, sizeof(unsigned), s), "zfv_state_import parity");
    }

    int state_export(const void* Q, const char* scratch, double* Q64, cudaStream_t s) override {
        const TileBufs B = bufs(Q, const_cast<char*>(scratch));
        typename F::M64::VP p;
        for (int k = 0; k < NP; ++k) p(k, 0) = L.p[k];
        const int nb = int(std::min<long long>((L.plane + 255) / 256, 148LL * 16));
        k32t_export<F><<<std::max(nb, 1), 256, 0, s>>>(B.bed, B.Qs, B.alt, B.lo, B.st, Q64, aux_bound, p, L.plane);
        return cuda_check(cudaGetLastError(), "zfv_state_export launch (FP32 tile)");
    }

    // the aux that export refreshes: the last aux pointer begin / evolve saw
    double* aux_bound = nullptr;

    int update_state(void*, void*, double, cudaStream_t) override {
        return fail(-2, "zfv_update_state: validation entry of the FP64 form only");
    }
    int compute_dt(const void*, const void*, char*, cudaStream_t) override {
        return fail(-2, "zfv_compute_dt: validation entry of the FP64 form only");
    }
    int rhs(const void*, void*, double, cudaStream_t) override {
        return fail(-2, "zfv_rhs: validation entry of the FP64 form only");
    }
    int fill_ghosts(const void*, const void*, void*, void*, double, cudaStream_t) override {
        return fail(-2, "zfv_fill_ghosts: validation entry of the FP64 form only");
    }
    int set_variant(int v, cudaStream_t) override {
        if (v < 0 || v >= kTileVariants) return fail(-1, "zfv_set_variant: unknown tile shape %d", v);
        if (v >= kTileShapes && L.nx % 4 != 0)
            return fail(-1, "zfv_set_variant: the TMA tile variants need nx %% 4 == 0 (nx = %d)", L.nx);
        var = v;
        maps_q = nullptr;      // re-encode for the new box
        maps_scratch = nullptr;
        return 0;
    }
    int variant() const override { return var; }
};

}  // namespace zfv32t

namespace zfvi {
Runner* make_runner_fp32_generic(zfv_handle* h) {
    using F = zfv32t::Fam<zb::SME<double, 2, 2>, zb::SMENumerics<double, 2, 2>, zb::SME<float, 2, 2>,
                          zb::SMENumerics<float, 2, 2>>;
    using FS = zfv32t::Fam<zb::SWE<double, 2>, zb::SWENumerics<double, 2>, zb::SWE<float, 2>,
                           zb::SWENumerics<float, 2>>;
    switch (h->cfg.model) {
    case ZFV_MODEL_SME2D_L2: return new zfv32t::RunnerTile<F>(h);
    case ZFV_MODEL_SWE2D: return new zfv32t::RunnerTile<FS>(h);
    default: return nullptr;
    }
}
int fp32_tile_variants() { return zfv32t::kTileVariants; }
}  // namespace zfvi

extern "C" int zfv_generic_tile_variants(int* tx, int* ty, int* tma, int max_n) {
    for (int v = 0; v < zfv32t::kTileVariants && v < max_n; ++v) {
        const int s = v % zfv32t::kTileShapes;
        if (tx) tx[v] = zfv32t::kTileTX[s];
        if (ty) ty[v] = zfv32t::kTileTY[s];
        if (tma) tma[v] = v >= zfv32t::kTileShapes;
    }
    return zfv32t::kTileVariants;
}
