// The FP32 chosen form of the 2-D shallow-water step (ZFV_PREC_FP32).
//
// Same scheme as the FP64 plain form — MUSCL/minmod reconstruction of b and h,
// Audusse hydrostatic reconstruction, central flux + Rusanov D± fluctuations,
// point-implicit Manning source, SSP-RK2 (Heun) — evaluated so that FP32
// storage and arithmetic lose as little as possible:
//  * the state is stored as [b, eta = h + b, hu, hv] in FP32, and the slopes of
//    h are taken as d(eta) - d(b), so a lake at rest (eta constant, u = 0)
//    reconstructs eta at every face bit for bit: the face depths on both sides
//    of a face are equal and the hydrostatic pressure P(h) = (g/2) h^2 enters
//    the flux and the well-balancing bed source as the same FP32 values, which
//    cancel exactly;
//  * the update is compensated: stage 1 stores only its FP32 increment inc1,
//    stage 2 forms the small part t = lo + (inc1 + inc2)/2 in FP32 and adds it
//    to the stored value by an exact two-sum, giving Q^{n+1} = hi' + lo' as an
//    FP32 value (hi', the state the fluxes read) and an FP32 remainder (lo',
//    kept in scratch); so round-off of the stored state does not accumulate
//    step after step (only the FP32 rounding of t, relative to the step's
//    increment, enters);
//  * FP64 is used only in the point-implicit source solve of near-dry cells
//    (h < 1e-3) and in the mass sum.
// Kernels are compiled with FMA contraction on (this file only).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>
#include <cuda_runtime.h>

#include "zfv_internal.H"
#include "fv_kernels.cuh"
#include "swe.H"
#include "zb_portable_math.H"

using namespace zfvi;

#include "fv32_common.cuh"
#include "fv32_batch.cuh"
#include "fv32_shapes.H"
#include "fv32_amr.cuh"

namespace zfv32 {

#define ZFV32_SHAPE_PTR(k) &kShapeOps##k,
const ShapeOps* const kShapeTable[kNumVariants] = {ZFV32_SHAPE_LIST(ZFV32_SHAPE_PTR)};
#undef ZFV32_SHAPE_PTR

Params make_params(const zfv_config& c) {
    Params L;
    L.nx = c.nx; L.ny = c.ny; L.plane = (long long)c.nx * c.ny;
    L.dx = (c.prob_hi[0] - c.prob_lo[0]) / c.nx;
    L.dy = (c.prob_hi[1] - c.prob_lo[1]) / c.ny;
    L.plox = c.prob_lo[0]; L.ploy = c.prob_lo[1];
    L.fdx = float(L.dx); L.fdy = float(L.dy);
    L.rdx = float(1.0 / L.dx); L.rdy = float(1.0 / L.dy);
    L.rfdx = 1.0f / L.fdx; L.rfdy = 1.0f / L.fdy;
    L.gd = c.params[zb::swe_g]; L.exd = c.params[zb::swe_ex]; L.eyd = c.params[zb::swe_ey];
    L.nmd = c.params[zb::swe_n_m]; L.hfloord = c.params[zb::swe_h_floor]; L.epsd = c.params[zb::swe_eps];
    L.g = float(L.gd); L.ex = float(L.exd); L.ey = float(L.eyd); L.nm = float(L.nmd);
    L.hfloor = float(L.hfloord); L.eps = float(L.epsd);
    L.hwet = float(std::pow(L.epsd, 0.25) * 1.001);
    for (int s = 0; s < 4; ++s) L.bc_tag[s] = c.bc_tag[s];
    L.cfl = c.cfl; L.dtmin = c.dtmin; L.dtmax = c.dtmax; L.time_end = c.time_end;
    L.max_step = c.max_step; L.cfl_dimension = c.cfl_dimension; L.cfl_degree_factor = c.cfl_degree_factor;
    L.frame = nullptr;
    return L;
}

int units_of(const zfv_config& c, int v) {
    const int rows = kVarNW[v] * kVarCPT[v], sw = 30 * kVarPK[v];
    return ((c.nx + sw - 1) / sw) * ((c.ny + rows - 1) / rows);
}
int max_units_of(const zfv_config& c) {
    int m = 0;
    for (int v = 0; v < kNumVariants; ++v) m = std::max(m, units_of(c, v));
    return m;
}

// The batch engine: any number of FP32 SWE2D instances sharing one scheme
// (order 2, the same well_balanced / implicit_source flags).
struct BatchCore {
    static constexpr int n_aux = zb::SWE<double, 2>::n_dof_qaux;
    std::vector<zfv_config> cfg;
    std::vector<int> group;      // run-record group of each instance (own record if none)
    std::vector<const float*> frames;
    int n = 0;
    bool wb = false, impl = false;
    int variant = kDefaultVariant;
    // scratch layout
    size_t off_desc = 0, off_units = 0, off_status = 0;
    std::vector<size_t> off_state, off_part, off_log, off_alt, off_inc, off_lo;
    size_t total = 0;
    int max_units_total = 0;
    // bound buffers
    std::vector<BInst> desc;
    std::vector<int2> units;
    char* scratch = nullptr;
    bool bound = false;

    int init(const zfv_config* cfgs, int count, const int* groups = nullptr) {
        if (count < 1) return fail(-1, "zfv_batch_create: empty batch");
        n = count;
        cfg.assign(cfgs, cfgs + count);
        group.resize(n);
        for (int k = 0; k < n; ++k) {
            group[k] = groups ? groups[k] : k;
            if (group[k] < 0 || group[k] >= n) return fail(-1, "zfv_batch: group id %d out of range", group[k]);
        }
        frames.assign(n, nullptr);
        wb = cfg[0].well_balanced != 0;
        impl = cfg[0].implicit_source != 0;
        for (auto& c : cfg) {
            if (c.model != ZFV_MODEL_SWE2D || c.precision != ZFV_PREC_FP32)
                return fail(-1, "zfv_batch: instances must be ZFV_MODEL_SWE2D / ZFV_PREC_FP32");
            if (c.spatial_order != 2)
                return fail(-2, "zfv_batch: the FP32 form implements spatial_order 2 only");
            if ((c.well_balanced != 0) != wb || (c.implicit_source != 0) != impl)
                return fail(-1, "zfv_batch: all instances must share well_balanced and implicit_source");
            if (c.positivity_mood) return fail(-2, "zfv_batch: the FP32 form does not implement MOOD");
            if (c.clamp_positivity) return fail(-1, "zfv_batch: the FP32 form does not implement clamp_positivity");
            if (c.nx < 2 || c.ny < 2) return fail(-1, "zfv_batch: order 2 needs at least 2 cells per direction");
        }
        size_t o = 0;
        off_desc = o; o += align_up(sizeof(BInst) * n);
        max_units_total = 0;
        for (auto& c : cfg) max_units_total += max_units_of(c);
        off_units = o; o += align_up(sizeof(int2) * max_units_total);
        off_status = o; o += align_up(sizeof(zfv::DevState) * n);
        off_state.resize(n); off_part.resize(n); off_log.resize(n);
        off_alt.resize(n); off_inc.resize(n); off_lo.resize(n);
        // one run record, partials array and log per group (its first member's)
        std::vector<int> first(n, -1);
        std::vector<long long> group_units(n, 0);
        for (int k = 0; k < n; ++k) group_units[group[k]] += max_units_of(cfg[k]);
        for (int k = 0; k < n; ++k) {
            const size_t pb = size_t(cfg[k].nx) * cfg[k].ny * sizeof(float);
            const int g = group[k];
            if (first[g] < 0) {
                first[g] = k;
                off_state[k] = o; o += align_up(sizeof(zfv::DevState));
                off_part[k] = o; o += align_up(sizeof(double) * 2 * size_t(group_units[g]));
                off_log[k] = o; o += align_up(sizeof(double) * 3 * kLogCap);
            } else {
                off_state[k] = off_state[first[g]];
                off_part[k] = off_part[first[g]];
                off_log[k] = off_log[first[g]];
            }
            off_inc[k] = o; o += align_up(pb * 3);
            off_alt[k] = o; o += align_up(pb * 3);
            off_lo[k] = o; o += align_up(pb * 3);
        }
        total = o;
        desc.resize(n);
        return 0;
    }

    void build_units() {
        units.clear();
        const int rows = kVarNW[variant] * kVarCPT[variant], sw = 30 * kVarPK[variant];
        std::vector<int> base(n, 0);
        for (int k = 0; k < n; ++k) {
            const int nbx = (cfg[k].nx + sw - 1) / sw, nby = (cfg[k].ny + rows - 1) / rows;
            desc[k].nbx = nbx;
            desc[k].nby = nby;
            desc[k].unit_base = base[group[k]];     // this instance's first unit in its group
            base[group[k]] += nbx * nby;
            for (int u = 0; u < nbx * nby; ++u) units.push_back(make_int2(k, u));
        }
        for (int k = 0; k < n; ++k) desc[k].group_units = base[group[k]];
    }

    int upload(cudaStream_t s) {
        build_units();
        int rc = cuda_check(cudaMemcpyAsync(scratch + off_desc, desc.data(), sizeof(BInst) * n,
                                            cudaMemcpyHostToDevice, s), "zfv_batch descriptor upload");
        if (rc) return rc;
        rc = cuda_check(cudaMemcpyAsync(scratch + off_units, units.data(), sizeof(int2) * units.size(),
                                        cudaMemcpyHostToDevice, s), "zfv_batch unit upload");
        if (rc) return rc;
        return cuda_check(cudaStreamSynchronize(s), "zfv_batch upload sync");
    }

    int bind(void* const* Q, double* const* aux, char* scr, cudaStream_t s) {
        scratch = scr;
        for (int k = 0; k < n; ++k) {
            BInst& D = desc[k];
            std::memset(&D, 0, sizeof D);
            D.P = make_params(cfg[k]);
            const long long pl = D.P.plane;
            float* q = static_cast<float*>(Q[k]);
            D.bed = q;
            D.Qs = q + pl;
            D.alt = reinterpret_cast<float*>(scr + off_alt[k]);
            D.inc = reinterpret_cast<float*>(scr + off_inc[k]);
            D.lo = reinterpret_cast<float*>(scr + off_lo[k]);
            D.aux = aux ? aux[k] : nullptr;
            D.st = reinterpret_cast<zfv::DevState*>(scr + off_state[k]);
            D.partials = reinterpret_cast<double*>(scr + off_part[k]);
            D.log3 = reinterpret_cast<double*>(scr + off_log[k]);
            D.log_cap = kLogCap;
            D.P.frame = frames[k];
        }
        bound = true;
        return upload(s);
    }

    const BInst* d_desc() const { return reinterpret_cast<const BInst*>(scratch + off_desc); }
    const int2* d_units() const { return reinterpret_cast<const int2*>(scratch + off_units); }
    int nunits() const { return int(units.size()); }

    int set_frames(const float* const* f, cudaStream_t s) {
        for (int k = 0; k < n; ++k) {
            frames[k] = f ? f[k] : nullptr;
            desc[k].P.frame = frames[k];
        }
        return bound ? upload(s) : 0;
    }

    int set_dt(const double* dts_dev, cudaStream_t s) {
        k32b_set_dt<<<(n + 127) / 128, 128, 0, s>>>(d_desc(), n, dts_dev);
        return cuda_check(cudaGetLastError(), "zfv_batch_set_dt launch");
    }

    int set_variant(int v, cudaStream_t s) {
        if (v < 0 || v >= kNumVariants) return fail(-1, "zfv_batch_set_variant: unknown variant %d", v);
        variant = v;
        return bound ? upload(s) : 0;
    }

    const ShapeOps& ops() const { return *kShapeTable[variant]; }

    int convert(const double* const* q64, bool exp, cudaStream_t s) {
        for (int k = 0; k < n; ++k) desc[k].q64 = q64[k];
        int rc = upload(s);
        if (rc) return rc;
        ops().convert(nunits(), s, d_desc(), d_units(), n_aux, exp);
        rc = cuda_check(cudaGetLastError(), "zfv_batch import/export launch");
        if (rc) return rc;
        return cuda_check(cudaStreamSynchronize(s), "zfv_batch import/export sync");
    }

    int begin(cudaStream_t s) {
        k32b_init<<<(n + 127) / 128, 128, 0, s>>>(d_desc(), n);
        ops().reduce(nunits(), s, d_desc(), d_units(), n_aux, 0);
        return cuda_check(cudaGetLastError(), "zfv_batch begin launch");
    }

    int mass(cudaStream_t s) {
        ops().reduce(nunits(), s, d_desc(), d_units(), n_aux, 1);
        return cuda_check(cudaGetLastError(), "zfv_batch mass launch");
    }

    int compute_dt(cudaStream_t s) {
        ops().reduce(nunits(), s, d_desc(), d_units(), n_aux, 2);
        return cuda_check(cudaGetLastError(), "zfv_batch_compute_dt launch");
    }

    // stages: 3 = both stages of `nsteps` steps; 1 or 2 = that stage alone,
    // once (AMR boxes refill their ghost frames between the stages)
    int evolve(int nsteps, cudaStream_t s, int stages = 3) {
        ops().step(nunits(), s, d_desc(), d_units(), wb, impl, nsteps, stages);
        return cuda_check(cudaGetLastError(), "zfv_batch evolve launch");
    }

    int status(zfv_status* out, cudaStream_t s) {
        static_assert(sizeof(zfv_status) <= sizeof(zfv::DevState), "status fits the run record");
        zfv::DevState* dst = reinterpret_cast<zfv::DevState*>(scratch + off_status);
        k32b_status<<<(n + 127) / 128, 128, 0, s>>>(d_desc(), n, dst);
        std::vector<zfv::DevState> tmp(n);
        int rc = cuda_check(cudaMemcpyAsync(tmp.data(), dst, sizeof(zfv::DevState) * n,
                                            cudaMemcpyDeviceToHost, s), "zfv_batch status copy");
        if (rc) return rc;
        rc = cuda_check(cudaStreamSynchronize(s), "zfv_batch status sync");
        for (int k = 0; k < n; ++k) std::memcpy(&out[k], &tmp[k], sizeof(zfv_status));
        return rc;
    }
};

// ---------------------------------------------------------------------------
// Single level (zfv_create with ZFV_PREC_FP32): a batch of one. Q / aux /
// scratch are bound on first use and re-bound (a synchronous upload) if a
// later call passes different buffers; keep them fixed across CUDA-graph
// captured calls.
struct Runner32 final : Runner {
    zfv_handle* h;
    BatchCore core;
    const void* bq = nullptr; const void* ba = nullptr; const char* bs = nullptr;

    explicit Runner32(zfv_handle* hh) : h(hh) {}

    int setup() override { return core.init(&h->cfg, 1); }
    void layout(ScratchLayout& S) const override {
        S.state = core.off_state[0];
        S.partials = core.off_part[0];
        S.log = core.off_log[0];
        S.stage = core.off_inc[0];
        S.alt = core.off_alt[0];
        S.lo = core.off_lo[0];
        S.total = core.total;
    }
    int ensure_bound(const void* Q, const void* A, char* scratch, cudaStream_t s) {
        if (core.bound && Q == bq && A == ba && scratch == bs) return 0;
        void* qp = const_cast<void*>(Q);
        double* ap = static_cast<double*>(const_cast<void*>(A));
        int rc = core.bind(&qp, &ap, scratch, s);
        if (rc) return rc;
        bq = Q; ba = A; bs = scratch;
        return 0;
    }
    int begin(const void* Q, const void* A, char* scratch, cudaStream_t s) override {
        int rc = ensure_bound(Q, A, scratch, s);
        return rc ? rc : core.begin(s);
    }
    int evolve(void* Q, void* A, char* scratch, int n, cudaStream_t s) override {
        int rc = ensure_bound(Q, A, scratch, s);
        return rc ? rc : core.evolve(n, s);
    }
    int total_mass(const void* Q, char* scratch, cudaStream_t s) override {
        int rc = ensure_bound(Q, ba, scratch, s);
        return rc ? rc : core.mass(s);
    }
    int state_import(const double* Q64, void* Q, char* scratch, cudaStream_t s) override {
        int rc = ensure_bound(Q, ba, scratch, s);
        return rc ? rc : core.convert(&Q64, false, s);
    }
    int state_export(const void* Q, const char* scratch, double* Q64, cudaStream_t s) override {
        int rc = ensure_bound(Q, ba, const_cast<char*>(scratch), s);
        const double* q = Q64;
        return rc ? rc : core.convert(&q, true, s);
    }
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
    int set_variant(int v, cudaStream_t s) override { return core.set_variant(v, s); }
    int variant() const override { return core.variant; }
};

}  // namespace zfv32

namespace zfvi {
Runner* make_runner_fp32_swe2d(zfv_handle* h) { return new zfv32::Runner32(h); }
}

// ---------------------------------------------------------------------------
// Batch C ABI (include/zoomy_fv.h).
struct zfv_batch {
    zfv32::BatchCore core;
};

extern "C" {

int zfv_tile_variants(int* nw, int* cpt, int* cols, int* flags, int max_n) {
    for (int v = 0; v < zfv32::kNumVariants && v < max_n; ++v) {
        if (nw) nw[v] = zfv32::kVarNW[v];
        if (cpt) cpt[v] = zfv32::kVarCPT[v];
        if (cols) cols[v] = zfv32::kVarPK[v];
        if (flags) flags[v] = zfv32::kVarPF[v];
    }
    return zfv32::kNumVariants;
}

int zfv_batch_create(const zfv_config* cfgs, int n_inst, zfv_batch** out) {
    if (!cfgs || !out) return fail(-1, "zfv_batch_create: null argument");
    *out = nullptr;
    zfv_batch* b = new (std::nothrow) zfv_batch();
    if (!b) return fail(-4, "zfv_batch_create: out of host memory");
    const int rc = b->core.init(cfgs, n_inst);
    if (rc) { delete b; return rc; }
    *out = b;
    return 0;
}

int zfv_batch_create_grouped(const zfv_config* cfgs, int n_inst, const int* groups, zfv_batch** out) {
    if (!cfgs || !out || !groups) return fail(-1, "zfv_batch_create_grouped: null argument");
    *out = nullptr;
    zfv_batch* b = new (std::nothrow) zfv_batch();
    if (!b) return fail(-4, "zfv_batch_create_grouped: out of host memory");
    for (int k = 1; k < n_inst; ++k) {
        const zfv_config &a = cfgs[k], &f = cfgs[0];
        if (a.cfl != f.cfl || a.cfl_dimension != f.cfl_dimension || a.cfl_degree_factor != f.cfl_degree_factor) {
            delete b;
            return fail(-1, "zfv_batch_create_grouped: instances must share the CFL constants");
        }
    }
    const int rc = b->core.init(cfgs, n_inst, groups);
    if (rc) { delete b; return rc; }
    *out = b;
    return 0;
}

int zfv_batch_set_frames(zfv_batch* b, const float* const* frames, void* stream) {
    if (!b) return fail(-1, "zfv_batch_set_frames: null batch");
    return b->core.set_frames(frames, (cudaStream_t)stream);
}

int zfv_batch_compute_dt(zfv_batch* b, void* stream) {
    if (!b || !b->core.bound) return fail(-1, "zfv_batch_compute_dt: bind the batch first");
    return b->core.compute_dt((cudaStream_t)stream);
}

int zfv_batch_set_dt(zfv_batch* b, const double* dts, void* stream) {
    if (!b || !dts || !b->core.bound) return fail(-1, "zfv_batch_set_dt: bind the batch first");
    return b->core.set_dt(dts, (cudaStream_t)stream);
}

int zfv_batch_stage(zfv_batch* b, int stage, void* stream) {
    if (!b || !b->core.bound) return fail(-1, "zfv_batch_stage: bind the batch first");
    if (stage != 1 && stage != 2) return fail(-1, "zfv_batch_stage: stage must be 1 or 2");
    return b->core.evolve(1, (cudaStream_t)stream, stage);
}

const void* zfv_batch_descriptors(const zfv_batch* b) {
    return (b && b->core.bound) ? static_cast<const void*>(b->core.d_desc()) : nullptr;
}

int zfv_batch_destroy(zfv_batch* b) { delete b; return 0; }

// ---- AMR (include/zoomy_fv.h) ----------------------------------------------
static_assert(sizeof(zfv_amr_level) == sizeof(zfv32::amr::LevelView), "zfv_amr_level layout");

static zfv32::amr::LevelView view_of(const zfv_amr_level* l) {
    zfv32::amr::LevelView v{};
    if (l) std::memcpy(&v, l, sizeof v);
    return v;
}

static int amr_grid(int n_patches, int max_blocks, long long per_patch, dim3& g) {
    if (n_patches < 1 || n_patches > 65535)
        return fail(-1, "zfv_amr: %d patches (1 .. 65535 per call)", n_patches);
    constexpr int kMax = zfv32::amr::kMaxPatchSide * zfv32::amr::kMaxPatchSide;
    if (max_blocks < 1 || max_blocks > kMax)
        return fail(-1, "zfv_amr: %d blocks per patch (1 .. %d)", max_blocks, kMax);
    g = dim3(unsigned((per_patch + 255) / 256), unsigned(n_patches), 1);
    return 0;
}

int zfv_amr_fill(const zfv_amr_level* fine, const zfv_amr_level* coarse, const int* patches, float* const* frames,
                 int n_patches, int max_blocks, int stage, void* stream) {
    if (!fine || !patches || !frames) return fail(-1, "zfv_amr_fill: null argument");
    if (stage != 1 && stage != 2) return fail(-1, "zfv_amr_fill: stage must be 1 or 2");
    // a patch of nbx x nby <= max_blocks blocks has a ring of 2 (W + H) + 16 <= 2 B (max_blocks + 1) + 16 cells per layer
    const long long B = fine->B;
    dim3 g;
    int rc = amr_grid(n_patches, max_blocks, 4 * B * (max_blocks + 1) + 16, g);
    if (rc) return rc;
    zfv32::amr::k32a_fill<<<g, 256, 0, (cudaStream_t)stream>>>(
        view_of(fine), view_of(coarse), reinterpret_cast<const int4*>(patches), frames, n_patches, stage);
    return cuda_check(cudaGetLastError(), "zfv_amr_fill launch");
}

int zfv_amr_average_down(const zfv_amr_level* fine, const zfv_amr_level* coarse, const int* patches, int n_patches,
                         int max_blocks, void* stream) {
    if (!fine || !coarse || !patches) return fail(-1, "zfv_amr_average_down: null argument");
    if (fine->B % 2) return fail(-1, "zfv_amr_average_down: the block side must be even");
    const long long h = fine->B / 2;
    dim3 g;
    int rc = amr_grid(n_patches, max_blocks, (long long)max_blocks * h * h, g);
    if (rc) return rc;
    zfv32::amr::k32a_average_down<<<g, 256, 0, (cudaStream_t)stream>>>(
        view_of(fine), view_of(coarse), reinterpret_cast<const int4*>(patches), n_patches);
    return cuda_check(cudaGetLastError(), "zfv_amr_average_down launch");
}

int zfv_amr_tag(const zfv_amr_level* level, const int* patches, int n_patches, int max_blocks, double dx, double dy,
                double threshold, int criterion, double b_max, int* flags, void* stream) {
    if (!level || !patches || !flags) return fail(-1, "zfv_amr_tag: null argument");
    if (criterion != 0 && criterion != 1) return fail(-1, "zfv_amr_tag: criterion must be 0 or 1");
    dim3 g;
    const long long B = level->B;
    int rc = amr_grid(n_patches, max_blocks, (long long)max_blocks * B * B, g);
    if (rc) return rc;
    zfv32::amr::k32a_tag<<<g, 256, 0, (cudaStream_t)stream>>>(view_of(level), reinterpret_cast<const int4*>(patches),
                                                            n_patches, float(dx), float(dy), float(threshold),
                                                            criterion, float(fmin(b_max, 3.0e38)), flags);
    return cuda_check(cudaGetLastError(), "zfv_amr_tag launch");
}

int zfv_amr_set_dt(const void* const* level_descs, double* const* dts, const int* n_inst, int n_levels,
                   double cfl, double cfl_divisor, double dtmin, double dtmax, double time_end, double* time,
                   void* stream) {
    if (!level_descs || !dts || !n_inst) return fail(-1, "zfv_amr_set_dt: null argument");
    if (n_levels < 1 || n_levels > zfv32::amr::kMaxLevels)
        return fail(-1, "zfv_amr_set_dt: %d levels (1 .. %d)", n_levels, zfv32::amr::kMaxLevels);
    zfv32::amr::DtArgs a{};
    for (int l = 0; l < n_levels; ++l) {
        a.lev[l] = static_cast<const zfv32::BInst*>(level_descs[l]);
        a.dts[l] = dts[l];
        a.n_inst[l] = n_inst[l];
    }
    a.n_levels = n_levels;
    a.cfl = cfl; a.div = cfl_divisor; a.dtmin = dtmin; a.dtmax = dtmax; a.time_end = time_end;
    a.time = time;
    zfv32::amr::k32a_set_dt<<<1, 256, 0, (cudaStream_t)stream>>>(a);
    return cuda_check(cudaGetLastError(), "zfv_amr_set_dt launch");
}

int zfv_amr_level_dt(const void* level_desc, double time_end, double* time, void* stream) {
    if (!level_desc || !time) return fail(-1, "zfv_amr_level_dt: null argument");
    zfv32::amr::k32a_level_dt<<<1, 1, 0, (cudaStream_t)stream>>>(static_cast<const zfv32::BInst*>(level_desc),
                                                                  time_end, time);
    return cuda_check(cudaGetLastError(), "zfv_amr_level_dt launch");
}

int zfv_amr_regrid_fill(const zfv_amr_level* level, const zfv_amr_level* old_level, const zfv_amr_level* coarse,
                        const int* patches, int n_patches, int max_blocks, void* stream) {
    if (!level || !patches) return fail(-1, "zfv_amr_regrid_fill: null argument");
    if (!old_level && !coarse) return fail(-1, "zfv_amr_regrid_fill: needs an old level or a coarser level");
    dim3 g;
    const long long B = level->B;
    int rc = amr_grid(n_patches, max_blocks, (long long)max_blocks * B * B, g);
    if (rc) return rc;
    zfv32::amr::k32a_regrid_fill<<<g, 256, 0, (cudaStream_t)stream>>>(
        view_of(level), view_of(old_level), view_of(coarse), reinterpret_cast<const int4*>(patches), n_patches);
    return cuda_check(cudaGetLastError(), "zfv_amr_regrid_fill launch");
}

size_t zfv_batch_scratch_bytes(const zfv_batch* b) { return b ? b->core.total : 0; }

int zfv_batch_bind(zfv_batch* b, void* const* Q, double* const* aux, void* scratch, void* stream) {
    if (!b || !Q || !aux || !scratch) return fail(-1, "zfv_batch_bind: null argument");
    return b->core.bind(Q, aux, static_cast<char*>(scratch), (cudaStream_t)stream);
}

int zfv_batch_import(zfv_batch* b, const double* const* Q64, void* stream) {
    if (!b || !Q64 || !b->core.bound) return fail(-1, "zfv_batch_import: bind the batch first");
    return b->core.convert(Q64, false, (cudaStream_t)stream);
}

int zfv_batch_export(zfv_batch* b, double* const* Q64, void* stream) {
    if (!b || !Q64 || !b->core.bound) return fail(-1, "zfv_batch_export: bind the batch first");
    return b->core.convert(const_cast<const double* const*>(Q64), true, (cudaStream_t)stream);
}

int zfv_batch_begin(zfv_batch* b, void* stream) {
    if (!b || !b->core.bound) return fail(-1, "zfv_batch_begin: bind the batch first");
    return b->core.begin((cudaStream_t)stream);
}

int zfv_batch_evolve(zfv_batch* b, int n_steps, void* stream) {
    if (!b || !b->core.bound) return fail(-1, "zfv_batch_evolve: bind the batch first");
    if (n_steps < 0) return fail(-1, "zfv_batch_evolve: negative step count");
    return b->core.evolve(n_steps, (cudaStream_t)stream);
}

int zfv_batch_status(zfv_batch* b, zfv_status* out, void* stream) {
    if (!b || !out || !b->core.bound) return fail(-1, "zfv_batch_status: bind the batch first");
    return b->core.status(out, (cudaStream_t)stream);
}

int zfv_batch_set_variant(zfv_batch* b, int variant, void* stream) {
    if (!b) return fail(-1, "zfv_batch_set_variant: null batch");
    return b->core.set_variant(variant, (cudaStream_t)stream);
}

int zfv_batch_units(const zfv_batch* b) { return b ? b->core.nunits() : 0; }

}  // extern "C"
