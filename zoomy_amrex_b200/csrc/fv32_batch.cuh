// FP32 chosen form: one launch per stage over a work list of strips drawn
// from any number of independent levels ("instances": the boxes of an AMR
// level or the members of an ensemble, each with its own size, bathymetry,
// parameters, boundary conditions, dt, time and stop test).
//
// A block takes work unit `blockIdx.x` = (instance, strip) from the unit
// table, stages its instance's descriptor in shared memory and runs a warp
// column sweep on the strip: one column per lane (fv32_sweep.cuh, strips 30
// columns wide, PK = 1) or a column pair per lane in packed FP32
// (fv32_sweep2.cuh, 60 columns, PK = 2). The CFL max / mass of an
// instance are reduced over that instance's units only: the last of its units
// to finish advances its run record. A single level is a batch of one.
//
// The state of an instance ping-pongs between Q rows 1..3 and `alt`; which
// of the two holds it is the instance's device-side `parity`, flipped by the
// block that finishes a step. A step is therefore the same two launches
// whatever came before, so one captured CUDA graph of one step can be replayed
// any number of times; an instance that has stopped is left untouched.
#pragma once
#include "fv32_sweep.cuh"
#include "fv32_sweep2.cuh"

namespace zfv32 {

// Device descriptor of one instance.
struct BInst {
    Params P;
    const float* bed;      // Q row 0 (FP32 bed)
    float* Qs;             // Q rows 1..3 (eta, hu, hv): state buffer 0
    float* alt;            // state buffer 1 (3 planes)
    float* inc;            // 3 planes: stage-1 increment
    float* lo;             // 3 planes: compensation remainders
    double* aux;           // n_aux FP64 planes
    const double* q64;    // FP64 reference-layout state (import / export only)
    zfv::DevState* st;
    double* partials;      // 2 doubles per unit
    double* log3;
    int log_cap;
    int nbx, nby;          // units in x / y for the current strip shape
    int unit_base;         // index of this instance's first unit within its run-record group
    int group_units;       // units of the whole group (the CFL / mass reduction runs over them)
    int pad_;
};

// Copy the instance descriptor into shared memory (one per block).
__device__ __forceinline__ void stage_desc(const BInst* __restrict__ insts, int k, BInst& sD) {
    constexpr int nw = int(sizeof(BInst) / sizeof(int));
    static_assert(sizeof(BInst) % sizeof(int) == 0, "BInst is word-sized");
    const int* src = reinterpret_cast<const int*>(insts + k);
    int* dst = reinterpret_cast<int*>(&sD);
    for (int t = threadIdx.x; t < nw; t += blockDim.x) dst[t] = __ldg(src + t);
    __syncthreads();
}

// The buffer holding instance D's state, and the other one.
__device__ __forceinline__ const float* state_in(const BInst& D, unsigned parity) {
    return parity ? D.alt : D.Qs;
}

template <int MODE, bool WB, bool IMPL, int NW, int CPT, int PK, int PF>
__device__ __forceinline__ void stage_body(const BInst* __restrict__ insts, const int2* __restrict__ units)
{
    constexpr int SW = 30 * PK;                  // owned columns per strip
    constexpr int NT = 32 * NW;
    __shared__ double red[2 * NW];
    __shared__ BInst sD;
    // stage-2 staging of the update's own inputs (PF bit 0): 9 values per lane per warp
    __shared__ __align__(16) float cstage[(PF & 1) ? NW * 9 * 32 * PK : 1];
    const int2 u = units[blockIdx.x];
    stage_desc(insts, u.x, sD);
    const Params& L = sD.P;
    const int w = threadIdx.x >> 5;
    float* wstage = cstage + ((PF & 1) ? w * 9 * 32 * PK : 0);
    const int bx = u.y % sD.nbx, by = u.y / sD.nbx;
    const int x0 = bx * SW, y0 = by * (NW * CPT), j0 = y0 + w * CPT;
    zfv::DevState* st = sD.st;
    if (*(volatile unsigned*)&st->flags & zfv::kFlagDone) return;   // stopped: state stays put
    const unsigned parity = *(volatile unsigned*)&st->parity;
    const float* X = parity ? sD.alt : sD.Qs;
    float* Y = parity ? sD.Qs : sD.alt;
    const double dtd = *(volatile double*)&st->dt;
    const double time = *(volatile double*)&st->time;
    double m_loc = 0.0, s_loc = 0.0;
    const float* inc_in = (MODE == S2) ? sD.inc : nullptr;   // stage 2 reads inc1
    float* inc_out = (MODE == S1) ? sD.inc : nullptr;        // stage 1 writes it
    if constexpr (PK == 1) {
        if (strip_interior<NW, CPT>(L, x0, y0))
            sweep_strip<MODE, WB, IMPL, CPT, true, (PF & 1) != 0>(sD.bed, X, inc_in, inc_out, Y, sD.lo, L, x0, j0,
                                                   float(dtd), dtd, m_loc, s_loc, wstage);
        else
            sweep_strip<MODE, WB, IMPL, CPT, false, (PF & 1) != 0>(sD.bed, X, inc_in, inc_out, Y, sD.lo, L, x0, j0,
                                                    float(dtd), dtd, m_loc, s_loc, wstage);
    } else {
        // 8-byte accesses need an even row length (x0 is even)
        if (pk::strip_interior2<NW, CPT>(L, x0, y0)) {
            if ((L.nx & 1) == 0)
                pk::sweep_strip2<MODE, WB, IMPL, CPT, true, true, (PF & 1) != 0>(sD.bed, X, inc_in, inc_out, Y, sD.lo, L, x0,
                                                                  j0, float(dtd), dtd, m_loc, s_loc,
                                                                reinterpret_cast<float2*>(wstage));
            else
                pk::sweep_strip2<MODE, WB, IMPL, CPT, true, false, (PF & 1) != 0>(sD.bed, X, inc_in, inc_out, Y, sD.lo, L, x0,
                                                                   j0, float(dtd), dtd, m_loc, s_loc,
                                                                reinterpret_cast<float2*>(wstage));
        } else {
            pk::sweep_strip2<MODE, WB, IMPL, CPT, false, false, (PF & 1) != 0>(sD.bed, X, inc_in, inc_out, Y, sD.lo, L, x0,
                                                                j0, float(dtd), dtd, m_loc, s_loc,
                                                                reinterpret_cast<float2*>(wstage));
        }
    }
    if constexpr (MODE == S2) {
        const bool last = zfv::finish_step_units<NT>(m_loc, s_loc, red, sD.partials, sD.log3, sD.log_cap,
                                                      st, L, dtd, time, false, unsigned(sD.group_units),
                                                      unsigned(sD.unit_base + u.y));
        if (last && threadIdx.x == 0) {   // every unit of the step has read parity by now
            st->parity = parity ^ 1u;
            __threadfence();
        }
    }
}

// One RK stage of every unit of the batch.
template <int MODE, bool WB, bool IMPL, int NW, int CPT, int PK, int PF>
__global__ void __launch_bounds__(32 * NW)
k32b_stage(const BInst* __restrict__ insts, const int2* __restrict__ units) {
    stage_body<MODE, WB, IMPL, NW, CPT, PK, PF>(insts, units);
}

// The same, held to 128 registers so that 4 blocks of 128 threads fit an SM
// (the stage-2 kernel of the shapes with PF bit 1).
template <int MODE, bool WB, bool IMPL, int NW, int CPT, int PK, int PF>
__global__ void __launch_bounds__(32 * NW, 4)
k32b_stage_r128(const BInst* __restrict__ insts, const int2* __restrict__ units) {
    stage_body<MODE, WB, IMPL, NW, CPT, PK, PF>(insts, units);
}

template <int MODE, bool WB, bool IMPL, int NW, int CPT, int PK, int PF>
inline void launch_stage(int n_units, cudaStream_t s, const BInst* insts, const int2* units) {
    if constexpr (MODE == S2 && (PF & 2) != 0)
        k32b_stage_r128<MODE, WB, IMPL, NW, CPT, PK, PF><<<n_units, 32 * NW, 0, s>>>(insts, units);
    else
        k32b_stage<MODE, WB, IMPL, NW, CPT, PK, PF><<<n_units, 32 * NW, 0, s>>>(insts, units);
}

// Per-cell helpers over the same unit table: each block covers its strip's
// owned cells (30 PK x NW*CPT).
template <int NW, int CPT, int PK, class F>
__device__ __forceinline__ void for_strip_cells(const BInst& D, int2 u, F&& f) {
    constexpr int SW = 30 * PK;
    const int bx = u.y % D.nbx, by = u.y / D.nbx;
    const int x0 = bx * SW, y0 = by * (NW * CPT);
    for (int k = threadIdx.x; k < SW * NW * CPT; k += blockDim.x) {
        const int i = x0 + k % SW, j = y0 + k / SW;
        if (i < D.P.nx && j < D.P.ny) f((long long)j * D.P.nx + i);
    }
}

// FP64 reference layout [b, h, hu, hv] -> FP32 [b, eta, hu, hv] in Q plus
// FP32 remainders: eta = h + b is formed in FP64 and split, so a lake at rest
// imports as a constant eta. The state is left in Q (parity 0).
template <int NW, int CPT, int PK>
__global__ void k32b_import(const BInst* __restrict__ insts, const int2* __restrict__ units) {
    __shared__ BInst sD;
    const int2 u = units[blockIdx.x];
    stage_desc(insts, u.x, sD);
    if (sD.unit_base + u.y == 0 && threadIdx.x == 0) sD.st->parity = 0u;
    const long long pl = sD.P.plane;
    const double* Q64 = sD.q64;
    float* Qb = const_cast<float*>(sD.bed);
    for_strip_cells<NW, CPT, PK>(sD, u, [&](long long c) {
        const float b = float(Q64[c]);
        const double eta = Q64[pl + c] + Q64[c];
        const double hu = Q64[2 * pl + c], hv = Q64[3 * pl + c];
        const float e = float(eta), fu = float(hu), fv = float(hv);
        Qb[c] = b; sD.Qs[c] = e; sD.Qs[pl + c] = fu; sD.Qs[2 * pl + c] = fv;
        sD.lo[c] = float(eta - double(e));
        sD.lo[pl + c] = float(hu - double(fu));
        sD.lo[2 * pl + c] = float(hv - double(fv));
    });
}
// The state in the reference layout (FP64, depth measured from the FP32 bed),
// and the aux row hinv of that state (UpdateState's aux refresh; the carried
// aux rows are untouched).
template <int NW, int CPT, int PK>
__global__ void k32b_export(const BInst* __restrict__ insts, const int2* __restrict__ units, int n_aux) {
    __shared__ BInst sD;
    const int2 u = units[blockIdx.x];
    stage_desc(insts, u.x, sD);
    const long long pl = sD.P.plane;
    double* Q64 = const_cast<double*>(sD.q64);
    const float* X = state_in(sD, *(volatile unsigned*)&sD.st->parity);
    for_strip_cells<NW, CPT, PK>(sD, u, [&](long long c) {
        const double b = double(sD.bed[c]);
        const double eta = double(X[c]) + double(sD.lo[c]);
        const double h = eta - b;
        if (Q64) {
            Q64[c] = b;
            Q64[pl + c] = h;
            Q64[2 * pl + c] = double(X[pl + c]) + double(sD.lo[pl + c]);
            Q64[3 * pl + c] = double(X[2 * pl + c]) + double(sD.lo[2 * pl + c]);
        }
        if (sD.aux) sD.aux[(n_aux - 1) * pl + c] = kp_hinv_d(h, sD.P.epsd);
    });
}

// Start of a run for every instance: time 0, step 0, stop flag.
static __global__ void k32b_init(const BInst* __restrict__ insts, int n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    zfv::DevState* st = insts[k].st;
    const Params& L = insts[k].P;
    st->time = 0.0; st->dt = 0.0; st->mass = 0.0; st->max_inv = 0.0;
    st->step = 0; st->flags = zfv::run_done(0.0, 0, L) ? zfv::kFlagDone : 0u; st->mood_redos = 0;
    st->counter = 0u; st->troubled = 0u;
}

// ComputeDt (WHAT 0, clamped to time_end, from the stored aux as the
// reference's first ComputeDt; WHAT 2 the same with hinv taken from the
// current state) or the FP64 mass (WHAT 1), per instance.
template <int NW, int CPT, int PK, int WHAT>
__global__ void __launch_bounds__(32 * NW)
k32b_reduce(const BInst* __restrict__ insts, const int2* __restrict__ units, int n_aux) {
    constexpr int NT = 32 * NW;
    __shared__ double red[2 * NW];
    __shared__ unsigned s_last;
    __shared__ BInst sD;
    const int2 u = units[blockIdx.x];
    stage_desc(insts, u.x, sD);
    const Params& L = sD.P;
    const long long pl = L.plane;
    const float* X = state_in(sD, *(volatile unsigned*)&sD.st->parity);
    double m = 0.0, s = 0.0;
    for_strip_cells<NW, CPT, PK>(sD, u, [&](long long c) {
        const double b = double(sD.bed[c]);
        const double h = (double(X[c]) + double(sD.lo[c])) - b;
        if constexpr (WHAT != 1) {
            const double hinv = (WHAT == 0) ? sD.aux[(n_aux - 1) * pl + c] : kp_hinv_d(h, L.epsd);
            const double c0 = sqrt(L.gd * fmax(h, 0.0));
            const double hu = double(X[pl + c]) + double(sD.lo[pl + c]);
            const double hv = double(X[2 * pl + c]) + double(sD.lo[2 * pl + c]);
            const double ix = (fabs(hu * hinv) + c0) / L.dx, iy = (fabs(hv * hinv) + c0) / L.dy;
            if (ix > m) m = ix;
            if (iy > m) m = iy;
        } else {
            s = s + h;
        }
    });
    zfv::block_reduce_max_sum<NT>(m, s, red);
    const unsigned nblk = unsigned(sD.group_units);
    const unsigned blk = unsigned(sD.unit_base + u.y);
    zfv::DevState* st = sD.st;
    if (threadIdx.x == 0) {
        sD.partials[2 * blk] = m;
        sD.partials[2 * blk + 1] = s;
        __threadfence();
        s_last = (atomicAdd(&st->counter, 1u) == nblk - 1) ? 1u : 0u;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    double gm = 0.0, gs = 0.0;
#pragma unroll 8
    for (unsigned b = threadIdx.x; b < nblk; b += NT) {
        const double pm = __ldcg(&sD.partials[2 * b]), ps = __ldcg(&sD.partials[2 * b + 1]);
        if (pm > gm) gm = pm;
        gs = gs + ps;
    }
    zfv::block_reduce_max_sum<NT>(gm, gs, red);
    if (threadIdx.x == 0) {
        if constexpr (WHAT != 1) {
            const double dt = zfv::dt_from_max(gm, st->time, L);
            st->max_inv = gm;
            st->dt = dt;
            if (!isfinite(dt)) st->flags |= zfv::kFlagNonfiniteDt;
        } else {
            st->mass = gs * (L.dx * L.dy);
        }
        st->counter = 0u;
        __threadfence();
    }
}

// Host-chosen step size per instance (AMR levels step with dt_0 / 2^l).
static __global__ void k32b_set_dt(const BInst* __restrict__ insts, int n, const double* __restrict__ dt) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) insts[k].st->dt = dt[k];
}

// Gather every instance's 64-byte status record into one array.
static __global__ void k32b_status(const BInst* __restrict__ insts, int n, zfv::DevState* out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) out[k] = *insts[k].st;
}

}  // namespace zfv32
