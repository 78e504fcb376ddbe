// Block-structured AMR on top of the FP32 batch engine.
//
// Each level lives on a regular grid of B x B blocks. The blocks present at a
// level are grouped into patches: rectangles of nbx x nby blocks, each patch
// one batch instance of (nbx * B) x (nby * B) cells (wide patches keep the
// 30- and 60-column strips of the stage kernels full; tall ones let most
// strips take the interior path). `map` gives, per block position,
// (instance << 10) | (block row offset << 5) | (block column offset) inside
// the patch, or -1 when the level has no such block. All patches of a level
// share one run record (one dt, one CFL reduction). Refinement ratio 2: a
// level-(l+1) block covers a quarter of a level-l block.
//
// Kernels (the reference's AmrCore pieces, ZoomyAmr.cpp:161-288, 733-762):
//   k32a_fill          ghost frames of every patch of a level before a stage:
//                      same-level neighbour (FillBoundary), else conservative
//                      linear interpolation of the next coarser level
//                      (FillPatchTwoLevels with cell_cons_interp), and the
//                      physical boundary by mirroring (FillPhysicalBC_mf);
//   k32a_average_down  fine -> coarse averages under each fine patch;
//   k32a_tag           per block: any cell with |grad eta| > threshold (ErrorEst);
//   k32a_regrid_fill   fill new patches from the old patches of the same
//                      level where they overlap, else from the coarser level
//                      (RemakeLevel / MakeNewLevelFromCoarse).
// The coarse data used for a fine patch's ghosts is the coarse level's
// current state (the reference fills from Q[lev-1] at t_new only).
// Patch descriptors: int4 {first block x, first block row y, nbx, nby}.
#pragma once

namespace zfv32 {
namespace amr {

struct LevelView {
    const BInst* insts;   // the level's batch descriptors (device)
    const int* map;       // [nby * nbx] block position -> (instance << 10) | (oy << 5) | ox, -1 absent
    int nbx, nby;         // block grid
    int B;                // cells per block side
    int nx, ny;           // level grid (cells)
    int wall;             // bit s: side s (x_lo, x_hi, y_lo, y_hi) is a reflective wall
    int pad_;
};

constexpr int kMaxPatchSide = 32;      // blocks per patch side: the offset fields of a map entry

// Instance and in-instance cell index of level cell (I, J) inside the
// domain; false when no patch of the level holds it.
__device__ __forceinline__ bool locate(const LevelView& V, int I, int J, int& k, long long& c) {
    const int bx = I / V.B, by = J / V.B;
    const int code = V.map[by * V.nbx + bx];
    if (code < 0) return false;
    k = code >> 10;
    const int ox = code & (kMaxPatchSide - 1), oy = (code >> 5) & (kMaxPatchSide - 1);
    c = (long long)(J - (by - oy) * V.B) * V.insts[k].P.nx + (I - (bx - ox) * V.B);
    return true;
}

// The stage input of level cell (I, J): mirrored into the domain with the
// wall sign flips; false when no patch of the level holds the cell.
__device__ __forceinline__ bool lookup(const LevelView& V, int I, int J, bool with_inc, C4& out) {
    bool fu = false, fv = false;
    if (I < 0) { I = -1 - I; fu = (V.wall & 1) != 0; }
    else if (I >= V.nx) { I = 2 * V.nx - 1 - I; fu = (V.wall & 2) != 0; }
    if (J < 0) { J = -1 - J; fv = (V.wall & 4) != 0; }
    else if (J >= V.ny) { J = 2 * V.ny - 1 - J; fv = (V.wall & 8) != 0; }
    if (I < 0 || I >= V.nx || J < 0 || J >= V.ny) return false;
    int k;
    long long c;
    if (!locate(V, I, J, k, c)) return false;
    const BInst& D = V.insts[k];
    const unsigned parity = *(volatile const unsigned*)&D.st->parity;
    const float* X = parity ? D.alt : D.Qs;
    const long long pl = D.P.plane;
    out.b = D.bed[c];
    out.e = X[c];
    out.u = X[pl + c];
    out.v = X[2 * pl + c];
    if (with_inc) {
        out.e += D.inc[c];
        out.u += D.inc[pl + c];
        out.v += D.inc[2 * pl + c];
    }
    if (fu) out.u = -out.u;
    if (fv) out.v = -out.v;
    return true;
}

// Conservative linear interpolation of level-(l-1) data at level-l cell
// (I, J) (inside the domain): minmod-limited slopes, so a constant field (a
// lake at rest's eta) interpolates exactly and the 2 x 2 average of the fine
// values is the coarse value.
__device__ __forceinline__ C4 coarse_interp(const LevelView& C, int I, int J) {
    const int ic = I >> 1, jc = J >> 1;
    C4 c0{0.0f, 0.0f, 0.0f, 0.0f};
    if (!lookup(C, ic, jc, false, c0)) return c0;
    C4 xm = c0, xp = c0, ym = c0, yp = c0;
    lookup(C, ic - 1, jc, false, xm);
    lookup(C, ic + 1, jc, false, xp);
    lookup(C, ic, jc - 1, false, ym);
    lookup(C, ic, jc + 1, false, yp);
    const float ox = (I & 1) ? 0.25f : -0.25f, oy = (J & 1) ? 0.25f : -0.25f;
    C4 r;
    r.b = c0.b + ox * mm(c0.b - xm.b, xp.b - c0.b) + oy * mm(c0.b - ym.b, yp.b - c0.b);
    r.e = c0.e + ox * mm(c0.e - xm.e, xp.e - c0.e) + oy * mm(c0.e - ym.e, yp.e - c0.e);
    r.u = c0.u + ox * mm(c0.u - xm.u, xp.u - c0.u) + oy * mm(c0.u - ym.u, yp.u - c0.u);
    r.v = c0.v + ox * mm(c0.v - xm.v, xp.v - c0.v) + oy * mm(c0.v - ym.v, yp.v - c0.v);
    return r;
}

// Ring cells of a (W+4) x (H+4) frame, enumerated: bottom two rows, top two
// rows, then the two left and two right columns of the patch rows.
__device__ __forceinline__ void ring_cell(int k, int W, int H, int& fi, int& fj) {
    const int FW = W + 4;
    if (k < 2 * FW) { fj = k / FW; fi = k % FW; return; }
    k -= 2 * FW;
    if (k < 2 * FW) { fj = H + 2 + k / FW; fi = k % FW; return; }
    k -= 2 * FW;
    fj = 2 + k / 4;
    const int col = k % 4;
    fi = col < 2 ? col : W + col;
}

// Ghost frames of all patches of level F (coarse level C; C.insts == nullptr
// for level 0). stage 1 fills the stage input Q; stage 2 fills Q + inc1 for
// same-level neighbours (their stage-2 input) and the coarse state otherwise.
__global__ void k32a_fill(LevelView F, LevelView C, const int4* __restrict__ patches, float* const* __restrict__ frames,
                          int n_patches, int stage) {
    const int pi = blockIdx.y;
    if (pi >= n_patches) return;
    const int4 p = patches[pi];
    const int H = p.w * F.B, W = p.z * F.B, FW = W + 4;
    const int ring = FW * (H + 4) - W * H;
    const long long fp = (long long)FW * (H + 4);
    float* fr = frames[pi];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < ring; k += gridDim.x * blockDim.x) {
        int fi, fj;
        ring_cell(k, W, H, fi, fj);
        const int I = p.x * F.B + fi - 2, J = p.y * F.B + fj - 2;
        C4 q{0.0f, 0.0f, 0.0f, 0.0f};
        const bool inside = I >= 0 && I < F.nx && J >= 0 && J < F.ny;
        bool ok = lookup(F, I, J, stage == 2, q);
        if (!ok && inside && C.insts) q = coarse_interp(C, I, J);
        const long long f = (long long)fj * FW + fi;
        fr[f] = q.b; fr[fp + f] = q.e; fr[2 * fp + f] = q.u; fr[3 * fp + f] = q.v;
    }
}

// Fine -> coarse: each 2 x 2 group of fine cells of a fine patch replaces
// the coarse cell under it (eta, hu, hv as the FP64 mean of value +
// remainder; the coarse bed is kept).
__global__ void k32a_average_down(LevelView F, LevelView C, const int4* __restrict__ patches, int n_patches) {
    const int pi = blockIdx.y;
    if (pi >= n_patches) return;
    const int4 p = patches[pi];
    const int hb = F.B / 2, hw = p.z * hb, hh = p.w * hb;
    const int code = F.map[p.y * F.nbx + p.x];
    if (code < 0) return;
    const BInst& D = F.insts[code >> 10];
    const float* X = (*(volatile const unsigned*)&D.st->parity) ? D.alt : D.Qs;
    const long long pl = D.P.plane;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < hw * hh; k += gridDim.x * blockDim.x) {
        const int a = k % hw, c = k / hw;
        const int ic = p.x * hb + a, jc = p.y * hb + c;   // coarse cell
        int kc;
        long long cc;
        if (!locate(C, ic, jc, kc, cc)) continue;
        double s[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            const long long cf = (long long)(2 * c + (d >> 1)) * D.P.nx + (2 * a + (d & 1));
#pragma unroll
            for (int q = 0; q < 3; ++q) s[q] += double(X[q * pl + cf]) + double(D.lo[q * pl + cf]);
        }
        const BInst& E = C.insts[kc];
        float* Y = (*(volatile const unsigned*)&E.st->parity) ? E.alt : E.Qs;
        const long long plc = E.P.plane;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const double m = 0.25 * s[q];
            const float hi = float(m);
            Y[q * plc + cc] = hi;
            E.lo[q * plc + cc] = float(m - double(hi));
        }
    }
}

// flags[by * nbx + bx] = 1 (others untouched) for blocks with a tagged cell.
// criterion 0: |grad eta| > threshold (centred differences per unit length);
// criterion 1: the reference's ErrorEst (ZoomyAmr.cpp:224-252): cells with
// b < b_max whose undivided |(h(i+1) - h(i-1), h(j+1) - h(j-1))| exceeds the
// threshold, or with h > 1e-2.
__global__ void k32a_tag(LevelView V, const int4* __restrict__ patches, int n_patches, float dx, float dy,
                         float threshold, int criterion, float b_max, int* __restrict__ flags) {
    const int pi = blockIdx.y;
    if (pi >= n_patches) return;
    const int B = V.B;
    const int4 p = patches[pi];
    const int W = p.z * B, H = p.w * B;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < W * H; k += gridDim.x * blockDim.x) {
        const int i = k % W, j = k / W;
        const int I = p.x * B + i, J = p.y * B + j;
        C4 xm, xp, ym, yp;
        if (!lookup(V, I - 1, J, false, xm) || !lookup(V, I + 1, J, false, xp) ||
            !lookup(V, I, J - 1, false, ym) || !lookup(V, I, J + 1, false, yp))
            continue;
        bool hit;
        if (criterion == 0) {
            const float gx = (xp.e - xm.e) / (2.0f * dx), gy = (yp.e - ym.e) / (2.0f * dy);
            hit = gx * gx + gy * gy > threshold * threshold;
        } else {
            C4 c;
            lookup(V, I, J, false, c);
            if (c.b >= b_max) continue;
            const float hx = (xp.e - xp.b) - (xm.e - xm.b), hy = (yp.e - yp.b) - (ym.e - ym.b);
            hit = sqrtf(hx * hx + hy * hy) > threshold || (c.e - c.b) > 1.0e-2f;
        }
        if (hit) flags[(p.y + j / B) * V.nbx + p.x + i / B] = 1;
    }
}

// New patches of a level: copy the old patches of the same level where
// present (value + remainder), else interpolate the coarser level
// (remainder 0). New patches start with parity 0 (their run record is fresh).
__global__ void k32a_regrid_fill(LevelView N, LevelView O, LevelView C, const int4* __restrict__ patches,
                                 int n_patches) {
    const int pi = blockIdx.y;
    if (pi >= n_patches) return;
    const int B = N.B;
    const int4 p = patches[pi];
    const int W = p.z * B, H = p.w * B;
    const int code = N.map[p.y * N.nbx + p.x];
    if (code < 0) return;
    const BInst& D = N.insts[code >> 10];
    const long long pl = D.P.plane;
    float* bed = const_cast<float*>(D.bed);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < W * H; k += gridDim.x * blockDim.x) {
        const int i = k % W, j = k / W;
        const int I = p.x * B + i, J = p.y * B + j;
        const long long c = (long long)j * D.P.nx + i;
        int ko;
        long long co;
        if (O.insts && locate(O, I, J, ko, co)) {
            const BInst& E = O.insts[ko];
            const float* X = (*(volatile const unsigned*)&E.st->parity) ? E.alt : E.Qs;
            const long long plo = E.P.plane;
            bed[c] = E.bed[co];
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                D.Qs[q * pl + c] = X[q * plo + co];
                D.lo[q * pl + c] = E.lo[q * plo + co];
            }
        } else {
            const C4 q = coarse_interp(C, I, J);
            bed[c] = q.b;
            D.Qs[c] = q.e; D.Qs[pl + c] = q.u; D.Qs[2 * pl + c] = q.v;
            D.lo[c] = 0.0f; D.lo[pl + c] = 0.0f; D.lo[2 * pl + c] = 0.0f;
        }
    }
}

// dt_0 of the hierarchy from every level's last CFL maximum (the largest
// step whose dt_0 / 2^l every level's CFL law allows, ZoomyAmr.cpp:448-515),
// written as dt_0 / 2^l into each level's per-instance dt array, and the
// hierarchy time advanced by dt_0 (dt_0 clamped to land on time_end; zero
// once time_end is reached). One block; no host round trip, so a coarse step
// can be replayed from a CUDA graph.
constexpr int kMaxLevels = 8;
struct DtArgs {
    const BInst* lev[kMaxLevels];
    double* dts[kMaxLevels];
    int n_inst[kMaxLevels];
    int n_levels;
    double cfl, div, dtmin, dtmax, time_end;
    double* time;
};

__global__ void k32a_set_dt(DtArgs a) {
    __shared__ double s_dt0;
    if (threadIdx.x == 0) {
        double dt0 = a.dtmax;
        for (int l = 0; l < a.n_levels; ++l) {
            const double m = *(volatile const double*)&a.lev[l][0].st->max_inv;
            if (m > 1e-14) dt0 = fmin(dt0, double(1 << l) * (a.cfl / (a.div * m)));
        }
        dt0 = fmax(dt0, a.dtmin);
        if (a.time) {
            // land on time_end (ZoomyAmr.cpp:746-749); past it, steps are no-ops
            const double remaining = a.time_end - *a.time;
            dt0 = remaining > 0.0 ? fmin(dt0, remaining) : 0.0;
            *a.time += dt0;
        }
        s_dt0 = dt0;
    }
    __syncthreads();
    for (int l = 0; l < a.n_levels; ++l) {
        const double dl = s_dt0 / double(1 << l);
        for (int k = threadIdx.x; k < a.n_inst[l]; k += blockDim.x) a.dts[l][k] = dl;
    }
}

// The reference's per-level step law (ZoomyAmr.cpp:739-749) for the base
// level: its run record's dt (ComputeDt of its current state) clamped to land
// on time_end (0 once time_end is reached), and the hierarchy time advanced
// by it. One thread.
__global__ void k32a_level_dt(const BInst* __restrict__ lev, double time_end, double* time) {
    zfv::DevState* st = lev[0].st;
    const double remaining = time_end - *time;
    double dt = *(volatile double*)&st->dt;
    dt = remaining > 0.0 ? fmin(dt, remaining) : 0.0;
    st->dt = dt;
    *time += dt;
}

}  // namespace amr
}  // namespace zfv32
