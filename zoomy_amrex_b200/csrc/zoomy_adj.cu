// The adjoint of the FP64 2-D shallow-water step: tape layout and the launch
// sequence of the reverse of one recorded step (kernels in fv_adjoint.cuh).
// Compiled with FMA contraction on: the reverse is checked against finite
// differences and FP64 autograd, not bit for bit.
#include <atomic>
#include <cuda_runtime.h>
#include "zfv_internal.H"
#include "fv_adjoint.cuh"

namespace zfvi {

namespace {
constexpr int kCellNT = 256;
constexpr int kDtBlocks = 592;   // 4 x 148 SMs

// Tile shapes of the face-reverse kernel: (TX, TY, threads NT, minimum
// resident blocks per SM). The kernel is register-heavy (FP64 reverse of a
// whole face), so the shapes trade tile halo overhead, the share of threads
// busy in the face pass (a tile has NF = (TX+3) TY + TX (TY+3) faces, spread
// over NT threads) and occupancy. 32 x 8 with 256 threads and two blocks per
// SM runs 3 face rounds per cell (632 faces); 32 x 6 with 256 threads runs
// 2.67 (498 faces in two rounds); 32 x 13 with 512 threads 2.46 (967 faces)
// at one block per SM. Default: 32 x 13 x 512, the fastest measured at 1024^2
// (backward of 200 steps 179 ms against 187 for 32 x 8 x 256).
constexpr int kAdjVariants = 7;
std::atomic<int> g_adj_variant{6};

template <class F>
int with_adj_variant(int v, F&& f) {
    switch (v) {
    case 0: return f.template operator()<32, 8, 256, 1>();
    case 1: return f.template operator()<32, 4, 128, 3>();
    case 2: return f.template operator()<32, 8, 256, 2>();
    case 3: return f.template operator()<16, 8, 128, 3>();
    case 4: return f.template operator()<32, 6, 256, 2>();
    case 5: return f.template operator()<32, 10, 384, 1>();
    case 6: return f.template operator()<32, 13, 512, 1>();
    default: return fail(-1, "unknown adjoint tile variant %d", v);
    }
}
}

AdjLayout adj_layout(long long plane) {
    AdjLayout A;
    const size_t pb = size_t(plane) * sizeof(double);
    size_t o = 0;
    A.off_X = o;   o += align_up(4 * pb);
    A.off_Y1 = o;  o += align_up(4 * pb);
    A.off_qs1 = o; o += align_up(3 * pb);
    A.off_qs2 = o; o += align_up(3 * pb);
    A.off_meta = o; o += align_up(2 * sizeof(double));
    A.step_bytes = o;
    A.nbA = int((plane + kCellNT - 1) / kCellNT);
    A.nbD = kDtBlocks;
    o = 0;
    A.w_lamq = o;    o += align_up(4 * pb);
    A.w_loc = o;     o += align_up(pb);
    A.w_lamY1 = o;   o += align_up(4 * pb);
    A.w_part = o;    o += align_up(sizeof(double) * 2 * 2 * size_t(A.nbA));
    A.w_amax = o;    o += align_up(sizeof(double) * 2 * size_t(A.nbD));
    A.w_counter = o; o += align_up(sizeof(unsigned));
    A.w_total = o;
    return A;
}

namespace {

template <bool WB, bool IMPL, int TX, int TY, int NT, int MINB>
int step_impl(const zfv::adj::P6& L, const AdjLayout& A, const char* tape, double* lam, double* grad,
              const double* aux0, int n_aux, char* work, cudaStream_t s) {
    using namespace zfv::adj;
    using Tile = AdjTile<TX, TY, NT>;
    // per device: cheap, so set on every call
    int rc = cuda_check(cudaFuncSetAttribute(k_adj_face<WB, TX, TY, NT, MINB>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             int(Tile::smem_bytes)), "k_adj_face attribute");
    if (rc) return rc;
    const double* X = reinterpret_cast<const double*>(tape + A.off_X);
    const double* Y1 = reinterpret_cast<const double*>(tape + A.off_Y1);
    const double* qs1 = reinterpret_cast<const double*>(tape + A.off_qs1);
    const double* qs2 = reinterpret_cast<const double*>(tape + A.off_qs2);
    const double* meta = reinterpret_cast<const double*>(tape + A.off_meta);
    double* lamq = reinterpret_cast<double*>(work + A.w_lamq);
    double* loc = reinterpret_cast<double*>(work + A.w_loc);
    double* lamY1 = reinterpret_cast<double*>(work + A.w_lamY1);
    double* part = reinterpret_cast<double*>(work + A.w_part);
    double* amax = reinterpret_cast<double*>(work + A.w_amax);
    unsigned* counter = reinterpret_cast<unsigned*>(work + A.w_counter);
    const dim3 fgrid((L.nx + TX - 1) / TX, (L.ny + TY - 1) / TY);
    // stage 2: Y2 = stage(Y1), Q^{n+1} = (Q^n + Y2)/2 -> lam_Y2 = lam/2
    k_adj_cell<IMPL, kCellNT><<<A.nbA, kCellNT, 0, s>>>(lam, 0.5, Y1, qs2, L, meta, lamq, loc, part);
    k_adj_face<WB, TX, TY, NT, MINB><<<fgrid, NT, Tile::smem_bytes, s>>>(
        Y1, X, lamq, loc, nullptr, 0.0, L, meta, lamY1);
    // stage 1: Y1 = stage(Q^n); lam_n = (dY1/dQ^n)^T lam_Y1 + lam/2
    k_adj_cell<IMPL, kCellNT><<<A.nbA, kCellNT, 0, s>>>(lamY1, 1.0, X, qs1, L, meta, lamq, loc,
                                                        part + 2 * A.nbA);
    k_adj_face<WB, TX, TY, NT, MINB><<<fgrid, NT, Tile::smem_bytes, s>>>(
        X, X, lamq, loc, lam, 0.5, L, meta, lam);
    // dt_n = dt(Q^n)
    k_adj_dt<256><<<A.nbD, 256, 0, s>>>(X, aux0, n_aux, L, meta, part, 2 * A.nbA, amax, counter, lam, grad);
    return cuda_check(cudaGetLastError(), "zfv_adj_step launch");
}

template <bool WB, bool IMPL>
struct StepF {
    const zfv::adj::P6& L; const AdjLayout& A; const char* tape; double* lam; double* grad;
    const double* aux0; int n_aux; char* work; cudaStream_t s;
    template <int TX, int TY, int NT, int MINB> int operator()() {
        return step_impl<WB, IMPL, TX, TY, NT, MINB>(L, A, tape, lam, grad, aux0, n_aux, work, s);
    }
};

}  // namespace

int adj_step_swe2d(const void* Lp, bool wb, bool impl, const AdjLayout& A, const char* tape_step,
                   double* lam, double* grad, const double* aux0, int n_aux, char* work,
                   cudaStream_t s) {
    const auto& L = *static_cast<const zfv::adj::P6*>(Lp);
    const int v = g_adj_variant.load();
    if (wb) return impl ? with_adj_variant(v, StepF<true, true>{L, A, tape_step, lam, grad, aux0, n_aux, work, s})
                        : with_adj_variant(v, StepF<true, false>{L, A, tape_step, lam, grad, aux0, n_aux, work, s});
    return impl ? with_adj_variant(v, StepF<false, true>{L, A, tape_step, lam, grad, aux0, n_aux, work, s})
                : with_adj_variant(v, StepF<false, false>{L, A, tape_step, lam, grad, aux0, n_aux, work, s});
}

int adj_set_variant(int v) {
    if (v < 0 || v >= kAdjVariants) return fail(-1, "zfv_adj_set_variant: unknown variant %d", v);
    g_adj_variant.store(v);
    return 0;
}

int adj_variants() { return kAdjVariants; }

}  // namespace zfvi
