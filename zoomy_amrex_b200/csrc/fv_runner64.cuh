// The FP64 plain form's runner: one compiled Model::/Numerics:: pair behind
// the Runner interface of zfv_internal.H (fused stage kernels, MOOD, the
// global implicit source, the adjoint's forward recording, validation
// entries). Each model family instantiates it in a translation unit of its own
// (zoomy_fv64_swe.cu, zoomy_fv64_sme.cu), so the families compile in parallel.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <cuda_runtime.h>

#include "zoomy_fv.h"
#include "zfv_internal.H"
#include "swe.H"
#include "fv_kernels.cuh"
#include "fv_jfnk.cuh"

namespace zfv64 {

using namespace zfvi;

template <class Model, class Numerics, int TX, int TY>
struct RunnerT final : Runner {
    static constexpr int NP = Model::n_parameters;
    static constexpr int nq = Model::n_dof_q;
    using PL = zfv::LevelParams<double, NP>;

    zfv_handle* h;
    PL L;
    dim3 grid, block;

    explicit RunnerT(zfv_handle* hh) : h(hh) {
        const zfv_config& c = h->cfg;
        std::memset(&L, 0, sizeof L);
        L.nx = c.nx; L.ny = c.ny;
        L.plane = (long long)c.nx * c.ny;
        L.dx = (c.prob_hi[0] - c.prob_lo[0]) / c.nx;
        L.dy = (c.prob_hi[1] - c.prob_lo[1]) / c.ny;
        L.plox = c.prob_lo[0]; L.ploy = c.prob_lo[1];
        for (int k = 0; k < NP; ++k) L.p[k] = c.params[k];
        for (int s = 0; s < 4; ++s) L.bc_tag[s] = c.bc_tag[s];
        L.clamp = c.clamp_positivity && !c.positivity_mood;   // ZoomyAmr.cpp:303
        L.well_balanced = c.well_balanced;
        L.implicit_source = c.implicit_source;
        L.cfl = c.cfl; L.dtmin = c.dtmin; L.dtmax = c.dtmax; L.time_end = c.time_end;
        L.max_step = c.max_step;
        L.cfl_dimension = c.cfl_dimension; L.cfl_degree_factor = c.cfl_degree_factor;
        grid = dim3((c.nx + TX - 1) / TX, (c.ny + TY - 1) / TY, 1);
        block = dim3(TX * TY, 1, 1);
    }

    bool mood() const { return h->cfg.positivity_mood && h->cfg.spatial_order == 2; }

    void layout(ScratchLayout& S) const override {
        const size_t plane_bytes = size_t(L.plane) * sizeof(double);
        const int nblk = std::max(int(grid.x * grid.y), kReduceBlocksMax);
        S.state = 0;
        S.partials = align_up(sizeof(zfv::DevState));
        S.log = S.partials + align_up(sizeof(double) * 2 * nblk);
        S.stage = S.log + align_up(sizeof(double) * 3 * kLogCap);
        S.lo = 0;
        S.jfnk = 0;
        if (mood() || jfnk()) {   // second stage buffer: the MOOD candidate / the stage-2 Newton state
            S.alt = S.stage + align_up(plane_bytes * nq);
            S.total = S.alt + align_up(plane_bytes * nq);
        } else {
            S.alt = 0;
            S.total = S.stage + align_up(plane_bytes * nq);
        }
        if (jfnk()) {
            S.jfnk = S.total;
            S.total += jfnk_bytes();
        }
    }

    int state_import(const double* Q64, void* Q, char*, cudaStream_t s) override {
        return cuda_check(cudaMemcpyAsync(Q, Q64, size_t(L.plane) * nq * sizeof(double),
                                          cudaMemcpyDeviceToDevice, s), "zfv_state_import copy");
    }
    int state_export(const void* Q, const char*, double* Q64, cudaStream_t s) override {
        return cuda_check(cudaMemcpyAsync(Q64, Q, size_t(L.plane) * nq * sizeof(double),
                                          cudaMemcpyDeviceToDevice, s), "zfv_state_export copy");
    }

    template <int ORDER, int MODE, bool WB, bool IMPL>
    static auto kfn() { return &zfv::k_stage<Model, Numerics, ORDER, MODE, WB, IMPL, TX, TY>; }

    template <int ORDER, int MODE>
    using ShapeOf = zfv::TileShape<Model, ORDER, TX, TY, zfv::static_bed<Model>::value && MODE != zfv::MODE_RHS>;

    template <int ORDER, int MODE, bool WB, bool IMPL>
    int set_smem() {
        using Sh = ShapeOf<ORDER, MODE>;
        return cuda_check(cudaFuncSetAttribute(kfn<ORDER, MODE, WB, IMPL>(),
                                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               int(Sh::smem_bytes)),
                          "cudaFuncSetAttribute");
    }

    template <int ORDER, bool WB, bool IMPL>
    int setup_combo() {
        int rc = 0;
        if constexpr (IMPL) rc |= set_smem<ORDER, zfv::MODE_X, WB, IMPL>();
        rc |= set_smem<ORDER, zfv::MODE_RHS, WB, IMPL>();
        if constexpr (ORDER == 2) {
            rc |= set_smem<ORDER, zfv::MODE_S1, WB, IMPL>();
            rc |= set_smem<ORDER, zfv::MODE_S2, WB, IMPL>();
            rc |= set_smem<ORDER, zfv::MODE_S2M, WB, IMPL>();
            rc |= set_smem<1, zfv::MODE_R1, WB, IMPL>();
            rc |= set_smem<1, zfv::MODE_R2, WB, IMPL>();
        } else {
            rc |= set_smem<ORDER, zfv::MODE_ONE, WB, IMPL>();
        }
        return rc;
    }

    // Runtime flags -> compile-time instantiation.
    template <class F>
    int with_combo(F&& f) {
        const zfv_config& c = h->cfg;
        const bool wb = c.well_balanced != 0, im = c.implicit_source != 0;
        if (c.spatial_order == 2) {
            if (wb) return im ? f.template operator()<2, true, true>() : f.template operator()<2, true, false>();
            return im ? f.template operator()<2, false, true>() : f.template operator()<2, false, false>();
        }
        if (wb) return im ? f.template operator()<1, true, true>() : f.template operator()<1, true, false>();
        return im ? f.template operator()<1, false, true>() : f.template operator()<1, false, false>();
    }

    struct SetupF {
        RunnerT* r;
        template <int O, bool W, bool I> int operator()() { return r->template setup_combo<O, W, I>(); }
    };
    int setup() override { return with_combo(SetupF{this}); }

    zfv::DevState* st(char* scratch) const { return reinterpret_cast<zfv::DevState*>(scratch + h->lay.state); }
    double* partials(char* scratch) const { return reinterpret_cast<double*>(scratch + h->lay.partials); }
    double* log3(char* scratch) const { return reinterpret_cast<double*>(scratch + h->lay.log); }
    double* stage(char* scratch) const { return reinterpret_cast<double*>(scratch + h->lay.stage); }
    double* stage2(char* scratch) const { return reinterpret_cast<double*>(scratch + h->lay.alt); }

    int reduce_blocks() const {
        long long need = (L.plane + kReduceNT - 1) / kReduceNT;
        return int(need < kReduceBlocksMax ? (need > 0 ? need : 1) : kReduceBlocksMax);
    }

    int begin(const void* Q, const void* A, char* scratch, cudaStream_t s) override {
        jfnk_newton = jfnk_gmres = jfnk_solves = 0;
        zfv::k_begin<<<1, 1, 0, s>>>(st(scratch), L);
        zfv::k_reduce<Model, Numerics, kReduceNT, 0, true><<<reduce_blocks(), kReduceNT, 0, s>>>(
            (const double*)Q, (const double*)A, L, st(scratch), partials(scratch));
        return cuda_check(cudaGetLastError(), "zfv_begin launch");
    }

    int update_state(void* Q, void* A, double time, cudaStream_t s) override {
        const int nb = int((L.plane + 255) / 256);
        zfv::k_update_state<Model><<<nb, 256, 0, s>>>((double*)Q, (double*)A, L, time);
        return cuda_check(cudaGetLastError(), "zfv_update_state launch");
    }

    int compute_dt(const void* Q, const void* A, char* scratch, cudaStream_t s) override {
        zfv::k_reduce<Model, Numerics, kReduceNT, 0, false><<<reduce_blocks(), kReduceNT, 0, s>>>(
            (const double*)Q, (const double*)A, L, st(scratch), partials(scratch));
        return cuda_check(cudaGetLastError(), "zfv_compute_dt launch");
    }

    int total_mass(const void* Q, char* scratch, cudaStream_t s) override {
        zfv::k_reduce<Model, Numerics, kReduceNT, 1, false><<<reduce_blocks(), kReduceNT, 0, s>>>(
            (const double*)Q, nullptr, L, st(scratch), partials(scratch));
        return cuda_check(cudaGetLastError(), "zfv_total_mass launch");
    }

    template <int ORDER, int MODE, bool WB, bool IMPL>
    void launch(const double* qin, const double* qbed, const double* qold, double* qout,
                char* scratch, cudaStream_t s, double time_arg = 0.0, double* qstar = nullptr) {
        using Sh = ShapeOf<ORDER, MODE>;
        auto kernel = kfn<ORDER, MODE, WB, IMPL>();
        kernel<<<grid, block, Sh::smem_bytes, s>>>(
            qin, qbed, qold, qout, L, scratch ? st(scratch) : nullptr,
            scratch ? partials(scratch) : nullptr, scratch ? log3(scratch) : nullptr,
            scratch ? kLogCap : 0, time_arg, qstar);
    }

    struct EvolveF {
    RunnerT* r; double* Q; double* Q1; char* scratch; int n; cudaStream_t s; bool sbed;
    template <int O, bool W, bool I> int operator()() {
        bool in_q1 = false;
        const bool mood = r->mood();
        double* Q2 = mood ? r->stage2(scratch) : nullptr;
        for (int k = 0; k < n; ++k) {
            if constexpr (O == 2) {
                r->template launch<2, zfv::MODE_S1, W, I>(Q, Q, nullptr, Q1, scratch, s);
                if (!mood) {
                    r->template launch<2, zfv::MODE_S2, W, I>(Q1, Q, Q, Q, scratch, s);
                } else {
                    // ZoomyAmr.cpp:699-720: candidate, then commit or whole-step order-1 redo
                    r->template launch<2, zfv::MODE_S2M, W, I>(Q1, Q, Q, Q2, scratch, s);
                    const int nb = int((r->L.plane + kReduceNT - 1) / kReduceNT);
                    zfv::k_mood_commit<Model, Numerics, kReduceNT><<<nb, kReduceNT, 0, s>>>(
                        Q2, Q, r->L, r->st(scratch), r->partials(scratch), r->log3(scratch), kLogCap);
                    r->template launch<1, zfv::MODE_R1, W, I>(Q, Q, nullptr, Q1, scratch, s);
                    r->template launch<1, zfv::MODE_R2, W, I>(Q1, Q, Q, Q, scratch, s);
                }
            } else {
                double* src = in_q1 ? Q1 : Q;
                double* dst = in_q1 ? Q : Q1;
                r->template launch<1, zfv::MODE_ONE, W, I>(src, Q, nullptr, dst, scratch, s);
                in_q1 = !in_q1;
            }
        }
        if (in_q1) {   // order-1 ping-pong ended in the stage buffer: copy the state back
            const size_t pb = size_t(r->L.plane) * sizeof(double);
            const int n0 = sbed ? 1 : 0;
            cudaError_t e = cudaMemcpyAsync(Q + n0 * r->L.plane, Q1 + n0 * r->L.plane,
                                            pb * (nq - n0), cudaMemcpyDeviceToDevice, s);
            if (e != cudaSuccess) return cuda_check(e, "zfv_evolve copy-back");
        }
        return cuda_check(cudaGetLastError(), "zfv_evolve launch");
    }
    };

    int evolve(void* Qv, void* Av, char* scratch, int n, cudaStream_t s) override {
        double* Q = (double*)Qv;
        double* Q1 = stage(scratch);
        const bool sbed = zfv::static_bed<Model>::value;
        int rc = jfnk() ? with_combo(JfnkEvolveF{this, Q, scratch, n, s})
                        : with_combo(EvolveF{this, Q, Q1, scratch, n, s, sbed});
        if (rc) return rc;
        const int nb = int((L.plane + 255) / 256);
        zfv::k_aux_from_state<Model><<<nb, 256, 0, s>>>(Q, (double*)Av, L, st(scratch));
        return cuda_check(cudaGetLastError(), "zfv_evolve aux launch");
    }

    // -- global implicit source (solver.implicit_global, imex_solver.H) ---------
    // Newton: at most 12 iterations, stop at |F| < 1e-12 or |F| < 1e-9 |F_0|,
    // linear tolerance 1e-4 relative (imex_solver.H:124-140). GMRES: restarted
    // every 30 iterations, at most 40 iterations per solve, classical
    // Gram-Schmidt applied twice (two host round trips per iteration: the
    // second pass also returns |w|^2), Givens rotations on the host.
    static constexpr int n0 = zfv::static_bed<Model>::value ? 1 : 0;
    static constexpr int kNewtonMax = 12;
    static constexpr int kRestart = 30;
    static constexpr int kMaxIter = 40;
    static_assert(kRestart + 2 <= zfv::jfnk::kMaxDots, "Krylov basis larger than one multi-dot launch");

    bool jfnk() const { return h->cfg.implicit_source && h->cfg.implicit_global; }
    long long jN() const { return (long long)(nq - n0) * L.plane; }
    int jvec_blocks() const {
        const long long b = (jN() + zfv::jfnk::kNT - 1) / zfv::jfnk::kNT;
        return int(std::min<long long>(b, kReduceBlocksMax));
    }
    int jcell_blocks() const { return int((L.plane + zfv::jfnk::kNT - 1) / zfv::jfnk::kNT); }
    size_t jpart_elems() const {
        return std::max<size_t>(size_t(jcell_blocks()), size_t(zfv::jfnk::kMaxDots) * jvec_blocks());
    }
    size_t jvec_bytes() const { return align_up(size_t(jN()) * sizeof(double)); }
    size_t jfnk_bytes() const {
        return jvec_bytes() * (5 + kRestart + 1) + align_up(jpart_elems() * sizeof(double)) +
               align_up(zfv::jfnk::kMaxDots * sizeof(double));
    }
    struct JW {
        double *qexp, *S, *F, *x, *w, *V, *part, *out;
    };
    JW jwork(char* scratch) const {
        const size_t vb = jvec_bytes();
        char* b = scratch + h->lay.jfnk;
        JW W;
        W.qexp = (double*)(b);
        W.S = (double*)(b + vb);
        W.F = (double*)(b + 2 * vb);
        W.x = (double*)(b + 3 * vb);
        W.w = (double*)(b + 4 * vb);
        W.V = (double*)(b + 5 * vb);
        W.part = (double*)(b + (5 + kRestart + 1) * vb);
        W.out = (double*)(b + (5 + kRestart + 1) * vb + align_up(jpart_elems() * sizeof(double)));
        return W;
    }
    long long jstride() const { return (long long)(jvec_bytes() / sizeof(double)); }

    // host[k] = w . V_k for k < nv, and with self_last host[nv] = w . w
    // (synchronizes the stream).
    int jdots(const JW& W, const double* w, const double* V, long long vstride, int nv, long long n,
              double* host, cudaStream_t s, bool self_last = false) {
        const int nb = jvec_blocks();
        const int nt = nv + (self_last ? 1 : 0);
        zfv::jfnk::k_dots<<<dim3(nb, nt), zfv::jfnk::kNT, 0, s>>>(w, V, vstride, n, W.part, self_last ? 1 : 0);
        zfv::jfnk::k_sum_partials<<<nt, zfv::jfnk::kNT, 0, s>>>(W.part, nb, W.out);
        int rc = cuda_check(cudaMemcpyAsync(host, W.out, sizeof(double) * nt, cudaMemcpyDeviceToHost, s),
                            "implicit_global dot read-back");
        if (!rc) rc = cuda_check(cudaStreamSynchronize(s), "implicit_global dot");
        return rc;
    }
    void jcombine(double* y, double a, const double* V, int nv, const double* c, cudaStream_t s) {
        zfv::jfnk::Coefs cf{};
        for (int k = 0; k < nv; ++k) cf.c[k] = c[k];
        zfv::jfnk::k_combine<<<jvec_blocks(), zfv::jfnk::kNT, 0, s>>>(y, a, V, jstride(), nv, cf, jN());
    }
    void jscale(double* dst, const double* src, double f, cudaStream_t s) {
        zfv::jfnk::k_scale<<<jvec_blocks(), zfv::jfnk::kNT, 0, s>>>(dst, src, f, jN());
    }
    // Ax = J x at Qv (ImpSrcOp::apply): eps = 1e-7 (1 + |Q|) / |x|
    int jjvp(const double* Qv, const double* qbed, const JW& W, const zfv::DevState* state, const double* x,
             double xnorm, double nrmQ, double* Ax, cudaStream_t s) {
        if (xnorm == 0.0)
            return cuda_check(cudaMemsetAsync(Ax, 0, sizeof(double) * jN(), s), "implicit_global memset");
        const double eps = 1e-7 * (1.0 + nrmQ) / xnorm;
        zfv::jfnk::k_jvp<Model><<<jcell_blocks(), zfv::jfnk::kNT, 0, s>>>(Qv, qbed, W.S, x, eps, Ax, L, state);
        return cuda_check(cudaGetLastError(), "implicit_global J x launch");
    }

    // GMRES on J x = b from x = 0 (x, b: vectors; J at the Newton iterate Qv
    // with S(Qv) in W.S).
    int jgmres(const double* Qv, const double* qbed, const JW& W, const zfv::DevState* state, const double* b,
               double* x, double nrmQ, double rtol, cudaStream_t s) {
        const long long N = jN(), vs = jstride();
        double beta;
        int rc = jdots(W, b, b, 0, 1, N, &beta, s);
        if (rc) return rc;
        beta = std::sqrt(beta);
        if (!(beta > 0.0)) return 0;
        const double target = rtol * beta;
        double H[kRestart + 1][kRestart], cs[kRestart], sn[kRestart], g[kRestart + 1], hcol[kRestart + 1],
            h2[kRestart + 1], y[kRestart];
        int iters = 0;
        jscale(W.V, b, 1.0 / beta, s);                      // V_0 = r / beta, r = b
        for (;;) {
            for (int k = 0; k <= kRestart; ++k) g[k] = 0.0;
            g[0] = beta;
            int kdim = 0;
            double res = beta;
            for (int j = 0; j < kRestart && iters < kMaxIter; ++j) {
                double* Vj = W.V + j * vs;
                rc = jjvp(Qv, qbed, W, state, Vj, 1.0, nrmQ, W.w, s);   // |V_j| = 1
                if (!rc) rc = jdots(W, W.w, W.V, vs, j + 1, N, hcol, s);
                if (rc) return rc;
                for (int k = 0; k <= j; ++k) hcol[k] = -hcol[k];
                jcombine(W.w, 1.0, W.V, j + 1, hcol, s);
                // second pass, with |w|^2 in the same reduction: after it
                // |w'|^2 = |w|^2 - |h2|^2 (V orthonormal; h2 is round-off
                // small after the first pass, so nothing cancels)
                rc = jdots(W, W.w, W.V, vs, j + 1, N, h2, s, true);
                if (rc) return rc;
                double hn = h2[j + 1];
                for (int k = 0; k <= j; ++k) {
                    hn -= h2[k] * h2[k];
                    hcol[k] = -hcol[k] + h2[k];
                    h2[k] = -h2[k];
                }
                jcombine(W.w, 1.0, W.V, j + 1, h2, s);
                hn = std::sqrt(std::max(hn, 0.0));
                for (int k = 0; k <= j; ++k) H[k][j] = hcol[k];
                H[j + 1][j] = hn;
                for (int k = 0; k < j; ++k) {              // previous rotations
                    const double t = cs[k] * H[k][j] + sn[k] * H[k + 1][j];
                    H[k + 1][j] = -sn[k] * H[k][j] + cs[k] * H[k + 1][j];
                    H[k][j] = t;
                }
                const double den = std::hypot(H[j][j], H[j + 1][j]);
                cs[j] = den > 0.0 ? H[j][j] / den : 1.0;
                sn[j] = den > 0.0 ? H[j + 1][j] / den : 0.0;
                H[j][j] = den;
                H[j + 1][j] = 0.0;
                g[j + 1] = -sn[j] * g[j];
                g[j] = cs[j] * g[j];
                res = std::fabs(g[j + 1]);
                ++iters;
                ++jfnk_gmres;
                kdim = j + 1;
                if (hn > 0.0) jscale(W.V + (j + 1) * vs, W.w, 1.0 / hn, s);
                if (res <= target || !(hn > 0.0)) break;
            }
            for (int i = kdim - 1; i >= 0; --i) {         // H y = g
                double t = g[i];
                for (int k = i + 1; k < kdim; ++k) t -= H[i][k] * y[k];
                y[i] = H[i][i] != 0.0 ? t / H[i][i] : 0.0;
            }
            jcombine(x, 1.0, W.V, kdim, y, s);
            if (res <= target || iters >= kMaxIter || kdim == 0) break;
            // restart: r = b - J x into V_0
            double xn;
            rc = jdots(W, x, x, 0, 1, N, &xn, s);
            if (rc) return rc;
            rc = jjvp(Qv, qbed, W, state, x, std::sqrt(xn), nrmQ, W.w, s);
            if (rc) return rc;
            jscale(W.V, b, 1.0, s);
            const double m1 = -1.0;
            jcombine(W.V, 1.0, W.w, 1, &m1, s);
            rc = jdots(W, W.V, W.V, 0, 1, N, &beta, s);
            if (rc) return rc;
            beta = std::sqrt(beta);
            if (!(beta > target)) break;
            jscale(W.V, W.V, 1.0 / beta, s);
        }
        return cuda_check(cudaGetLastError(), "implicit_global GMRES launch");
    }

    // SolveImplicitSourceGlobal (imex_solver.H:102-160) on the stage state Qv
    // (a vector; it holds Qexp on entry and the Newton solution on exit).
    int jsolve(double* Qv, const double* qbed, char* scratch, cudaStream_t s) {
        const JW W = jwork(scratch);
        const long long N = jN();
        int rc = cuda_check(cudaMemcpyAsync(W.qexp, Qv, sizeof(double) * N, cudaMemcpyDeviceToDevice, s),
                            "implicit_global copy");
        if (rc) return rc;
        double resid0 = -1.0;
        ++jfnk_solves;
        for (int it = 0; it < kNewtonMax; ++it) {
            zfv::jfnk::k_residual<Model><<<jcell_blocks(), zfv::jfnk::kNT, 0, s>>>(
                Qv, qbed, W.qexp, W.S, W.F, L, st(scratch), W.part);
            zfv::jfnk::k_sum_partials<<<1, zfv::jfnk::kNT, 0, s>>>(W.part, jcell_blocks(), W.out);
            double r2;
            rc = cuda_check(cudaMemcpyAsync(&r2, W.out, sizeof(double), cudaMemcpyDeviceToHost, s),
                            "implicit_global residual read-back");
            if (!rc) rc = cuda_check(cudaStreamSynchronize(s), "implicit_global residual");
            if (rc) return rc;
            const double resid = std::sqrt(r2);
            if (it == 0) resid0 = resid;
            if (resid < 1e-12 || (resid0 > 0.0 && resid < 1e-9 * resid0)) break;
            ++jfnk_newton;
            jscale(W.F, W.F, -1.0, s);                      // rhs = -F
            double qq, bb = 0.0;                            // |Q| over all components
            rc = jdots(W, Qv, Qv, 0, 1, N, &qq, s);
            if (!rc && n0 == 1) rc = jdots(W, qbed, qbed, 0, 1, L.plane, &bb, s);
            if (rc) return rc;
            const double nrmQ = std::sqrt(qq + bb);
            rc = cuda_check(cudaMemsetAsync(W.x, 0, sizeof(double) * N, s), "implicit_global memset");
            if (!rc) rc = jgmres(Qv, qbed, W, st(scratch), W.F, W.x, nrmQ, 1e-4, s);
            if (rc) return rc;
            const double one = 1.0;
            jcombine(Qv, 1.0, W.x, 1, &one, s);             // Q += delta
        }
        return cuda_check(cudaGetLastError(), "implicit_global launch");
    }

    struct JfnkEvolveF {
        RunnerT* r; double* Q; char* scratch; int n; cudaStream_t s;
        template <int O, bool W, bool I> int operator()() {
            if constexpr (!I) {
                return fail(-2, "implicit_global needs implicit_source");
            } else {
                cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
                int rc = cuda_check(cudaStreamIsCapturing(s, &cap), "cudaStreamIsCapturing");
                if (rc) return rc;
                if (cap != cudaStreamCaptureStatusNone)
                    return fail(-2, "zfv_evolve: implicit_global reads Newton-Krylov norms on the host and "
                                    "cannot run inside a CUDA graph capture");
                const long long pl = r->L.plane;
                double* E1 = r->stage(scratch);
                double* E2 = r->stage2(scratch);
                for (int k = 0; k < n; ++k) {
                    unsigned flags = 0;
                    rc = cuda_check(cudaMemcpyAsync(&flags, &r->st(scratch)->flags, sizeof flags,
                                                    cudaMemcpyDeviceToHost, s), "implicit_global flags");
                    if (!rc) rc = cuda_check(cudaStreamSynchronize(s), "implicit_global flags");
                    if (rc) return rc;
                    if (flags & zfv::kFlagDone) break;
                    const int nbc = r->jcell_blocks();
                    if constexpr (O == 2) {
                        r->template launch<2, zfv::MODE_X, W, I>(Q, Q, nullptr, E1, scratch, s);
                        rc = r->jsolve(E1 + n0 * pl, Q, scratch, s);
                        if (rc) return rc;
                        r->template launch<2, zfv::MODE_X, W, I>(E1, Q, nullptr, E2, scratch, s);
                        rc = r->jsolve(E2 + n0 * pl, Q, scratch, s);
                        if (rc) return rc;
                        zfv::jfnk::k_finish<Model, Numerics, true><<<nbc, zfv::jfnk::kNT, 0, s>>>(
                            E2 + n0 * pl, Q, r->L, r->st(scratch), r->partials(scratch), r->log3(scratch), kLogCap);
                    } else {
                        r->template launch<1, zfv::MODE_X, W, I>(Q, Q, nullptr, E1, scratch, s);
                        rc = r->jsolve(E1 + n0 * pl, Q, scratch, s);
                        if (rc) return rc;
                        zfv::jfnk::k_finish<Model, Numerics, false><<<nbc, zfv::jfnk::kNT, 0, s>>>(
                            E1 + n0 * pl, Q, r->L, r->st(scratch), r->partials(scratch), r->log3(scratch), kLogCap);
                    }
                    rc = cuda_check(cudaGetLastError(), "implicit_global step launch");
                    if (rc) return rc;
                }
                return 0;
            }
        }
    };

    struct RhsF {
        RunnerT* r; const double* Q; double* out; double time; cudaStream_t s;
        template <int O, bool W, bool I> int operator()() {
            r->template launch<O, zfv::MODE_RHS, W, I>(Q, Q, nullptr, out, nullptr, s, time);
            return cuda_check(cudaGetLastError(), "zfv_rhs launch");
        }
    };

    int rhs(const void* Q, void* out, double time, cudaStream_t s) override {
        return with_combo(RhsF{this, (const double*)Q, (double*)out, time, s});
    }

    // -- adjoint (SWE2D, order 2, FP64) ------------------------------------------
    static constexpr bool kAdj = std::is_same<Model, zb::SWE<double, 2>>::value;

    int adj_check(const char* what) const {
        const zfv_config& c = h->cfg;
        if (!kAdj || c.spatial_order != 2)
            return fail(-2, "%s: the adjoint is implemented for the FP64 SWE2D form, order 2", what);
        if (c.positivity_mood || c.clamp_positivity)
            return fail(-2, "%s: the adjoint does not differentiate clamp_positivity / MOOD", what);
        if (c.implicit_source && c.implicit_global)
            return fail(-2, "%s: the adjoint differentiates the point-implicit source, not implicit_global", what);
        return 0;
    }

    struct RecordF {
        RunnerT* r; double* Q; char* scratch; char* tape; int n; cudaStream_t s;
        template <int O, bool W, bool I> int operator()() {
            if constexpr (O != 2 || !RunnerT::kAdj) {
                return fail(-2, "zfv_adj_record: order 2 only");
            } else {
                const AdjLayout A = adj_layout(r->L.plane);
                const size_t pb = size_t(r->L.plane) * sizeof(double);
                for (int k = 0; k < n; ++k) {
                    char* t = tape + size_t(k) * A.step_bytes;
                    double* X = reinterpret_cast<double*>(t + A.off_X);
                    double* Y1 = reinterpret_cast<double*>(t + A.off_Y1);
                    double* qs1 = reinterpret_cast<double*>(t + A.off_qs1);
                    double* qs2 = reinterpret_cast<double*>(t + A.off_qs2);
                    int rc = cuda_check(cudaMemcpyAsync(X, Q, 4 * pb, cudaMemcpyDeviceToDevice, s),
                                        "zfv_adj_record state copy");
                    // (time, dt) of the step about to run: the first two doubles of DevState
                    if (!rc) rc = cuda_check(cudaMemcpyAsync(t + A.off_meta, r->st(scratch), 2 * sizeof(double),
                                                             cudaMemcpyDeviceToDevice, s),
                                             "zfv_adj_record dt copy");
                    if (rc) return rc;
                    r->template launch<2, zfv::MODE_S1, W, I>(Q, Q, nullptr, Y1, scratch, s, 0.0, qs1);
                    r->template launch<2, zfv::MODE_S2, W, I>(Y1, Q, Q, Q, scratch, s, 0.0, qs2);
                }
                return cuda_check(cudaGetLastError(), "zfv_adj_record launch");
            }
        }
    };

    int adj_record(void* Q, void* Av, char* scratch, char* tape, int n, cudaStream_t s) override {
        int rc = adj_check("zfv_adj_record");
        if (rc) return rc;
        rc = with_combo(RecordF{this, (double*)Q, scratch, tape, n, s});
        if (rc) return rc;
        const int nb = int((L.plane + 255) / 256);
        zfv::k_aux_from_state<Model><<<nb, 256, 0, s>>>((double*)Q, (double*)Av, L, st(scratch));
        return cuda_check(cudaGetLastError(), "zfv_adj_record aux launch");
    }

    int adj_step(const char* tape, int k, double* lam, double* grad, const double* aux0, char* work,
                 cudaStream_t s) override {
        int rc = adj_check("zfv_adj_step");
        if (rc) return rc;
        const AdjLayout A = adj_layout(L.plane);
        return adj_step_swe2d(&L, h->cfg.well_balanced != 0, h->cfg.implicit_source != 0, A,
                              tape + size_t(k) * A.step_bytes, lam, grad, aux0, Model::n_dof_qaux,
                              work, s);
    }

    int fill_ghosts(const void* Q, const void* A, void* Qg, void* Ag, double time,
                    cudaStream_t s) override {
        const int ng = (h->cfg.spatial_order == 2) ? 2 : 1;
        const long long gp = (long long)(L.nx + 2 * ng) * (L.ny + 2 * ng);
        const int nb = int((gp + 255) / 256);
        zfv::k_fill_ghosts<Model><<<nb, 256, 0, s>>>((const double*)Q, (const double*)A,
                                                    (double*)Qg, (double*)Ag, L, ng, time);
        return cuda_check(cudaGetLastError(), "zfv_fill_ghosts launch");
    }
};

}  // namespace zfv64
