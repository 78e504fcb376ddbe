// Host build of the hand-written stage adjoint (zoomy_amrex_b200/csrc/swe_adjoint.H)
// for CPU tests: a plain loop version of one SSP-RK2 stage of the 2-D SWE
// scheme (forward) and of its reverse, over a single box with mirrored ghost
// cells (walls flip the normal momentum, extrapolation copies).
//
// Built by tests/test_adjoint_cpu.py with g++ -O2 -ffp-contract=off.
#include <cmath>
#include <cstring>
#include <vector>
#include "swe_adjoint.H"

using R = double;
using zadj::SweP;

namespace {

struct Grid {
    int nx, ny;
    R dx, dy;
    int bc[4];   // x_lo, x_hi, y_lo, y_hi: 0 extrapolation, 1 wall
    size_t pl() const { return size_t(nx) * ny; }
};

// Cell (i, j) possibly outside: mirrored interior cell and the sign of the
// normal momentum component (wall) or +1.
inline void ghost(const Grid& G, int i, int j, int& ii, int& jj, int& flip_comp) {
    ii = i; jj = j; flip_comp = -1;
    if (i < 0) { ii = -1 - i; if (G.bc[0] == 1) flip_comp = 2; }
    else if (i >= G.nx) { ii = 2 * G.nx - 1 - i; if (G.bc[1] == 1) flip_comp = 2; }
    if (j < 0) { jj = -1 - j; if (G.bc[2] == 1 && flip_comp < 0) flip_comp = 3; }
    else if (j >= G.ny) { jj = 2 * G.ny - 1 - j; if (G.bc[3] == 1 && flip_comp < 0) flip_comp = 3; }
}

inline void load(const Grid& G, const R* Q, int i, int j, R out[4]) {
    int ii, jj, f;
    ghost(G, i, j, ii, jj, f);
    const size_t c = size_t(jj) * G.nx + ii;
    for (int n = 0; n < 4; ++n) out[n] = Q[n * G.pl() + c];
    if (f >= 0) out[f] = -out[f];
}

inline void scatter(const Grid& G, R* L, int i, int j, const R v[4]) {
    int ii, jj, f;
    ghost(G, i, j, ii, jj, f);
    const size_t c = size_t(jj) * G.nx + ii;
    for (int n = 0; n < 4; ++n) L[n * G.pl() + c] += (n == f) ? -v[n] : v[n];
}

// The face on the low side of cell (i, j) in direction D (stencil i-2 .. i+1).
template <int D, bool WB>
void face_at(const Grid& G, const R* Q, int i, int j, SweP<R> const& p, R o[zadj::kFaceOut]) {
    R c[4][4];
    for (int k = 0; k < 4; ++k) load(G, Q, D == 0 ? i - 2 + k : i, D == 0 ? j : j - 2 + k, c[k]);
    zadj::face_fwd<D, WB>(c, p, o);
}

// q* = X + dt * RHS(X) (before the implicit source), face-based.
template <bool WB>
void explicit_part(const Grid& G, const R* X, R dt, SweP<R> const& p, R* qs) {
    const size_t pl = G.pl();
    std::memcpy(qs, X, sizeof(R) * 4 * pl);
    for (int j = 0; j < G.ny; ++j)
        for (int i = 0; i < G.nx; ++i) {
            R l[11], r[11], b[11], t[11];
            face_at<0, WB>(G, X, i, j, p, l);        // face i-1/2 (cells i-1, i)
            face_at<0, WB>(G, X, i + 1, j, p, r);    // face i+1/2 (cells i, i+1)
            face_at<1, WB>(G, X, i, j, p, b);
            face_at<1, WB>(G, X, i, j + 1, p, t);
            const size_t c = size_t(j) * G.nx + i;
            for (int n = 0; n < 3; ++n) {
                const R Fx = -(r[n] - l[n]) - r[6 + n] - l[3 + n];
                const R Fy = -(t[n] - b[n]) - t[6 + n] - b[3 + n];
                R rhs = Fx / G.dx + Fy / G.dy;
                if (WB) {
                    if (n == 1) rhs += R(0.5) * p.g * (r[9] * r[9] - l[10] * l[10]) / G.dx;
                    if (n == 2) rhs += R(0.5) * p.g * (t[9] * t[9] - b[10] * b[10]) / G.dy;
                }
                qs[(n + 1) * pl + c] += dt * rhs;
            }
        }
}

}  // namespace

extern "C" {

// One stage: Y = q* + dq(q*) (implicit) or q* (explicit source off).
int adj_stage_fwd(int nx, int ny, R dx, R dy, const int* bc, const R* par, int wb, int impl,
                  const R* X, R dt, R* Y) {
    Grid G{nx, ny, dx, dy, {bc[0], bc[1], bc[2], bc[3]}};
    SweP<R> p{par[0], par[1], par[2], par[3], par[4], par[5]};
    if (wb) explicit_part<true>(G, X, dt, p, Y);
    else explicit_part<false>(G, X, dt, p, Y);
    if (impl) {
        const size_t pl = G.pl();
        for (size_t c = 0; c < pl; ++c) {
            const R hv = zadj::hinv(X[pl + c], p.eps);
            R dq[2];
            zadj::implicit_fwd(Y[pl + c], Y[2 * pl + c], Y[3 * pl + c], hv, dt, p, dq);
            Y[2 * pl + c] += dq[0];
            Y[3 * pl + c] += dq[1];
        }
    }
    return 0;
}

// lamX = (dY/dX)^T lamY; lnm += dL/dn_m, ldt += dL/ddt.
int adj_stage_rev(int nx, int ny, R dx, R dy, const int* bc, const R* par, int wb, int impl,
                  const R* X, R dt, const R* lamY, R* lamX, R* lnm, R* ldt) {
    Grid G{nx, ny, dx, dy, {bc[0], bc[1], bc[2], bc[3]}};
    SweP<R> p{par[0], par[1], par[2], par[3], par[4], par[5]};
    const size_t pl = G.pl();
    std::vector<R> qs(4 * pl), lq(4 * pl), Rhs(4 * pl);
    if (wb) explicit_part<true>(G, X, dt, p, qs.data());
    else explicit_part<false>(G, X, dt, p, qs.data());
    std::memset(lamX, 0, sizeof(R) * 4 * pl);
    // implicit part, per cell
    for (size_t c = 0; c < pl; ++c) {
        for (int n = 0; n < 4; ++n) lq[n * pl + c] = lamY[n * pl + c];
        if (!impl) continue;
        R lqc[4] = {0, 0, 0, 0}, lhv = 0;
        const R hv = zadj::hinv(X[pl + c], p.eps);
        const R lam[2] = {lamY[2 * pl + c], lamY[3 * pl + c]};
        zadj::implicit_rev(qs[pl + c], qs[2 * pl + c], qs[3 * pl + c], hv, dt, p, lam, lqc, lhv, *lnm, *ldt);
        for (int n = 1; n < 4; ++n) lq[n * pl + c] += lqc[n];
        lamX[pl + c] += lhv * zadj::dhinv(X[pl + c], p.eps);
    }
    // q* = X + dt RHS(X): identity + dt * (dRHS/dX)^T lq; ldt += lq . RHS
    for (size_t c = 0; c < pl; ++c)
        for (int n = 0; n < 4; ++n) {
            lamX[n * pl + c] += lq[n * pl + c];
            *ldt += lq[n * pl + c] * (qs[n * pl + c] - X[n * pl + c]) / dt;
        }
    for (int D = 0; D < 2; ++D) {
        const int nfx = (D == 0) ? nx + 1 : nx, nfy = (D == 0) ? ny : ny + 1;
        const R h = (D == 0) ? dx : dy;
        for (int j = 0; j < nfy; ++j)
            for (int i = 0; i < nfx; ++i) {
                // face between cell A = (i-1, j) / (i, j-1) and B = (i, j)
                const int ia = (D == 0) ? i - 1 : i, ja = (D == 0) ? j : j - 1;
                const bool hasA = ia >= 0 && ja >= 0, hasB = i < nx && j < ny;
                R lA[4] = {0, 0, 0, 0}, lB[4] = {0, 0, 0, 0};
                if (hasA) for (int n = 0; n < 4; ++n) lA[n] = lq[n * pl + size_t(ja) * nx + ia];
                if (hasB) for (int n = 0; n < 4; ++n) lB[n] = lq[n * pl + size_t(j) * nx + i];
                R lo[11];
                const R sc = dt / h;
                for (int n = 0; n < 3; ++n) {
                    lo[n] = sc * (lB[n + 1] - lA[n + 1]);      // A: -f, B: +f
                    lo[3 + n] = -sc * lB[n + 1];               // D+ into B (its left face)
                    lo[6 + n] = -sc * lA[n + 1];               // D- into A (its right face)
                }
                R c[4][4];
                for (int k = 0; k < 4; ++k)
                    load(G, X, D == 0 ? i - 2 + k : i, D == 0 ? j : j - 2 + k, c[k]);
                lo[9] = 0; lo[10] = 0;
                // +0.5 g hL*^2 into A, -0.5 g hR*^2 into B (well-balanced only)
                const R wA = wb ? sc * p.g * lA[2 + D] : R(0), wB = wb ? -sc * p.g * lB[2 + D] : R(0);
                R lc[4][4] = {};
                if (D == 0) { if (wb) zadj::face_rev<0, true>(c, p, lo, wA, wB, lc); else zadj::face_rev<0, false>(c, p, lo, wA, wB, lc); }
                else { if (wb) zadj::face_rev<1, true>(c, p, lo, wA, wB, lc); else zadj::face_rev<1, false>(c, p, lo, wA, wB, lc); }
                for (int k = 0; k < 4; ++k)
                    scatter(G, lamX, D == 0 ? i - 2 + k : i, D == 0 ? j : j - 2 + k, lc[k]);
            }
    }
    return 0;
}

// The face map alone (for FD checks of face_rev).
int adj_face_fwd(int D, int wb, const R* par, const R* c16, R* o) {
    SweP<R> p{par[0], par[1], par[2], par[3], par[4], par[5]};
    R c[4][4];
    std::memcpy(c, c16, sizeof c);
    if (D == 0) { if (wb) zadj::face_fwd<0, true>(c, p, o); else zadj::face_fwd<0, false>(c, p, o); }
    else { if (wb) zadj::face_fwd<1, true>(c, p, o); else zadj::face_fwd<1, false>(c, p, o); }
    return 0;
}
int adj_face_rev(int D, int wb, const R* par, const R* c16, const R* lo, R* lc16) {
    SweP<R> p{par[0], par[1], par[2], par[3], par[4], par[5]};
    R c[4][4], lc[4][4] = {};
    std::memcpy(c, c16, sizeof c);
    if (D == 0) { if (wb) zadj::face_rev<0, true>(c, p, lo, R(0), R(0), lc); else zadj::face_rev<0, false>(c, p, lo, R(0), R(0), lc); }
    else { if (wb) zadj::face_rev<1, true>(c, p, lo, R(0), R(0), lc); else zadj::face_rev<1, false>(c, p, lo, R(0), R(0), lc); }
    std::memcpy(lc16, lc, sizeof lc);
    return 0;
}

}  // extern "C"
