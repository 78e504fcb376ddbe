// Portable, bit-reproducible elementary functions for model code.
//
// The Model:: functions run both in the CPU oracle (g++, -ffp-contract=off)
// and in the sm_100a kernels (nvcc --fmad=false). +,-,*,/ and sqrt are IEEE
// correctly rounded on both, so a model written only with those gives the
// same bits on both sides. pow/cbrt are not correctly rounded in either libm,
// and they differ between glibc and CUDA's libdevice, so the one non-algebraic
// power the shallow-water friction law needs, x^(-1/3), is computed here from
// exact bit-level exponent reduction, a fixed polynomial first guess and a
// fixed number of multiply-only Newton steps. Same operation sequence => same
// bits on CPU and GPU, and no division (FP64 division is a long software
// sequence on the GPU).
#pragma once
#include <cstring>
#include "AMReX_Extension.H"

namespace zb {

template <class T> struct FloatBits;
template <> struct FloatBits<double> {
    using U = unsigned long long;
    static constexpr int mbits = 52, bias = 1023;
    static constexpr U emask = 0x7ffULL;
    static constexpr int newton = 3;       // 4.8e-4 -> 4.6e-7 -> 4.3e-13 -> round-off
};
template <> struct FloatBits<float> {
    using U = unsigned int;
    static constexpr int mbits = 23, bias = 127;
    static constexpr U emask = 0xffu;
    static constexpr int newton = 2;       // 4.8e-4 -> 4.6e-7 -> round-off
};

template <class T, class U>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE T bits_to(U u) { T v; std::memcpy(&v, &u, sizeof(T)); return v; }
template <class U, class T>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE U to_bits(T v) { U u; std::memcpy(&u, &v, sizeof(T)); return u; }

// x^(-1/3) for finite x > 0. NaN for NaN or x < 0, +inf for x == 0, 0 for +inf.
// Method: x = f * 2^e, f in [1,2), e = 3q + r (r in {0,1,2});
// y0 = P(f) * 2^(-r/3) with P the cubic least-squares fit of f^(-1/3) on [1,2)
// (max relative error 4.8e-4); Newton y <- y + y (1 - w y^3)/3 on w = f 2^r,
// which roughly squares the relative error per step; result y * 2^(-q).
template <class T>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE T inv_cbrt_pos(T x)
{
    using B = FloatBits<T>;
    using U = typename B::U;
    if (!(x > T(0))) return (x == T(0)) ? T(1) / x : (x - x) / (x - x);
    T scale = T(1);
    U u = to_bits<U>(x);
    int eb = int((u >> B::mbits) & B::emask);
    if (eb == int(B::emask)) return T(0);                  // +inf
    if (eb == 0) {                                         // subnormal: x * 2^48, result * 2^16
        x = x * bits_to<T>(U(B::bias + 48) << B::mbits);
        scale = bits_to<T>(U(B::bias + 16) << B::mbits);
        u = to_bits<U>(x);
        eb = int((u >> B::mbits) & B::emask);
    }
    const int e = eb - B::bias;
    const T f = bits_to<T>((u & ((U(1) << B::mbits) - 1)) | (U(B::bias) << B::mbits));
    const int q = (e >= 0) ? e / 3 : -((2 - e) / 3);       // floor(e / 3)
    const int r = e - 3 * q;
    const T w = f * (r == 0 ? T(1) : (r == 1 ? T(2) : T(4)));
    const T c = (r == 0 ? T(1) : (r == 1 ? T(0.7937005259840998) : T(0.6299605249474366)));
    T y = (T(1.53701885) + f * (T(-0.801366717) + f * (T(0.312967226) + f * T(-0.0490997445)))) * c;
#pragma unroll
    for (int it = 0; it < B::newton; ++it) {
        const T y3 = y * y * y;
        y = y + y * (T(1) - w * y3) * T(1.0 / 3.0);
    }
    return y * bits_to<T>(U(B::bias - q) << B::mbits) * scale;
}

}  // namespace zb
