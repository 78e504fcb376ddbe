// Portable, bit-reproducible elementary functions for model code.
//
// The Model:: functions run both in the CPU oracle (g++, -ffp-contract=off)
// and in the sm_100a kernels (nvcc --fmad=false). +,-,*,/ and sqrt are IEEE
// correctly rounded on both, so a model written only with those gives the
// same bits on both sides. pow/cbrt are not correctly rounded in either libm,
// and they differ between glibc and CUDA's libdevice, so the one non-algebraic
// power the shallow-water friction law needs, x^(1/3), is computed here from
// IEEE operations only: exact exponent reduction (frexp/ldexp) followed by a
// fixed number of Newton steps on y^3 = m. Same operation sequence => same
// bits on CPU and GPU.
#pragma once
#include <cmath>
#include "AMReX_Extension.H"

namespace zb {

// Cube root of x > 0 (returns 0 for x == 0, NaN for x < 0 or NaN).
// Method: x = m * 2^(3k), m in [1/16, 1/2); initial guess from a cubic
// least-squares fit of m^(1/3) on that interval (max relative error 1.7e-2),
// then 5 Newton iterations y <- y - (y^3 - m) / (3 y^2), which square the
// relative error each time (1.7e-2 -> 3e-4 -> 8e-8 -> 7e-15 -> round-off).
template <class T>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE T cbrt_pos(T x)
{
    if (!(x > T(0))) return (x == T(0)) ? T(0) : (x - x) / (x - x);   // 0, or NaN
    int e = 0;
    T m = std::frexp(x, &e);                 // x = m * 2^e, m in [0.5, 1)
    int r = e % 3; if (r < 0) r += 3;        // e = 3k + r with r in {0,1,2}
    int k = (e - r) / 3;
    // fold the remainder into the mantissa: m' = m * 2^(r-3) in [1/16, 1/2)
    m = std::ldexp(m, r - 3);
    k += 1;
    T y = T(0.286315) + m * (T(2.088355) + m * (T(-3.527888) + m * T(2.785641)));
    for (int it = 0; it < 5; ++it) {
        T y2 = y * y;
        y = y - (y2 * y - m) / (T(3) * y2);
    }
    return std::ldexp(y, k);
}

}  // namespace zb
