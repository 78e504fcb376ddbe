// Minimal AMReX API shim: amrex::Math::powi, the integer power the printer
// emits for symbolic x**N. The multiplication tree (x^N = (x^(N/2))^2, times x
// for odd N) fixes the rounding, and the golden aux data pin it:
// powi<4>(h) must be (h*h)*(h*h), not ((h*h)*h)*h.
#pragma once
#include "AMReX_Extension.H"
namespace amrex { namespace Math {
template <int P, class T>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr T powi(T x) noexcept
{
    if constexpr (P < 0) { return T(1) / powi<-P>(x); }
    else if constexpr (P == 0) { return T(1); }
    else if constexpr (P == 1) { return x; }
    else if constexpr (P == 2) { return x * x; }
    else if constexpr (P % 2 == 0) { T y = powi<P / 2>(x); return y * y; }
    else { return x * powi<P - 1>(x); }
}
}}
