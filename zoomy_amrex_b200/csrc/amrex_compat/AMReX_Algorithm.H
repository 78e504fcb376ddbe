// Minimal AMReX API shim: amrex::max / amrex::min with AMReX's semantics
// ((a < b) ? b : a and (a < b) ? a : b), so NaN propagation matches.
#pragma once
#include "AMReX_Extension.H"
namespace amrex {
template <class T>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr const T& max(const T& a, const T& b) noexcept
{ return (a < b) ? b : a; }
template <class T>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr const T& min(const T& a, const T& b) noexcept
{ return (b < a) ? b : a; }
}
