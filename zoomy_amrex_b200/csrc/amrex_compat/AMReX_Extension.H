// Minimal AMReX API shim: inlining / restrict macros.
#pragma once
#include "AMReX_GpuQualifiers.H"
#if defined(__CUDACC__)
#  define AMREX_FORCE_INLINE __forceinline__
#else
#  define AMREX_FORCE_INLINE inline __attribute__((always_inline))
#endif
#define AMREX_INLINE inline
#define AMREX_RESTRICT __restrict__
