// Minimal AMReX API shim: host/device qualifier macros.
// Lets code written against the AMReX device-function interface (the
// Model::/Numerics:: headers emitted by zoomy-amrex's printer, and make_rhs.H)
// compile with nvcc for sm_100a and with g++ for the CPU oracle, without AMReX.
#pragma once
#if defined(__CUDACC__)
#  define AMREX_GPU_DEVICE __device__
#  define AMREX_GPU_HOST __host__
#  define AMREX_GPU_HOST_DEVICE __host__ __device__
#else
#  define AMREX_GPU_DEVICE
#  define AMREX_GPU_HOST
#  define AMREX_GPU_HOST_DEVICE
#endif
