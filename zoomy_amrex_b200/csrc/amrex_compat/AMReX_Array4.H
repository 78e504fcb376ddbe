// Minimal AMReX API shim: amrex::Array4, the non-owning (i,j,k,n) view over
// a component-major box of data. Index = (i-lo.x) + (j-lo.y)*jstride
// + (k-lo.z)*kstride + n*nstride, as in AMReX.
#pragma once
#include "AMReX_REAL.H"
#include "AMReX_Extension.H"
#include "AMReX_SmallMatrix.H"
#include <type_traits>
namespace amrex {
struct Dim3 { int x, y, z; };
template <class T>
struct Array4
{
    T* p = nullptr;
    long long jstride = 0, kstride = 0, nstride = 0;
    Dim3 begin{0, 0, 0};
    Dim3 end{1, 1, 1};
    int ncomp = 1;

    constexpr Array4() = default;
    AMREX_GPU_HOST_DEVICE constexpr
    Array4(T* a_p, Dim3 a_begin, Dim3 a_end, int a_ncomp) noexcept
        : p(a_p),
          jstride(a_end.x - a_begin.x),
          kstride(jstride * (long long)(a_end.y - a_begin.y)),
          nstride(kstride * (long long)(a_end.z - a_begin.z)),
          begin(a_begin), end(a_end), ncomp(a_ncomp) {}
    template <class U, std::enable_if_t<std::is_same<const U, T>::value, int> = 0>
    AMREX_GPU_HOST_DEVICE constexpr Array4(Array4<U> const& rhs) noexcept
        : p(rhs.p), jstride(rhs.jstride), kstride(rhs.kstride), nstride(rhs.nstride),
          begin(rhs.begin), end(rhs.end), ncomp(rhs.ncomp) {}

    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE
    T& operator()(int i, int j, int k, int n) const noexcept {
        return p[(i - begin.x) + (j - begin.y) * jstride + (k - begin.z) * kstride + n * nstride];
    }
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE
    T& operator()(int i, int j, int k) const noexcept { return (*this)(i, j, k, 0); }
};
}
