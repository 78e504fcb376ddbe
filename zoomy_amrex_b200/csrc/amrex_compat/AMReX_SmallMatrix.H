// Minimal AMReX API shim: amrex::SmallMatrix, the fixed-size column-major
// matrix the printer's Model::/Numerics:: functions take and return.
// Default construction leaves entries uninitialised (as AMReX does);
// `SmallMatrix<...> m{}` zero-fills them. All indexing is by compile-time
// bounds, so nvcc keeps every entry in registers once loops unroll.
#pragma once
#include "AMReX_REAL.H"
#include "AMReX_Extension.H"
#include "AMReX_Algorithm.H"
#include "AMReX_Math.H"
#include <initializer_list>
namespace amrex {
enum struct Order { C, F };
template <class T, int NRows, int NCols, Order ORDER = Order::F, int StartIndex = 0>
struct SmallMatrix
{
    static constexpr int row_size = NRows;
    static constexpr int column_size = NCols;
    using value_type = T;

    constexpr SmallMatrix() = default;

    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE
    const T& operator()(int i, int j) const noexcept {
        if constexpr (ORDER == Order::F) { return m_mat[(i - StartIndex) + (j - StartIndex) * NRows]; }
        else { return m_mat[(j - StartIndex) + (i - StartIndex) * NCols]; }
    }
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE
    T& operator()(int i, int j) noexcept {
        if constexpr (ORDER == Order::F) { return m_mat[(i - StartIndex) + (j - StartIndex) * NRows]; }
        else { return m_mat[(j - StartIndex) + (i - StartIndex) * NCols]; }
    }
    // Vector-style single index (column vectors are the common case).
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE
    const T& operator()(int i) const noexcept { return m_mat[i - StartIndex]; }
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE
    T& operator()(int i) noexcept { return m_mat[i - StartIndex]; }
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE
    const T& operator[](int i) const noexcept { return m_mat[i - StartIndex]; }
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE
    T& operator[](int i) noexcept { return m_mat[i - StartIndex]; }

    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE
    SmallMatrix& setVal(T v) noexcept {
        for (int k = 0; k < NRows * NCols; ++k) m_mat[k] = v;
        return *this;
    }
    // Size-0 matrices (a model with no aux rows) still need a valid array.
    T m_mat[(NRows * NCols) > 0 ? NRows * NCols : 1];
};
}
