// Minimal AMReX API shim: amrex::Vector (host-side std::vector).
#pragma once
#include <vector>
namespace amrex { template <class T> using Vector = std::vector<T>; }
