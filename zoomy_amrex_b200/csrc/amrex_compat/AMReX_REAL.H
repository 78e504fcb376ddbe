// Minimal AMReX API shim: the real type. amrex::Real is double, as in a
// default (USE_DOUBLE) AMReX build; every reference kernel computes in FP64.
#pragma once
namespace amrex { using Real = double; }
