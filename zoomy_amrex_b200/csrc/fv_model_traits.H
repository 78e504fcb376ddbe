// Types and optional traits of a Model:: struct as the printer emits it
// (zoomy_amrex/transformation/to_amrex.py:348-361 gives the constants).
//
// The optional traits let a hand-written model declare facts that let the
// kernels move less data; a generated header does not define them and gets
// the conservative defaults:
//   zb_aux_pure   — update_aux_variables' output rows are either a function of
//                   Q (and p, time, X) alone or copies of the input aux rows,
//                   and no Model::/Numerics:: function reads a copied row.
//                   Then the kernels never load or store aux inside a step:
//                   they recompute it from Q where the reference reads it.
//   zb_static_bed — state row 0 (the bed) never changes in a step, so it is
//                   read but never written back.
//   zb_implicit_blocks, zb_implicit_block_size, zb_implicit_row(b, i) — the
//                   point-implicit system's structure: rows 0 and 1 (bed,
//                   depth) have a zero source and zero Jacobian rows, the
//                   other rows fall into blocks (row indices ascending within
//                   a block), and the Jacobian couples no two blocks. The FP64
//                   elimination then runs block by block with the reference's
//                   operations on every nonzero value (implicit_source_cell).
#pragma once
#include <type_traits>
#include "AMReX_SmallMatrix.H"

namespace zfv {

template <class Model>
struct ModelTypes {
    using R = double;
    using VQ = amrex::SmallMatrix<amrex::Real, Model::n_dof_q, 1>;
    using V2Q = amrex::SmallMatrix<amrex::Real, 2 * Model::n_dof_q, 1>;
    using VA = amrex::SmallMatrix<amrex::Real, Model::n_dof_qaux, 1>;
    using VP = amrex::SmallMatrix<amrex::Real, Model::n_parameters, 1>;
    using VN = amrex::SmallMatrix<amrex::Real, Model::dimension, 1>;
    using VX = amrex::SmallMatrix<amrex::Real, 3, 1>;
};

template <class M, class = void> struct aux_pure : std::false_type {};
template <class M> struct aux_pure<M, std::void_t<decltype(M::zb_aux_pure)>>
    : std::integral_constant<bool, M::zb_aux_pure> {};

template <class M, class = void> struct static_bed : std::false_type {};
template <class M> struct static_bed<M, std::void_t<decltype(M::zb_static_bed)>>
    : std::integral_constant<bool, M::zb_static_bed> {};

template <class M, class = void> struct implicit_blocks : std::false_type {};
template <class M> struct implicit_blocks<M, std::void_t<decltype(M::zb_implicit_blocks)>> : std::true_type {};

}  // namespace zfv
