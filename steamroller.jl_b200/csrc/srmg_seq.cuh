// srmg_seq.cuh -- the operations of a per-operation V-cycle as records, so that the
// whole cycle runs in one cooperative launch (srmg_seq.cu) instead of one launch per
// operation.  A record names one of the grid-stride bodies of srmg_kernels.cuh and
// carries its arguments; the sequencer runs the records in order with a grid barrier
// between two records, which gives the same ordering and visibility as two launches on
// one stream, so the results are bit-identical to kernel-by-kernel launches.
#pragma once
#include "srmg_kernels.cuh"

namespace srmg {

enum SeqKind : int {
  SEQ_FILL = 1,        // d_fill_ghost(a, lv, sg, i0 = mask)
  SEQ_GS_COLOUR = 2,   // d_gs_colour(a, b, lv, p, wt, i0 = parity)
  SEQ_GS4 = 3,         // d_gs4(a, b, lv, p, i0, i1)
  SEQ_RESIDUAL = 4,    // d_residual(a, b, c, lv, p, wt)
  SEQ_POSTRESTRICT = 5,  // d_postrestrict(a, b, c, lv, coord_of, p, wt)
  SEQ_RESTRICT = 6,    // d_restrict(a, lv)
  SEQ_INTERP_ADD = 7,  // d_interp_add(a, b, lv)
  SEQ_COPY = 8,        // d_copy_level(a, b, lv)
  SEQ_DIFF = 9,        // d_diff_level(a, b, c, lv)
};

template <typename T>
struct SeqOp {
  int kind, i0, i1, pad;
  T *a;
  const T *b;
  const T *c;
  LevelView lv;
  OpParams<T> p;
  Signs sg;
};

}  // namespace srmg
