// srmg_ctx.h -- the context behind the C ABI: device copy of the tree, device mirrors
// of host fields, scratch and error state.
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include <map>
#include <cuda_runtime.h>

#include "srmg_kernels.cuh"
#include "../../include/srmg.h"

namespace srmg {

struct DevLevel {
  int nblk = 0;     // blocks of this level
  int nch = 0;      // Child edges whose fine block is on this level
  int4 *blocks = nullptr;
  int4 *faces = nullptr;
  int4 *child = nullptr;
  int4 *rec = nullptr;   // engine records: 5 int4 per block ({blk, cr, cz, child_mask}, face 0..3)
  LevelView view(int level) const { return LevelView{blocks, faces, child, nblk, nch, level}; }
};

// A device buffer that only grows.
struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
};

}  // namespace srmg

struct srmg_ctx {
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  std::string err;
  int64_t launches = 0;

  // tree
  bool has_tree = false;
  uint64_t generation = 0;
  int nlev = 0;
  int64_t max_blk = 0;      // largest 1-based block id in the tree
  int wtab_n = 0;           // entries of the radial weight tables
  std::vector<srmg::DevLevel> lv;      // index l-1
  std::vector<int> nblk_host;          // per level
  std::vector<int> nch_host;
  void *d_tree = nullptr;              // one allocation for all tree arrays
  int2 *d_coord_of = nullptr;          // [max_blk] coords by 0-based block id
  double *d_wm64 = nullptr, *d_wp64 = nullptr;
  float *d_wm32 = nullptr, *d_wp32 = nullptr;
  // block-id-indexed tables for the persistent engine
  int4 *d_info = nullptr;    // {coord_r, coord_z, child_mask, level}
  int4 *d_faceb = nullptr;   // [blk*4+f] {type, src, sb_r | sb_z << 8, push_to}
  int4 *d_kids = nullptr;    // child block per subblock, -1 if none

  // persistent engine
  srmg::DevBuf sync;         // {barrier counter, error word}
  int num_sms = 0;
  int engine_ctas = 0;       // cooperative grid size (0 = not yet known)
  int local_max_blocks = 16; // levels whose every coarser level has <= this many blocks run in CTA 0
  bool use_engine = true;
  unsigned refbnd_levels = 0;  // bit l: level l has refinement-boundary faces
  bool trace_on = false;
  srmg::DevBuf trace;        // %globaltimer stamps after every engine phase (CTA 0)

  // device mirrors of host fields (host-pointer entry points) and solver work buffers
  srmg::DevBuf f64[6];   // u, b, r, u1, bwork, spare
  srmg::DevBuf f32[6];   // FP32 work fields for the mixed solve
  srmg::DevBuf part;     // norm partials
  srmg::DevBuf small;    // small device scalars
  double *h_small = nullptr;  // pinned host mirror of `small`
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;

  // coarsest-level direct solver cache (mixed mode)
  srmg::DevBuf coarse_inv;
  std::vector<double> coarse_key;
  int coarse_n = 0;
  bool coarse_ok = false;
};
