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
  int4 *cfaces = nullptr;  // BoxStencil trees: 4 corner faces per block, else null
  LevelView view(int level) const { return LevelView{blocks, faces, child, nblk, nch, level, cfaces}; }
};

// Per-level device view of a three-dimensional tree (srmg_set_tree3): blocks
// {blk, c1, c2, c3}, child-octant masks, 27 pull faces per block by ghost direction
// (f1+1) + 3(f2+1) + 9(f3+1), child edges {fine, coarse, packed subblock}.
struct Level3View {
  const int4 *blocks;
  const int *mask;
  const int4 *faces;
  const int4 *child;
  int nblk;
  int nch;
};

struct Dev3Level {
  int nblk = 0;
  int nch = 0;
  int4 *blocks = nullptr;
  int *mask = nullptr;
  int4 *faces = nullptr;
  int4 *child = nullptr;
  Level3View view() const { return Level3View{blocks, mask, faces, child, nblk, nch}; }
};

// A device buffer that only grows.
struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
};

// Operator of one item (an independent problem of the context's forest).
struct ItemSpec {
  double s = 1.0;
  int op = 0;
  double k2 = 0.0;
  int8_t bc[9] = {1, 1, 1, 1, 1, 1, 1, 1, 1};
};

// Host copy of an uploaded tree (the arrays srmg_set_tree received), kept so that
// forests can be assembled from the trees of other contexts.
struct HostTree {
  int nlev = 0;
  int64_t max_blk = 0;
  std::vector<std::vector<srmg_pair>> pairs;
  std::vector<std::vector<srmg_neighbor>> nb;
  std::vector<std::vector<srmg_boundary>> bd;
  std::vector<std::vector<srmg_refbnd>> rb;
  std::vector<std::vector<srmg_child>> ch;
};

}  // namespace srmg

struct srmg_ctx {
  int device = 0;
  int D = 2;                 // dimension of the tree: 2, or 3 (per-operation FP64 path only)
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
  std::vector<srmg::Dev3Level> lv3;    // D = 3 trees, index l-1
  std::vector<int> nblk_host;          // per level
  std::vector<int> nch_host;
  void *d_tree = nullptr;              // one allocation for all tree arrays
  int2 *d_coord_of = nullptr;          // [max_blk] coords by 0-based block id
  double *d_wm64 = nullptr, *d_wp64 = nullptr;
  float *d_wm32 = nullptr, *d_wp32 = nullptr;
  double *d_wrow64 = nullptr;  // the weight tables as rows per block coordinate (2 x 20 values)
  float *d_wrow32 = nullptr;
  // block-id-indexed tables for the persistent engine
  int4 *d_info = nullptr;    // {coord_r, coord_z, child_mask, level}
  int4 *d_faceb = nullptr;   // [blk*4+f] {type, src, sb_r | sb_z << 8, push_to}
  int4 *d_kids = nullptr;    // child block per subblock, -1 if none

  // persistent engine
  srmg::DevBuf sync;         // {barrier counter, error word}
  int num_sms = 0;
  int engine_ctas = 0;       // cooperative grid size (0 = not yet known)
  int engine_threads = 0;    // threads per CTA of the persistent kernel: 768 or 1024 (0 = by tree size)
  int local_max_blocks = 4;  // levels whose every coarser level has <= this many blocks run in CTA 0
                             // (4 measured fastest on the 1.5M- and 10M-leaf trees)
  bool use_engine = true;
  unsigned refbnd_levels = 0;  // bit l: level l has refinement-boundary faces
  bool has_corners = false;    // the tree came with a BoxStencil connectivity (diagonal edges)
  bool merge_fill = true;      // 3D: copy and boundary fill passes may share a launch
  // 2D per-operation Gauss-Seidel: colour sweeps that write their own copy and boundary
  // ghosts (ensure_gs_push).  push_state 0 = tables not built for this tree, 1 = built,
  // -1 = not used on this tree.
  bool use_gs_push = true;
  int push_state = 0;
  bool push_ok2 = false, push_ok4 = false;  // race-free for red-black / four-colour sweeps
  srmg::DevBuf push_tab;
  std::vector<srmg::PushView> push_lv;      // per level, index l-1
  bool trace_on = false;
  srmg::DevBuf trace;        // %globaltimer stamps after every engine phase (CTA 0)

  // device mirrors of host fields (host-pointer entry points) and solver work buffers
  srmg::DevBuf f64[6];   // u, b, r, u1, bwork, spare
  srmg::DevBuf f32[6];   // FP32 work fields for the mixed solve
  srmg::DevBuf part;     // norm partials
  srmg::DevBuf small;    // small device scalars
  double *h_small = nullptr;  // pinned host mirror of `small`
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;

  // items: independent problems of one forest (a plain tree is one item)
  srmg::HostTree htree;
  int nitems = 1;
  int geom_forest = -1;                 // geometry fixed by srmg_batch_set (-1: any)
  std::vector<int64_t> item_first;      // per item: first 0-based block id of its range
  std::vector<int64_t> item_nblk;       // per item: blocks of its range
  std::vector<int2> it_lrange_host;     // [item * nlev + l - 1] {first, count} in level l's list
  int2 *d_it_lrange = nullptr;          // device copy (inside d_tree)
  int4 *d_chunks = nullptr;             // norm chunks {level, first, count, item} (inside d_tree)
  int2 *d_it_chunks = nullptr;          // per item: {first chunk, chunks}
  int nchunk = 0;
  int2 *d_leaf = nullptr;               // blocks with a leaf cell: {0-based id, level}
  int nleaf = 0;
  srmg::DevBuf cnn_work[3];             // learned warm start: db, candidate guess, samples
  int cnn_active_ppm = 0;               // > 0: network only on blocks with g energy >= ppm 1e-6 x max
  int cnn_last_active = 0;              // active blocks of the last prediction (when read back)
  std::vector<int4> l1_blocks, l1_faces;  // level 1 as uploaded (direct coarsest solve)
  std::vector<int4> l2_blocks, l2_faces;  // level 2 as uploaded (a lone tree's direct solve there)
  int direct_level = 0;                   // option "direct_level": 0 = 2 where possible, 1 or 2
  std::vector<srmg::ItemSpec> batch_items;       // operators given to srmg_batch_set

  // per-item operator tables of the persistent engine
  srmg::DevBuf it_tab;
  std::vector<char> it_tab_host;        // what it_tab holds
  // per-item results of the device loop, and their pinned host mirror
  srmg::DevBuf istat;
  double *h_items = nullptr;
  size_t h_items_n = 0;

  // batched solves: forest-layout fields (u, b) and the captured step sequence
  srmg::DevBuf forest[2];
  cudaGraphExec_t graph_exec = nullptr;
  std::vector<const void *> graph_key;  // field pointers and options the graph was captured for
  bool use_graph = false;
  // per-operation V-cycles replayed from captured graphs, by (fields, operator, sweep
  // counts, tree, stream); at most kOpGraphs kept, the oldest replaced first
  struct OpGraph {
    std::vector<char> key;
    cudaGraphExec_t exec = nullptr;
    int64_t launches = 0;
  };
  std::vector<OpGraph> op_graphs;
  bool use_op_graphs = true;
  // the same V-cycles as one cooperative launch of the sequencer (srmg_seq.cu): the
  // recorded operations by key, at most kOpGraphs kept; while seq_rec is set the
  // per-operation launchers append records (SeqOp<double>) to it instead of launching
  struct OpSeq {
    std::vector<char> key;
    srmg::DevBuf ops;
    int nops = 0;
  };
  std::vector<OpSeq> op_seqs;
  bool use_op_seq = false;
  std::vector<char> *seq_rec = nullptr;

  // free boundary conditions (srmg_freebc_set): f [n], sin table [4n], work [n], b [n]
  srmg::DevBuf fbc;
  int64_t fbc_n = 0;
  int fbc_dim = 0, fbc_level = 0;
  int64_t fbc_root[2] = {1, 1};
  bool fbc_direct = false;  // option "freebc_direct": direct-sum transforms even for power-of-two n
  // per-tree tables of srmg_freebc_dev (the outer-column gather, the level views and the
  // outer blocks), built on first use after srmg_freebc_set or a new tree
  srmg::DevBuf fbc_tabs;
  bool fbc_built = false;
  int fbc_nent = 0;
  size_t fbc_off_lvs = 0, fbc_off_ent = 0;

  // host-array entry points: b copied back to the host (off by default: leaf cells of b
  // are never written, and non-leaf b is unspecified after a V-cycle), and the host
  // ranges page-locked through srmg_host_register {address, bytes}
  bool b_copy_back = false;
  bool async_pending = false;  // srmg_solve_async enqueued a solve that srmg_solve_wait has not finished
  std::vector<std::pair<void *, size_t>> host_reg;

  // coarsest-level direct inverses, by operator and level-1 structure
  std::map<std::vector<double>, srmg::DevBuf> coarse_cache;
};
