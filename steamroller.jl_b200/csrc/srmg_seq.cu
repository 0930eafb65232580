// srmg_seq.cu -- the sequencer: a recorded per-operation V-cycle (srmg_seq.cuh) as one
// cooperative launch.
//
// The V-cycles that cannot use the persistent engine (order-4 stencils, BoxStencil
// trees with corner ghosts, the engine switched off) are several hundred small
// dependent operations per cycle: GS colours, ghost-fill passes, residuals,
// restrictions, prolongations.  Launched one by one (or replayed from a CUDA graph)
// each costs a kernel launch of ~7 us for a few microseconds of work.  The sequencer
// runs the same operations, the same grid-stride bodies, inside one launch: a record
// per operation, a grid barrier (release/acquire on a counter, bounded wait) between
// consecutive records.  The barrier orders the operations and makes each one's writes
// visible to the next as two stream-ordered launches would, so the results are
// bit-identical to the launches they replace.
#include <algorithm>
#include <cstring>

#include "srmg_ctx.h"
#include "srmg_engine.cuh"
#include "srmg_internal.h"
#include "srmg_seq.cuh"

using namespace srmg;

#define CK(call)                                              \
  do {                                                        \
    int _rc = cuda_check(ctx, (call), #call);                 \
    if (_rc) return _rc;                                      \
  } while (0)
#define RC(call)               \
  do {                         \
    int _rc = (call);          \
    if (_rc) return _rc;       \
  } while (0)

namespace {

constexpr int kSeqThreads = 512;
constexpr int kSeqPerSM = 1;  // resident CTAs per SM

template <typename T>
__global__ void __launch_bounds__(kSeqThreads, kSeqPerSM)
    k_sequencer(const SeqOp<T> *__restrict__ ops, int nops, WTab<T> wt, const int2 *__restrict__ coord_of,
                unsigned *bar, int *err, long long timeout_ns) {
  unsigned epoch = 0;
  for (int i = 0; i < nops; ++i) {
    const SeqOp<T> &op = ops[i];
    switch (op.kind) {
      case SEQ_FILL: d_fill_ghost<T>(op.a, op.lv, op.sg, op.i0); break;
      case SEQ_GS_COLOUR: d_gs_colour<T>(op.a, op.b, op.lv, op.p, wt, op.i0); break;
      case SEQ_GS4: d_gs4<T>(op.a, op.b, op.lv, op.p, op.i0, op.i1); break;
      case SEQ_RESIDUAL: d_residual<T>(op.a, op.b, op.c, op.lv, op.p, wt); break;
      case SEQ_POSTRESTRICT: d_postrestrict<T>(op.a, op.b, op.c, op.lv, coord_of, op.p, wt); break;
      case SEQ_RESTRICT: d_restrict<T>(op.a, op.lv); break;
      case SEQ_INTERP_ADD: d_interp_add<T>(op.a, op.b, op.lv); break;
      case SEQ_COPY: d_copy_level<T>(op.a, op.b, op.lv); break;
      case SEQ_DIFF: d_diff_level<T>(op.a, op.b, op.c, op.lv); break;
      default:
        if (threadIdx.x == 0) atomicCAS(err, 0, 4);
        return;
    }
    if (i + 1 < nops && !grid_barrier(bar, err, epoch, timeout_ns)) return;
  }
}

// Self-test of the barrier's failure path: every CTA but `absent` enters one grid
// barrier; the absent CTA returns at once, so the others' bounded wait runs out, the
// first to give up records error 1 and all of them return.
__global__ void k_barrier_selftest(unsigned *bar, int *err, long long timeout_ns, int absent) {
  if ((int)blockIdx.x == absent) return;
  unsigned epoch = 0;
  grid_barrier(bar, err, epoch, timeout_ns);
}

}  // namespace

extern "C" int srmg_selftest_barrier_timeout(srmg_ctx *ctx, int timeout_ms) {
  if (!ctx || timeout_ms < 1 || timeout_ms > 2000) return SRMG_ERR_BADARG;
  cudaSetDevice(ctx->device);
  if (ctx->num_sms == 0) CK(cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, ctx->device));
  RC(ensure(ctx, ctx->sync, 256 + sizeof(int) * (size_t)std::max(ctx->nitems, 1)));
  CK(cudaMemsetAsync(ctx->sync.p, 0, 256, ctx->stream));
  unsigned *bar = (unsigned *)ctx->sync.p;
  int *err = (int *)((char *)ctx->sync.p + 128);
  long long timeout = (long long)timeout_ms * 1000000LL;
  int absent = 0;
  void *args[] = {&bar, &err, &timeout, &absent};
  CK(cudaLaunchCooperativeKernel((const void *)k_barrier_selftest, dim3(ctx->num_sms), dim3(128), args, 0,
                                 ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  const int rc = engine_check(ctx);  // SRMG_ERR_TIMEOUT when the wait ran out
  // leave the barrier state clean for the next launch
  CK(cudaMemsetAsync(ctx->sync.p, 0, 256, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return rc;
}

// One launch of the sequencer over `nops` records at d_ops (device memory), on the
// context's stream.  The barrier counter and error word are the persistent engine's
// (zeroed here, read by engine_check).
int srmg::seq_launch(srmg_ctx *ctx, const void *d_ops, int nops) {
  if (nops <= 0) return SRMG_OK;
  const void *fn = (const void *)k_sequencer<double>;
  if (ctx->num_sms == 0) CK(cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, ctx->device));
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kSeqThreads, 0));
  if (per_sm < 1) return fail(ctx, SRMG_ERR_CUDA, "sequencer kernel cannot be resident (occupancy 0)");
  const size_t sync_bytes = 256 + sizeof(int) * (size_t)ctx->nitems;
  RC(ensure(ctx, ctx->sync, sync_bytes));
  CK(cudaMemsetAsync(ctx->sync.p, 0, 256, ctx->stream));
  const SeqOp<double> *ops = (const SeqOp<double> *)d_ops;
  WTab<double> wt{ctx->d_wm64, ctx->d_wp64};
  const int2 *coord_of = ctx->d_coord_of;
  unsigned *bar = (unsigned *)ctx->sync.p;
  int *err = (int *)((char *)ctx->sync.p + 128);
  long long timeout = 2000000000LL;  // 2 s per barrier wait
  void *args[] = {&ops, &nops, &wt, &coord_of, &bar, &err, &timeout};
  CK(cudaLaunchCooperativeKernel(fn, dim3(ctx->num_sms * std::min(per_sm, kSeqPerSM)), dim3(kSeqThreads), args, 0, ctx->stream));
  ctx->launches++;
  return SRMG_OK;
}

size_t srmg::seq_op_bytes() { return sizeof(SeqOp<double>); }
