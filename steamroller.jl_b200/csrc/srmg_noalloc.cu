// srmg_noalloc.cu -- srmg_resnorm_noalloc: the residual norm with no device allocation.
//
// Who needs it: callers that must not call cudaMalloc at the moment they compute a
// norm -- hosts whose device memory is owned by their own pool allocator (a Julia GPU
// array pool, a framework arena) and which forbid other allocations, and
// latency-critical loops that cannot afford an allocation's implicit synchronisation.
// srmg_resnorm_dev may grow its partial-sum buffer with cudaMalloc; this entry point
// never does.  2D trees only (check_call refuses D = 3 with SRMG_ERR_UNSUPPORTED).
//
// Its scratch is a file-scope __device__ array holding one partial sum per tree block,
// so the tree may hold at most kNoAllocMaxBlocks blocks.  Every GPU that loads the
// library holds this array (512 KiB) until the process exits.
#include <mutex>

#include "srmg_ctx.h"
#include "srmg_internal.h"

using namespace srmg;

namespace {

constexpr int kNoAllocMaxBlocks = 1 << 16;  // 65536 blocks -> 512 KiB of doubles

// One partial per block: every call overwrites the slots of the tree's blocks before
// the final reduction reads them, so nothing has to be cleared between calls.
static __device__ __align__(256) double g_noalloc_parts[kNoAllocMaxBlocks];

// Host code may not use g_noalloc_parts as an address: on the host it only names a
// stand-in.  The device address is looked up once per device with that device
// current, and cached here for the life of the process: the cache assumes that the
// device's primary context (which holds the array) lives as long as the process.  A
// caller that resets the device (cudaDeviceReset) and keeps using the library would
// pass a stale address; such a caller must not use this entry point after the reset.
constexpr int kMaxDevices = 64;
double *g_parts_addr[kMaxDevices] = {nullptr};
std::mutex g_parts_mu;

int parts_address(srmg_ctx *ctx, double **out) {
  const int dev = ctx->device;
  if (dev < 0 || dev >= kMaxDevices) return fail(ctx, SRMG_ERR_BADARG, "device %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_parts_mu);
  if (!g_parts_addr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_parts);
    if (e != cudaSuccess)
      return fail(ctx, SRMG_ERR_CUDA, "cudaGetSymbolAddress(g_noalloc_parts): %s", cudaGetErrorString(e));
    g_parts_addr[dev] = (double *)p;
  }
  *out = g_parts_addr[dev];
  return SRMG_OK;
}

// Weighted leaf sum of squares of the residual of one block per CTA.
template <int NT>
__global__ void __launch_bounds__(NT) k_leafsq_per_block(double *__restrict__ part,
                                                         const double *__restrict__ u,
                                                         const double *__restrict__ b, LevelView lv,
                                                         OpParams<double> p, WTab<double> wt,
                                                         double wl) {
  const int bi = blockIdx.x;
  const int4 bk = lv.blocks[bi];
  const int64_t base = (int64_t)bk.x * kSS;
  double acc = 0.0;
  for (int c = threadIdx.x; c < 256; c += NT) {
    const int x = 2 + (c & 15), y = 2 + (c >> 4);
    const int sub = ((x - 2) >> 3) + 2 * ((y - 2) >> 3);
    if ((bk.w >> sub) & 1) continue;
    const double Lu = lhs_apply<double>(u + base, x, y, p, wt, bk.y, bk.z);
    const int64_t o = base + x + kS * y;
    const double r = -(b[o] + Lu / p.s);
    acc = fma(r, r, acc);
  }
  __shared__ double sh[NT / 32];
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = (threadIdx.x < NT / 32) ? sh[threadIdx.x] : 0.0;
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if (threadIdx.x == 0) part[bi] = v * wl;
  }
}

}  // namespace

// See include/srmg.h.  All launches go to the context's stream; the result is written
// to the device address `out`; nothing is allocated and nothing is copied to the host.
extern "C" int srmg_resnorm_noalloc(srmg_ctx *ctx, const double *b, const double *u,
                                    int64_t nblk_alloc, double s, int op, double k2, int geom,
                                    double *out) {
  {
    const int rc = check_call(ctx, nblk_alloc, op, geom, nullptr);
    if (rc) return rc;
  }
  if (!b || !u || !out) return fail(ctx, SRMG_ERR_BADARG, "srmg_resnorm_noalloc: null argument");
  int64_t total = 0;
  for (int l = 1; l <= ctx->nlev; l++) total += ctx->nblk_host[l - 1];
  if (total > kNoAllocMaxBlocks)
    return fail(ctx, SRMG_ERR_BADARG,
                "srmg_resnorm_noalloc: the tree has %lld blocks; this entry point holds at most %d "
                "(use srmg_resnorm_dev)",
                (long long)total, kNoAllocMaxBlocks);
  double *parts = nullptr;
  {
    const int rc = parts_address(ctx, &parts);
    if (rc) return rc;
  }
  constexpr int NT = 256;
  int64_t off = 0;
  for (int l = 1; l <= ctx->nlev; l++) {
    const int n = ctx->nblk_host[l - 1];
    if (!n) continue;
    const OpParams<double> p = op_params<double>(op, geom, k2, level_scale(s, l), 1.0);
    const double wl = 1.0 / (double)((int64_t)1 << (2 * (l - 1)));
    k_leafsq_per_block<NT><<<n, NT, 0, ctx->stream>>>(parts + off, u, b, ctx->lv[l - 1].view(l), p,
                                                      WTab<double>{ctx->d_wm64, ctx->d_wp64}, wl);
    ctx->launches++;
    off += n;
  }
  if (total == 0) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double), ctx->stream);
    if (e != cudaSuccess) return fail(ctx, SRMG_ERR_CUDA, "cudaMemsetAsync: %s", cudaGetErrorString(e));
    return SRMG_OK;
  }
  k_reduce_sqrt<1024><<<1, 1024, 0, ctx->stream>>>(out, parts, (int)total);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(ctx, SRMG_ERR_CUDA, "srmg_resnorm_noalloc launch: %s", cudaGetErrorString(e));
  return SRMG_OK;
}
