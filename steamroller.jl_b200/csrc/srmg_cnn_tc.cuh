// srmg_cnn_tc.cuh -- the warm-start network's inference forward pass on the 5th-generation
// tensor cores (tcgen05): one CTA per SM streams samples; per layer one thread issues
// M=128 x N=32 x K=16 BF16 MMAs whose FP32 accumulators live in tensor memory (TMEM),
// and 8 warps read them back (tcgen05.ld) for the bias + ReLU epilogue.
//
// Implicit GEMM per layer: rows = output pixels, columns = output channels, K = 9 taps
// x input channels.  The 20 x 20 tile is laid out with rows of 24 pixels (the 4 extra
// columns and a 1-pixel ring are zero), output row q = y * 24 + x, q < 480 (4 M-tiles
// of 128).  A tap (dy, dx) reads input row q + (dy + 1) * 24 of the copy shifted by dx:
// three copies of the layer input, shifted by dx = -1, 0, +1, so that every A operand
// starts on an 8-row boundary.  Copies and weights use the canonical K-major layout
// without swizzle: core matrices of 8 rows x 16 bytes (8 channels) contiguous, the 4
// channel chunks of an 8-row group 128 bytes apart (leading byte offset), 8-row groups
// 512 bytes apart (stride byte offset).
//
// Every shared-memory operand stays inside its buffer: the largest A read (M-tile 3,
// dy = +1) covers row groups 54..69 of the 70 of a copy; B reads one tap's 2048-byte
// block; D uses TMEM columns mt * 32 + [0, 32) of the 128 allocated.  The MMA completion
// wait is bounded; on a timeout the kernel sets *err, frees its TMEM and returns.
//
// Measured against the mma.sync forward (k_cnn_fwd) on one B200 it is correct to the
// same tolerance but slower (0.92 vs 0.70 ms per 4096 samples).  It is latency-bound:
// one sample per CTA is in flight, and per layer the MMAs, their commit and wait, and
// the TMEM epilogue that writes the next layer's operands run one after another (tensor
// pipe 9.6% active, 8 warps, long-scoreboard stalls leading).  Overlapping two samples
// or two layers needs a second set of operand copies, which the 219 KB of copies and
// weights leave no room for.  It is therefore an opt-in path (srmg_cnn_use_tcgen05).

constexpr int kTcW = 24;                     // padded row length (a multiple of 8)
constexpr int kTcRows = 560;                 // rows per shifted copy: 512 + 2 * 24
constexpr int kTcCopyBytes = kTcRows / 8 * 512;
constexpr int kTcThreads = 256;
constexpr int kTcWBytes = kL * 9 * 2048;     // packed weights, all layers

struct TcSmem {
  alignas(128) unsigned char cp[3][kTcCopyBytes];  // the layer input, shifted by dx = -1, 0, +1
  alignas(128) unsigned char w[kTcWBytes];         // weights [layer][tap]: 32 rows (co) x 4 chunks (ci)
  float bias[kL][kC];
  alignas(8) uint64_t mbar;
  uint32_t tmem;
};

// Byte offset of (row r, 16-byte channel chunk c) in the canonical no-swizzle layout.
__host__ __device__ __forceinline__ int cm_off(int r, int c) { return (r >> 3) * 512 + c * 128 + (r & 7) * 16; }

__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(512 >> 4) << 32) |
         (1ull << 46);
}

// kind::f16 instruction descriptor: FP32 accumulate, BF16 A and B, both K-major, M = 128.
__host__ __device__ constexpr uint32_t tc_idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t *mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_addr(mbar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// TMEM load of 16 columns without the wait (the values are valid after tc_ld_wait).
__device__ __forceinline__ void tc_ld16_issue(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
// Wait for the thread's TMEM loads; the registers pass through so that no use of them
// is scheduled before the wait.
__device__ __forceinline__ void tc_ld_wait(uint32_t (&r)[16]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                 "+r"(r[15])
               :
               : "memory");
}

__device__ __forceinline__ void tc_mbar_init(uint64_t *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool tc_mbar_wait(uint64_t *bar, uint32_t parity, long long timeout_ns) {
  long long t0;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  while (true) {
    uint32_t ok;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
    long long t1;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
    if (t1 - t0 > timeout_ns) return false;
  }
}

// Write 16 channels (two 16-byte chunks, starting at chunk c0) of tile pixel (y, x) into
// the three shifted copies; pixels outside the 20 x 20 tile are never written, so the
// copies' ring and padding stay zero.
__device__ __forceinline__ void tc_put(TcSmem &S, int y, int x, int c0, uint4 lo, uint4 hi) {
  for (int d = 0; d < 3; ++d) {   // copy d holds the input shifted by dx = d - 1
    const int xc = x - (d - 1);
    if (xc < 0 || xc >= kTcW) continue;
    const int r = (y + 1) * kTcW + xc;
    *reinterpret_cast<uint4 *>(S.cp[d] + cm_off(r, c0)) = lo;
    *reinterpret_cast<uint4 *>(S.cp[d] + cm_off(r, c0 + 1)) = hi;
  }
}

__global__ void __launch_bounds__(kTcThreads, 1)
k_cnn_fwd_tc(const __nv_bfloat16 *__restrict__ x, int n, const unsigned char *__restrict__ wtc,
             const float *__restrict__ bias, float *__restrict__ yout, int *__restrict__ err,
             const int *__restrict__ n_dev) {
  extern __shared__ __align__(128) unsigned char smraw[];
  TcSmem &S = *reinterpret_cast<TcSmem *>(smraw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (n_dev) n = min(n, *n_dev);
  {
    uint4 *c = reinterpret_cast<uint4 *>(S.cp[0]);
    for (int i = tid; i < 3 * kTcCopyBytes / 16; i += blockDim.x) c[i] = make_uint4(0, 0, 0, 0);
    const uint4 *src = reinterpret_cast<const uint4 *>(wtc);
    uint4 *dst = reinterpret_cast<uint4 *>(S.w);
    for (int i = tid; i < kTcWBytes / 16; i += blockDim.x) dst[i] = src[i];
    for (int i = tid; i < kL * kC; i += blockDim.x) S.bias[i / kC][i % kC] = bias[i];
    if (tid == 0) tc_mbar_init(&S.mbar);
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&S.tmem)),
                 "r"(128)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem;
  const uint32_t cp_s = smem_addr(S.cp[0]), w_s = smem_addr(S.w);
  // epilogue role: TMEM lane quarter (rows) and column half (channels 0-15 / 16-31)
  const int quarter = warp & 3, chalf = warp >> 2;
  uint32_t phase = 0;
  bool ok = true;
  for (int s = blockIdx.x; s < n && ok; s += gridDim.x) {
    // the sample's input: channels 0, 1 = (f a, g c), channels 2..15 zero
    for (int p = tid; p < kNP; p += blockDim.x) {
      const __nv_bfloat162 v = reinterpret_cast<const __nv_bfloat162 *>(x)[(int64_t)s * kNP + p];
      tc_put(S, p / kT, p % kT, 0, make_uint4(*reinterpret_cast<const uint32_t *>(&v), 0, 0, 0),
             make_uint4(0, 0, 0, 0));
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    for (int l = 0; l < kL && ok; ++l) {
      const bool last = l == kL - 1;
      const int nn = last ? 16 : 32;
      const int khalves = l == 0 ? 1 : 2;
      if (tid == 0) {
        tc_fence_after();
        const uint32_t idesc = tc_idesc(nn);
        // descriptors differ only in the start address (bits 0..13, in 16-byte units)
        const uint64_t a0 = tc_desc(cp_s), b0 = tc_desc(w_s + l * 9 * 2048);
        for (int mt = 0; mt < 4; ++mt) {
          uint32_t acc = 0;
#pragma unroll
          for (int tap = 0; tap < 9; ++tap) {
            const int dy = tap / 3, dxi = tap % 3;  // dy + 1 and dx + 1
            // first A row mt * 128 + dy * 24: a multiple of 8, row group (mt * 128 + dy * 24) / 8
            const uint32_t aoff = (uint32_t)(dxi * kTcCopyBytes + (mt * 16 + dy * 3) * 512) >> 4;
            const uint32_t boff = (uint32_t)(tap * 2048) >> 4;
            for (int kh = 0; kh < khalves; ++kh) {
              tc_mma(tmem + mt * 32, a0 + aoff + kh * 16, b0 + boff + kh * 16, idesc, acc);
              acc = 1;
            }
          }
        }
        tc_commit(&S.mbar);
      }
      // every thread waits for the layer's MMAs (bounded); the outcome is made uniform
      const bool done = tc_mbar_wait(&S.mbar, phase, 1000000000LL);
      ok = __syncthreads_and(done) != 0;
      if (!ok && tid == 0) atomicCAS(err, 0, 1);
      phase ^= 1;
      tc_fence_after();
      if (ok && !(last && chalf)) {
        // the four M-tiles' accumulators: all loads in flight, then one wait
        uint32_t rv[4][16];
#pragma unroll
        for (int mt = 0; mt < 4; ++mt)
          tc_ld16_issue(tmem + ((uint32_t)(quarter * 32) << 16) + mt * 32 + chalf * 16, rv[mt]);
#pragma unroll
        for (int mt = 0; mt < 4; ++mt) tc_ld_wait(rv[mt]);
#pragma unroll
        for (int mt = 0; mt < 4; ++mt) {
          float v[16];
          for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(rv[mt][i]);
          const int q = mt * 128 + quarter * 32 + lane;
          const int yy = q / kTcW, xx = q % kTcW;
          if (q >= 480 || xx >= kT) continue;
          if (!last) {
            uint32_t pk[8];
            for (int i = 0; i < 8; ++i) {
              const int c = chalf * 16 + 2 * i;
              pk[i] = pack_bf16(fmaxf(v[2 * i] + S.bias[l][c], 0.f), fmaxf(v[2 * i + 1] + S.bias[l][c + 1], 0.f));
            }
            tc_put(S, yy, xx, chalf * 2, make_uint4(pk[0], pk[1], pk[2], pk[3]),
                   make_uint4(pk[4], pk[5], pk[6], pk[7]));
          } else if (yy >= 2 && yy < 18 && xx >= 2 && xx < 18) {
            yout[(int64_t)s * 256 + (yy - 2) * 16 + (xx - 2)] = v[0] + S.bias[l][0];
          }
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      tc_fence_before();
      __syncthreads();
    }
  }
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128) : "memory");
}
