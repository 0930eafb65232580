// srmg_cnn.cu -- the learned warm start: a small BF16 convolutional network that maps
// (previous potential, change of the right-hand side) on one block tile (16 x 16 cells
// plus the 2-cell ghost halo) to a guess of the new potential on the block's 16 x 16
// cells.  No reference counterpart: the reference starts every solve from the previous
// potential held in the field (src/streamer.jl:322-334).
//
// Network (per 20 x 20 tile, zero padding at the tile edge, ReLU after layers 1-5):
//   conv3x3  2 -> 32, conv3x3 32 -> 32 (x4), conv3x3 32 -> 1; output = centre 16 x 16.
// Parameters (FP32 master vector, layer by layer): W_l [9 taps][co][ci], then b_l [co].
// Every convolution is an implicit GEMM on the tensor cores (mma.sync m16n8k16, BF16
// operands, FP32 accumulation): M = 16 output pixels, N = 8 output channels, K = 16
// input channels of one tap.  Tiles live in shared memory with an 80-byte pixel pitch
// (conflict-free ldmatrix), weights with a 64-byte row pitch and an XOR swizzle of the
// 16-byte chunks.
//
// Training kernels: forward (storing every layer's activations), loss and output
// gradient, input gradient (the same convolution with the transposed, flipped
// weights, times the ReLU mask), weight gradient (per-CTA partial sums over pixels on
// the tensor cores, then a fixed-order reduction), and Adam.
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>

#include "srmg_ctx.h"
#include "srmg_internal.h"

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

namespace cnn {

constexpr int kL = 6;          // layers
constexpr int kC = 32;         // hidden channels
constexpr int kT = 20;         // tile side (16 cells + 2 ghosts each side)
constexpr int kTP = 22;        // padded tile side (1 zero pixel each side)
constexpr int kNP = kT * kT;   // pixels per tile
constexpr int kPP = 40;        // shared-memory pixel pitch (bf16): 80 bytes
constexpr int kTileElems = kTP * kTP * kPP;
constexpr int kWMat = kC * kC;           // one tap's 32 x 32 weight matrix (bf16)
constexpr int kWElems = kL * 9 * kWMat;  // packed weights of all layers
constexpr int kThreads = 512;            // 16 warps

__host__ __device__ constexpr int cin(int l) { return l == 0 ? 2 : kC; }
__host__ __device__ constexpr int cout(int l) { return l == kL - 1 ? 1 : kC; }

// Offsets of W_l and b_l in the FP32 master vector.
__host__ __device__ inline int woff(int l) {
  int o = 0;
  for (int k = 0; k < l; ++k) o += 9 * cout(k) * cin(k) + cout(k);
  return o;
}
__host__ __device__ inline int boff(int l) { return woff(l) + 9 * cout(l) * cin(l); }
constexpr int nparams() {
  int o = 0;
  for (int k = 0; k < kL; ++k) o += 9 * cout(k) * cin(k) + cout(k);
  return o;
}

// Byte offset of element (row r, column c) in a 32 x 32 bf16 matrix with 64-byte rows
// and the 16-byte chunks XOR-swizzled by (r / 2) % 4.
__host__ __device__ inline int swz(int r, int c) {
  return r * 64 + ((((c >> 3) ^ (r >> 1)) & 3) << 4) + (c & 7) * 2;
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void ldsm4(uint32_t a, uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3) : "r"(a));
}
__device__ __forceinline__ void ldsm4t(uint32_t a, uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3) : "r"(a));
}
__device__ __forceinline__ void ldsm2(uint32_t a, uint32_t &r0, uint32_t &r1) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];" : "=r"(r0), "=r"(r1) : "r"(a));
}
__device__ __forceinline__ void mma16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t *>(&v);
}

// Padded-tile offset (elements) of tile pixel p shifted by tap (dy, dx) = (tap/3-1, tap%3-1).
__device__ __forceinline__ int tap_pix(int p, int tap) {
  const int y = p / kT, x = p - kT * (p / kT);
  return (y + tap / 3) * kTP + (x + tap % 3);
}

// One 3x3 convolution over a tile held in `in` (padded, pitch kPP): for every output
// pixel p of the 20 x 20 tile and output channel co < 8 * ntiles,
//   acc[p][co] = sum_{tap, ci < 16 * khalves} in[p + off(tap)][ci] * W[tap][co][ci],
// W one 32 x 32 swizzled matrix per tap at `w` (flip: the tap order reversed).  The
// epilogue gets (pixel, co, value) pairs for the two channels a thread holds.
template <typename Epi>
__device__ __forceinline__ void conv_tile(const __nv_bfloat16 *in, const __nv_bfloat16 *w, int khalves, int ntiles,
                                          bool flip, const float *bias, Epi &&epi) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nw = blockDim.x >> 5;
  const int g = lane >> 2, t4 = lane & 3;
  const uint32_t in_s = smem_addr(in), w_s = smem_addr(w);
  for (int mt = warp; mt < kNP / 16; mt += nw) {
    const int p0 = mt * 16;
    float acc[4][4];
    for (int nt = 0; nt < 4; ++nt) {
      const float b0 = (bias && nt < ntiles) ? bias[nt * 8 + 2 * t4] : 0.f;
      const float b1 = (bias && nt < ntiles) ? bias[nt * 8 + 2 * t4 + 1] : 0.f;
      acc[nt][0] = b0;
      acc[nt][1] = b1;
      acc[nt][2] = b0;
      acc[nt][3] = b1;
    }
    // this lane's ldmatrix row: pixel p0 + (lane % 8) + 8 * ((lane / 8) % 2), chunk lane / 16
    const int arow = p0 + (lane & 7) + ((lane >> 3) & 1) * 8;
    const int achunk = lane >> 4;
    for (int tap = 0; tap < 9; ++tap) {
      const int wt = flip ? 8 - tap : tap;
      const uint32_t a_base = in_s + (uint32_t)(tap_pix(arow, tap) * kPP + achunk * 8) * 2;
      const uint32_t w_base = w_s + (uint32_t)(wt * kWMat) * 2;
      for (int kh = 0; kh < khalves; ++kh) {
        uint32_t a0, a1, a2, a3;
        ldsm4(a_base + kh * 32, a0, a1, a2, a3);
        if (ntiles == 1) {
          uint32_t b0, b1;
          // matrices: (co 0-7, ci kh*16 + 0-7), (co 0-7, ci kh*16 + 8-15)
          const int r = lane & 7, c = kh * 16 + ((lane >> 3) & 1) * 8;
          ldsm2(w_base + swz(r, c), b0, b1);
          mma16816(acc[0], a0, a1, a2, a3, b0, b1);
        } else {
          for (int np = 0; np < 4; np += 2) {
            uint32_t b0, b1, b2, b3;
            // matrices: (co np*8.., ci lo), (co np*8.., ci hi), (co (np+1)*8.., lo), (.., hi)
            const int r = (np + (lane >> 4)) * 8 + (lane & 7), c = kh * 16 + ((lane >> 3) & 1) * 8;
            ldsm4(w_base + swz(r, c), b0, b1, b2, b3);
            mma16816(acc[np], a0, a1, a2, a3, b0, b1);
            mma16816(acc[np + 1], a0, a1, a2, a3, b2, b3);
          }
        }
      }
    }
    for (int nt = 0; nt < ntiles; ++nt) {
      const int co = nt * 8 + 2 * t4;
      epi(p0 + g, co, acc[nt][0], acc[nt][1]);
      epi(p0 + g + 8, co, acc[nt][2], acc[nt][3]);
    }
  }
}

// Shared-memory layout of the forward / input-gradient kernels.
struct FwdSmem {
  __nv_bfloat16 w[kWElems];          // packed weights, all layers
  __nv_bfloat16 tile[2][kTileElems];  // ping-pong activation tiles
  float bias[kL][kC];
};

__device__ void zero_tile(__nv_bfloat16 *t) {
  uint4 *p = reinterpret_cast<uint4 *>(t);
  for (int i = threadIdx.x; i < kTileElems * 2 / 16; i += blockDim.x) p[i] = make_uint4(0, 0, 0, 0);
}

// Copy the 400 interior pixels (channels 0..31) of a padded tile to global [400][32].
__device__ void store_tile(const __nv_bfloat16 *t, __nv_bfloat16 *g) {
  for (int i = threadIdx.x; i < kNP * 4; i += blockDim.x) {
    const int p = i >> 2, c = (i & 3) * 8;
    const int y = p / kT, x = p % kT;
    const uint4 v = *reinterpret_cast<const uint4 *>(t + ((y + 1) * kTP + x + 1) * kPP + c);
    *reinterpret_cast<uint4 *>(g + p * kC + c) = v;
  }
}

// Load global [400][32] into the interior of a padded tile (the ring stays as it is).
__device__ void load_tile(__nv_bfloat16 *t, const __nv_bfloat16 *g) {
  for (int i = threadIdx.x; i < kNP * 4; i += blockDim.x) {
    const int p = i >> 2, c = (i & 3) * 8;
    const int y = p / kT, x = p % kT;
    *reinterpret_cast<uint4 *>(t + ((y + 1) * kTP + x + 1) * kPP + c) =
        *reinterpret_cast<const uint4 *>(g + p * kC + c);
  }
}

// Forward pass over n samples.  x: [n][400][2] bf16 (tile pixel order y * 20 + x).
// y: [n][16][16] FP32 output (the tile's centre).  acts (training): [n][6][400][32]
// bf16, the input of every layer.
__global__ void __launch_bounds__(kThreads, 1)
k_cnn_fwd(const __nv_bfloat16 *__restrict__ x, int n, const __nv_bfloat16 *__restrict__ wpk,
          const float *__restrict__ bias, float *__restrict__ y, __nv_bfloat16 *__restrict__ acts,
          const int *__restrict__ n_dev = nullptr) {
  extern __shared__ __align__(128) unsigned char smraw[];
  FwdSmem &S = *reinterpret_cast<FwdSmem *>(smraw);
  if (n_dev) n = min(n, *n_dev);  // sample count decided on the device
  {
    const uint4 *src = reinterpret_cast<const uint4 *>(wpk);
    uint4 *dst = reinterpret_cast<uint4 *>(S.w);
    for (int i = threadIdx.x; i < kWElems * 2 / 16; i += blockDim.x) dst[i] = src[i];
    for (int i = threadIdx.x; i < kL * kC; i += blockDim.x) S.bias[i / kC][i % kC] = bias[i];
    zero_tile(S.tile[0]);
    zero_tile(S.tile[1]);
  }
  __syncthreads();
  for (int s = blockIdx.x; s < n; s += gridDim.x) {
    // input: channels 0, 1 from x, 2..15 zero (layer 1 reads channels 0..15)
    for (int p = threadIdx.x; p < kNP; p += blockDim.x) {
      const int yy = p / kT, xx = p % kT;
      __nv_bfloat16 *d = S.tile[0] + ((yy + 1) * kTP + xx + 1) * kPP;
      const __nv_bfloat162 v = reinterpret_cast<const __nv_bfloat162 *>(x)[(int64_t)s * kNP + p];
      uint4 *d4 = reinterpret_cast<uint4 *>(d);
      d4[0] = make_uint4(*reinterpret_cast<const uint32_t *>(&v), 0, 0, 0);
      d4[1] = make_uint4(0, 0, 0, 0);
      if (acts) {
        uint4 *g4 = reinterpret_cast<uint4 *>(acts + ((int64_t)s * kL) * kNP * kC + p * kC);
        g4[0] = d4[0];
        g4[1] = d4[1];
        g4[2] = make_uint4(0, 0, 0, 0);
        g4[3] = make_uint4(0, 0, 0, 0);
      }
    }
    __syncthreads();
    for (int l = 0; l < kL; ++l) {
      const __nv_bfloat16 *in = S.tile[l & 1];
      __nv_bfloat16 *out = S.tile[(l + 1) & 1];
      const bool last = l == kL - 1;
      if (!last) {
        conv_tile(in, S.w + l * 9 * kWMat, l == 0 ? 1 : 2, 4, false, S.bias[l],
                  [&](int p, int co, float v0, float v1) {
                    const int yy = p / kT, xx = p % kT;
                    *reinterpret_cast<uint32_t *>(out + ((yy + 1) * kTP + xx + 1) * kPP + co) =
                        pack_bf16(fmaxf(v0, 0.f), fmaxf(v1, 0.f));
                  });
      } else {
        conv_tile(in, S.w + l * 9 * kWMat, 2, 1, false, S.bias[l], [&](int p, int co, float v0, float) {
          if (co != 0) return;
          const int yy = p / kT, xx = p % kT;
          if (yy >= 2 && yy < 18 && xx >= 2 && xx < 18 && y) y[(int64_t)s * 256 + (yy - 2) * 16 + (xx - 2)] = v0;
        });
      }
      __syncthreads();
      if (!last && acts) store_tile(out, acts + ((int64_t)s * kL + l + 1) * kNP * kC);
    }
    __syncthreads();
  }
}

// Radial stencil weights of cell column qx (0..15) of a sample whose block starts at
// global r index ir0 (cylindrical: w- = (2i-2)/(2i-1), w+ = 2i/(2i-1), i = ir0+qx+1).
__device__ __forceinline__ void rweights(int geom, int ir0, int qx, float &wm, float &wp) {
  if (geom == 1) {
    const float i = (float)(ir0 + qx + 1);
    wm = (2.f * i - 2.f) / (2.f * i - 1.f);
    wp = (2.f * i) / (2.f * i - 1.f);
  } else {
    wm = 1.f;
    wp = 1.f;
  }
}

// Normalised residual of the guess at interior cell (qy, qx) (1..14) of sample s:
// rho = L(y) + x1, the discrete operator applied to the output plus the normalised
// right-hand-side change (both in units where the output scale is s_l |db|).
__device__ __forceinline__ float resid(const float *ys, const __nv_bfloat16 *xs, int geom, int ir0, int qy, int qx) {
  float wm, wp;
  rweights(geom, ir0, qx, wm, wp);
  const float c = ys[qy * 16 + qx];
  const float L = wm * ys[qy * 16 + qx - 1] + wp * ys[qy * 16 + qx + 1] + ys[(qy - 1) * 16 + qx] +
                  ys[(qy + 1) * 16 + qx] - 4.f * c;
  return L + __bfloat162float(xs[((qy + 2) * kT + qx + 2) * 2 + 1]);
}

// Loss and output gradient.  Loss = mean_{n x 256} (y - t)^2 + lambda mean_{n x 196} rho^2
// (rho on the 14 x 14 interior cells); loss partials per CTA (fixed order) and
// dz[n][400][32] bf16 = dLoss/dy on the centre pixels of channel 0, else 0.
__global__ void k_cnn_loss(const float *__restrict__ y, const float *__restrict__ t,
                           const __nv_bfloat16 *__restrict__ x, const int *__restrict__ ir0s, float lambda, int geom,
                           int n, __nv_bfloat16 *__restrict__ dz, double *__restrict__ loss_part) {
  const double inv = 1.0 / (256.0 * (double)n), invr = 1.0 / (196.0 * (double)n);
  double acc = 0.0;
  const int64_t total = (int64_t)n * kNP;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int s = (int)(i / kNP), p = (int)(i % kNP);
    const int yy = p / kT, xx = p % kT;
    float g = 0.f;
    if (yy >= 2 && yy < 18 && xx >= 2 && xx < 18) {
      const int cy = yy - 2, cx = xx - 2;
      const int64_t k = (int64_t)s * 256 + cy * 16 + cx;
      const float d = y[k] - t[k];
      acc += (double)d * (double)d * inv;
      g = (float)(2.0 * inv) * d;
      if (lambda > 0.f) {
        const float *ys = y + (int64_t)s * 256;
        const __nv_bfloat16 *xs = x + (int64_t)s * kNP * 2;
        const int ir0 = ir0s[s];
        auto inner = [](int q) { return q >= 1 && q <= 14; };
        float gr = 0.f;
        if (inner(cy) && inner(cx)) {
          const float r0 = resid(ys, xs, geom, ir0, cy, cx);
          acc += (double)lambda * (double)r0 * (double)r0 * invr;
          gr += -4.f * r0;
        }
        // neighbours whose stencil reads this cell
        if (inner(cy) && inner(cx + 1)) {  // this cell is the r- neighbour of (cy, cx+1)
          float wm, wp;
          rweights(geom, ir0, cx + 1, wm, wp);
          gr += wm * resid(ys, xs, geom, ir0, cy, cx + 1);
        }
        if (inner(cy) && inner(cx - 1)) {  // r+ neighbour of (cy, cx-1)
          float wm, wp;
          rweights(geom, ir0, cx - 1, wm, wp);
          gr += wp * resid(ys, xs, geom, ir0, cy, cx - 1);
        }
        if (inner(cy + 1) && inner(cx)) gr += resid(ys, xs, geom, ir0, cy + 1, cx);
        if (inner(cy - 1) && inner(cx)) gr += resid(ys, xs, geom, ir0, cy - 1, cx);
        g += (float)(2.0 * invr) * lambda * gr;
      }
    }
    uint4 *o = reinterpret_cast<uint4 *>(dz + i * kC);
    __nv_bfloat16 gb = __float2bfloat16_rn(g);
    o[0] = make_uint4((uint32_t)*reinterpret_cast<uint16_t *>(&gb), 0, 0, 0);
    o[1] = make_uint4(0, 0, 0, 0);
    o[2] = make_uint4(0, 0, 0, 0);
    o[3] = make_uint4(0, 0, 0, 0);
  }
  __shared__ double sh[32];
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double c = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) c += sh[w];
    loss_part[blockIdx.x] = c;
  }
}

// dz[n][400][32] bf16 from a given output gradient dy[n][256] (centre pixels, channel 0).
__global__ void k_cnn_dz_from_dy(const float *__restrict__ dy, int n, __nv_bfloat16 *__restrict__ dz) {
  const int64_t total = (int64_t)n * kNP;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int s = (int)(i / kNP), p = (int)(i % kNP);
    const int yy = p / kT, xx = p % kT;
    float g = 0.f;
    if (yy >= 2 && yy < 18 && xx >= 2 && xx < 18) g = dy[(int64_t)s * 256 + (yy - 2) * 16 + (xx - 2)];
    uint4 *o = reinterpret_cast<uint4 *>(dz + i * kC);
    __nv_bfloat16 gb = __float2bfloat16_rn(g);
    o[0] = make_uint4((uint32_t)*reinterpret_cast<uint16_t *>(&gb), 0, 0, 0);
    o[1] = make_uint4(0, 0, 0, 0);
    o[2] = make_uint4(0, 0, 0, 0);
    o[3] = make_uint4(0, 0, 0, 0);
  }
}

// Input gradient of layer l (l >= 1): dz_out = (dz_in conv W_l^T flipped) * (A_l > 0).
// dz_in, dz_out: [n][400][32]; wt: transposed packed weights (rows = ci, columns = co);
// acts: the forward activations (A_l = acts[s][l]).
__global__ void __launch_bounds__(kThreads, 1)
k_cnn_dx(int l, const __nv_bfloat16 *__restrict__ dz_in, const __nv_bfloat16 *__restrict__ wt,
         const __nv_bfloat16 *__restrict__ acts, __nv_bfloat16 *__restrict__ dz_out, int n) {
  extern __shared__ __align__(128) unsigned char smraw[];
  FwdSmem &S = *reinterpret_cast<FwdSmem *>(smraw);
  {
    const uint4 *src = reinterpret_cast<const uint4 *>(wt + l * 9 * kWMat);
    uint4 *dst = reinterpret_cast<uint4 *>(S.w);
    for (int i = threadIdx.x; i < 9 * kWMat * 2 / 16; i += blockDim.x) dst[i] = src[i];
    zero_tile(S.tile[0]);
  }
  __syncthreads();
  const int khalves = (l == kL - 1) ? 1 : 2;  // input channels of the transposed conv = co of layer l
  for (int s = blockIdx.x; s < n; s += gridDim.x) {
    load_tile(S.tile[0], dz_in + (int64_t)s * kNP * kC);
    __syncthreads();
    const __nv_bfloat16 *A = acts + ((int64_t)s * kL + l) * kNP * kC;
    __nv_bfloat16 *o = dz_out + (int64_t)s * kNP * kC;
    conv_tile(S.tile[0], S.w, khalves, 4, true, nullptr, [&](int p, int ci, float v0, float v1) {
      const __nv_bfloat162 a = *reinterpret_cast<const __nv_bfloat162 *>(A + p * kC + ci);
      const float m0 = __low2float(a) > 0.f ? v0 : 0.f, m1 = __high2float(a) > 0.f ? v1 : 0.f;
      *reinterpret_cast<uint32_t *>(o + p * kC + ci) = pack_bf16(m0, m1);
    });
    __syncthreads();
  }
}

// Weight gradient of layer l: per CTA, over its samples,
//   dW[tap][co][ci] += sum_p dz[p][co] * A_l[p + off(tap)][ci],  db[co] += sum_p dz[p][co],
// written as partials [cta][9][32][32] and [cta][32].  18 warps: warp = (tap, co half).
constexpr int kDwThreads = 18 * 32;
struct DwSmem {
  __nv_bfloat16 a[kTileElems];   // A_l, padded, zero ring
  __nv_bfloat16 dz[kNP * kPP];   // dz_l, unpadded, pitch kPP
};

__global__ void __launch_bounds__(kDwThreads, 1)
k_cnn_dw(int l, const __nv_bfloat16 *__restrict__ dz, const __nv_bfloat16 *__restrict__ acts, int n,
         float *__restrict__ dw_part, float *__restrict__ db_part) {
  extern __shared__ __align__(128) unsigned char smraw[];
  DwSmem &S = *reinterpret_cast<DwSmem *>(smraw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t4 = lane & 3;
  const int tap = warp >> 1, mh = warp & 1;  // co rows mh*16 .. mh*16+15
  zero_tile(S.a);
  float acc[4][4];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
  float dbacc = 0.f;
  const int ntiles = (l == 0) ? 1 : 4;      // ci columns: layer 1 has 2 input channels
  const int mrows = (l == kL - 1) ? 1 : 2;  // co halves with real channels
  __syncthreads();
  for (int s = blockIdx.x; s < n; s += gridDim.x) {
    load_tile(S.a, acts + ((int64_t)s * kL + l) * kNP * kC);
    for (int i = threadIdx.x; i < kNP * 4; i += blockDim.x) {
      const int p = i >> 2, c = (i & 3) * 8;
      *reinterpret_cast<uint4 *>(S.dz + p * kPP + c) =
          *reinterpret_cast<const uint4 *>(dz + ((int64_t)s * kNP + p) * kC + c);
    }
    __syncthreads();
    if (mh < mrows) {
      const uint32_t a_s = smem_addr(S.a), z_s = smem_addr(S.dz);
      for (int k0 = 0; k0 < kNP; k0 += 16) {
        // A operand (rows co, k = pixels) from dz [p][co] by transposed ldmatrix:
        // matrices (co 0-7, p 0-7), (co 8-15, p 0-7), (co 0-7, p 8-15), (co 8-15, p 8-15)
        uint32_t a0, a1, a2, a3;
        {
          const int m = lane >> 3, r = lane & 7;
          const int p = k0 + r + (m >> 1) * 8, c = mh * 16 + (m & 1) * 8;
          ldsm4t(z_s + (uint32_t)(p * kPP + c) * 2, a0, a1, a2, a3);
        }
        for (int np = 0; np < ntiles; np += 2) {
          // B operand (k = pixels, n = ci) from A_l [p + off][ci] by transposed ldmatrix:
          // matrices (p 0-7, ci np*8..), (p 8-15, ci np*8..), (p 0-7, ci (np+1)*8..), (p 8-15, ..)
          const int m = lane >> 3, r = lane & 7;
          const int p = k0 + r + (m & 1) * 8, c = (np + (m >> 1)) * 8;
          uint32_t b0, b1, b2, b3;
          ldsm4t(a_s + (uint32_t)(tap_pix(p, tap) * kPP + c) * 2, b0, b1, b2, b3);
          mma16816(acc[np], a0, a1, a2, a3, b0, b1);
          if (np + 1 < ntiles) mma16816(acc[np + 1], a0, a1, a2, a3, b2, b3);
        }
      }
    }
    // db: warp 0..1 (tap 0) sum dz over pixels for their 16 channels
    if (tap == 0 && mh < mrows) {
      for (int c = lane; c < 16; c += 32) {
        float sacc = 0.f;
        for (int p = 0; p < kNP; ++p) sacc += __bfloat162float(S.dz[p * kPP + mh * 16 + c]);
        dbacc += sacc;
      }
    }
    __syncthreads();
  }
  float *o = dw_part + (int64_t)blockIdx.x * 9 * kWMat + tap * kWMat;
  for (int nt = 0; nt < 4; ++nt) {
    const int ci = nt * 8 + 2 * t4;
    const int co = mh * 16 + g;
    o[co * kC + ci] = acc[nt][0];
    o[co * kC + ci + 1] = acc[nt][1];
    o[(co + 8) * kC + ci] = acc[nt][2];
    o[(co + 8) * kC + ci + 1] = acc[nt][3];
  }
  if (tap == 0 && lane < 16) db_part[(int64_t)blockIdx.x * kC + mh * 16 + lane] = dbacc;
}

// Fixed-order sum of the per-CTA partials into the gradient (master layout) of layer l.
__global__ void k_cnn_reduce(int l, const float *__restrict__ dw_part, const float *__restrict__ db_part, int nparts,
                             float *__restrict__ grad) {
  const int co_n = cout(l), ci_n = cin(l);
  const int nw = 9 * co_n * ci_n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nw + co_n; i += gridDim.x * blockDim.x) {
    float s = 0.f;
    if (i < nw) {
      const int tap = i / (co_n * ci_n), rem = i % (co_n * ci_n), co = rem / ci_n, ci = rem % ci_n;
      for (int k = 0; k < nparts; ++k) s += dw_part[(int64_t)k * 9 * kWMat + tap * kWMat + co * kC + ci];
      grad[woff(l) + i] = s;
    } else {
      const int co = i - nw;
      for (int k = 0; k < nparts; ++k) s += db_part[(int64_t)k * kC + co];
      grad[boff(l) + co] = s;
    }
  }
}

#include "srmg_cnn_tc.cuh"

// Packed BF16 weights from the master vector: wpk (forward: rows co, columns ci) and
// wt (input gradient: rows ci, columns co), both [layer][tap][32 x 32 swizzled], zero
// where a layer has fewer channels; bias [layer][32].
__global__ void k_cnn_pack(const float *__restrict__ master, __nv_bfloat16 *__restrict__ wpk,
                           __nv_bfloat16 *__restrict__ wt, float *__restrict__ bias, unsigned char *__restrict__ wtc) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kL * 9 * kWMat; i += gridDim.x * blockDim.x) {
    const int l = i / (9 * kWMat), rem = i % (9 * kWMat), tap = rem / kWMat, r = (rem % kWMat) / kC,
              c = rem % kC;
    // forward: row co = r, column ci = c
    float vf = 0.f, vt = 0.f;
    if (r < cout(l) && c < cin(l)) vf = master[woff(l) + (tap * cout(l) + r) * cin(l) + c];
    // transposed: row ci = r, column co = c
    if (c < cout(l) && r < cin(l)) vt = master[woff(l) + (tap * cout(l) + c) * cin(l) + r];
    const int base = (l * 9 + tap) * kWMat * 2;
    *reinterpret_cast<__nv_bfloat16 *>(reinterpret_cast<char *>(wpk) + base + swz(r, c)) = __float2bfloat16_rn(vf);
    *reinterpret_cast<__nv_bfloat16 *>(reinterpret_cast<char *>(wt) + base + swz(r, c)) = __float2bfloat16_rn(vt);
    // tensor-core copy: canonical no-swizzle K-major, rows co, 16-byte chunks of ci
    *reinterpret_cast<__nv_bfloat16 *>(wtc + (l * 9 + tap) * 2048 + cm_off(r, c >> 3) + (c & 7) * 2) =
        __float2bfloat16_rn(vf);
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kL * kC; i += gridDim.x * blockDim.x) {
    const int l = i / kC, co = i % kC;
    bias[i] = co < cout(l) ? master[boff(l) + co] : 0.f;
  }
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters.
__global__ void k_cnn_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                           float *__restrict__ v, int np, float lr, float b1, float b2, float eps, float c1,
                           float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// Samples of a tree: for leaf-holding block k (leaf[k] = {block, level}) the 20 x 20
// tile of (f * a, g * bsc), pixel order y * 20 + x, and the output scale
// s_level * |g| of the block.
__global__ void k_cnn_gather(const double *__restrict__ phi, const double *__restrict__ db, const int2 *__restrict__ leaf,
                             int nleaf, const double *__restrict__ norms, double s, __nv_bfloat16 *__restrict__ x,
                             double *__restrict__ scale, int *__restrict__ blk, const int *__restrict__ list = nullptr,
                             const int *__restrict__ count = nullptr) {
  // norms[0] = |phi|, norms[1] = |db| (leaf norms); 0 counts as 1.  With a list, sample
  // k is leaf block list[k], k < *count.
  const double a = norms[0] > 0 ? 1.0 / norms[0] : 1.0, bsc = norms[1] > 0 ? 1.0 / norms[1] : 1.0;
  const double dbrms = norms[1] > 0 ? norms[1] : 1.0;
  const int n = count ? min(nleaf, *count) : nleaf;
  const int64_t total = (int64_t)n * kNP;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(i / kNP), p = (int)(i % kNP);
    const int2 lb = leaf[list ? list[k] : k];
    const int64_t o = (int64_t)lb.x * kNP + p;
    reinterpret_cast<__nv_bfloat162 *>(x)[i] =
        __floats2bfloat162_rn((float)(phi[o] * a), (float)(db[o] * bsc));
    if (p == 0) {
      const double f = (double)((int64_t)1 << (lb.y - 1));
      scale[k] = s / (f * f) * dbrms;
      blk[k] = lb.x;
    }
  }
}

// Guess on the valid cells of every leaf-holding block: u = phi + y * scale.
__global__ void k_cnn_scatter(double *__restrict__ u, const double *__restrict__ phi, const float *__restrict__ y,
                              const double *__restrict__ scale, const int2 *__restrict__ leaf, int nleaf,
                              const int *__restrict__ list = nullptr, const int *__restrict__ count = nullptr) {
  const int n = count ? min(nleaf, *count) : nleaf;
  const int64_t total = (int64_t)n * 256;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(i >> 8), c = (int)(i & 255);
    const int64_t o = (int64_t)leaf[list ? list[k] : k].x * kNP + (2 + (c >> 4)) * kT + 2 + (c & 15);
    u[o] = phi[o] + (double)y[i] * scale[k];
  }
}

// d = ca a + cb b + cc c (b, c optional).
__global__ void k_lin_field(double *__restrict__ d, const double *__restrict__ a, double ca,
                            const double *__restrict__ b, double cb, const double *__restrict__ c, double cc,
                            int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v = ca * a[i];
    if (b) v += cb * b[i];
    if (c) v += cc * c[i];
    d[i] = v;
  }
}

// Leaf-cell sums of squares of up to three fields over the leaf-holding blocks, one
// 256-thread block per tree block: part[k * 3 + j] = 4^-(l-1) sum over the block's leaf
// cells of f_j^2.  With `resid`, f_j is the residual -(b + L v_j / s_l) of candidate
// v_j instead of v_j itself.
__global__ void __launch_bounds__(256) k_leaf_sq3(const double *__restrict__ v0, const double *__restrict__ v1,
                                                  const double *__restrict__ v2, int nf, const double *__restrict__ b,
                                                  bool resid, double s, int op, double k2, int geom,
                                                  WTab<double> wt, const int2 *__restrict__ leaf,
                                                  const int4 *__restrict__ info, int nleaf,
                                                  double *__restrict__ part) {
  __shared__ double red[3][8];
  const int t = threadIdx.x;
  const int x = 2 + (t & 15), y = 2 + (t >> 4), o = x + kS * y;
  const int sub = ((x - 2) >> 3) + 2 * ((y - 2) >> 3);
  for (int k = blockIdx.x; k < nleaf; k += gridDim.x) {
    const int2 lb = leaf[k];
    const int4 bi = info[lb.x];
    const bool is_leaf = !(((bi.z & 15) >> sub) & 1);
    const double f = (double)((int64_t)1 << (lb.y - 1));
    const double sl = s / (f * f), wl = 1.0 / (f * f);
    const double centre = op == 1 ? -4.0 - sl * k2 : -4.0;
    const int64_t base = (int64_t)lb.x * kSS;
    const W5<double> w = weights<double>(wt, geom, bi.x, bi.y, x, y);
    double sq[3] = {0.0, 0.0, 0.0};
    const double *vs[3] = {v0, v1, v2};
    for (int j = 0; j < nf; ++j) {
      double val = vs[j][base + o];
      if (resid) val = -(b[base + o] + apply5<double>(vs[j] + base, x, y, w, centre) / sl);
      sq[j] = is_leaf ? val * val : 0.0;
    }
    for (int j = 0; j < 3; ++j) {
      double v = sq[j];
      for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
      if ((t & 31) == 0) red[j][t >> 5] = v;
    }
    __syncthreads();
    if (t < 3) {
      double c = 0.0;
      for (int q = 0; q < 8; ++q) c += red[t][q];
      part[(int64_t)k * 3 + t] = c * wl;
    }
    __syncthreads();
  }
}

// Fixed-order sums of the per-block partials: out[j] = sqrt(sum_k part[k * 3 + j]).
__global__ void __launch_bounds__(1024) k_leaf_sq3_reduce(const double *__restrict__ part, int nleaf, int nf,
                                                         double *__restrict__ out) {
  __shared__ double red[3][32];
  double v[3] = {0.0, 0.0, 0.0};
  for (int k = threadIdx.x; k < nleaf; k += blockDim.x)
    for (int j = 0; j < nf; ++j) v[j] += part[(int64_t)k * 3 + j];
  for (int j = 0; j < 3; ++j) {
    double a = v[j];
    for (int off = 16; off > 0; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
    if ((threadIdx.x & 31) == 0) red[j][threadIdx.x >> 5] = a;
  }
  __syncthreads();
  if (threadIdx.x < (unsigned)nf) {
    double c = 0.0;
    for (int q = 0; q < 32; ++q) c += red[threadIdx.x][q];
    out[threadIdx.x] = sqrt(c);
  }
}

// Active blocks: the leaf-holding blocks whose g energy (part[k * 3 + 1]) is at least
// theta times the largest, listed in leaf order (one CTA, fixed order).
__global__ void __launch_bounds__(1024) k_select_active(const double *__restrict__ part, int nleaf, double theta,
                                                       int *__restrict__ list, int *__restrict__ count) {
  __shared__ double smax[32];
  __shared__ int scnt[1024];
  double m = 0.0;
  for (int k = threadIdx.x; k < nleaf; k += blockDim.x) m = fmax(m, part[(int64_t)k * 3 + 1]);
  for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) smax[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double mm = 0.0;
    for (int q = 0; q < 32; ++q) mm = fmax(mm, smax[q]);
    smax[0] = mm;
  }
  __syncthreads();
  const double thr = theta * smax[0];
  const int chunk = (nleaf + blockDim.x - 1) / blockDim.x;
  const int k0 = threadIdx.x * chunk, k1 = min(nleaf, k0 + chunk);
  int c = 0;
  for (int k = k0; k < k1; ++k) c += part[(int64_t)k * 3 + 1] >= thr && part[(int64_t)k * 3 + 1] > 0.0;
  scnt[threadIdx.x] = c;
  __syncthreads();
  for (int off = 1; off < (int)blockDim.x; off <<= 1) {  // inclusive scan
    const int v = threadIdx.x >= (unsigned)off ? scnt[threadIdx.x - off] : 0;
    __syncthreads();
    scnt[threadIdx.x] += v;
    __syncthreads();
  }
  int w = scnt[threadIdx.x] - c;
  for (int k = k0; k < k1; ++k)
    if (part[(int64_t)k * 3 + 1] >= thr && part[(int64_t)k * 3 + 1] > 0.0) list[w++] = k;
  if (threadIdx.x == blockDim.x - 1) *count = scnt[threadIdx.x];
}

// f = u - phi2, g = b - 2 b1 + b2, ext = u + f, lrn = ext (every element).
__global__ void k_predict_prep(const double *__restrict__ u, const double *__restrict__ phi2,
                               const double *__restrict__ b, const double *__restrict__ b1,
                               const double *__restrict__ b2, double *__restrict__ f, double *__restrict__ g,
                               double *__restrict__ ext, double *__restrict__ lrn, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double ui = u[i], fi = ui - phi2[i];
    f[i] = fi;
    g[i] = b[i] - 2.0 * b1[i] + b2[i];
    ext[i] = ui + fi;
    lrn[i] = ui + fi;
  }
}

// Keep the candidate with the smallest residual norm (ties: the earlier one):
// r[0] previous potential (u itself), r[1] ext, r[2] lrn; copy it into u.
__global__ void k_predict_select(double *__restrict__ u, const double *__restrict__ ext,
                                 const double *__restrict__ lrn, const double *__restrict__ r, int *__restrict__ pick,
                                 int64_t n) {
  int p = 0;
  if (r[1] < r[0]) p = 1;
  if (r[2] < (p ? r[1] : r[0])) p = 2;
  if (blockIdx.x == 0 && threadIdx.x == 0) *pick = p;
  if (p == 0) return;
  const double *src = p == 1 ? ext : lrn;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    u[i] = src[i];
}

}  // namespace cnn

using namespace cnn;

struct srmg_cnn {
  int device = 0;
  cudaStream_t stream = nullptr;
  srmg_ctx *err_ctx = nullptr;  // error strings
  float *master = nullptr, *grad = nullptr, *adam_m = nullptr, *adam_v = nullptr;
  __nv_bfloat16 *wpk = nullptr, *wt = nullptr;
  float *bias = nullptr;
  unsigned char *wtc = nullptr;  // weights in the tcgen05 operand layout
  int *tc_err = nullptr;         // error word of the tcgen05 forward
  bool use_tc = false;           // the warm start's forward pass on tcgen05
  int adam_t = 0;
  int train_n = 0;  // samples of the last training forward
  DevBuf acts, dz0, dz1, dwp, dbp, lossp, y;
  int nsm = 0;
};

namespace {

int cnn_grid(srmg_cnn *net, int n) { return std::max(1, std::min(n, net->nsm)); }

int cnn_pack(srmg_cnn *net) {
  k_cnn_pack<<<64, 256, 0, net->stream>>>(net->master, net->wpk, net->wt, net->bias, net->wtc);
  return cuda_check(net->err_ctx, cudaGetLastError(), "k_cnn_pack");
}

int cnn_setup_attrs(srmg_cnn *net) {
  srmg_ctx *ctx = net->err_ctx;
  CK(cudaFuncSetAttribute(k_cnn_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(FwdSmem)));
  CK(cudaFuncSetAttribute(k_cnn_dx, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(FwdSmem)));
  CK(cudaFuncSetAttribute(k_cnn_dw, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(DwSmem)));
  CK(cudaFuncSetAttribute(k_cnn_fwd_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TcSmem)));
  return SRMG_OK;
}

// Forward pass keeping every layer's activations (training), outputs in net->y.
int cnn_fwd_train(srmg_cnn *net, const __nv_bfloat16 *x, int n) {
  srmg_ctx *ctx = net->err_ctx;
  const int grid = cnn_grid(net, n);
  RC(ensure(ctx, net->acts, (size_t)n * kL * kNP * kC * 2));
  RC(ensure(ctx, net->dz0, (size_t)n * kNP * kC * 2));
  RC(ensure(ctx, net->dz1, (size_t)n * kNP * kC * 2));
  RC(ensure(ctx, net->y, (size_t)n * 256 * 4));
  RC(ensure(ctx, net->dwp, (size_t)grid * 9 * kWMat * 4));
  RC(ensure(ctx, net->dbp, (size_t)grid * kC * 4));
  RC(ensure(ctx, net->lossp, 1024 * 8));
  k_cnn_fwd<<<grid, kThreads, sizeof(FwdSmem), net->stream>>>(x, n, net->wpk, net->bias, (float *)net->y.p,
                                                              (__nv_bfloat16 *)net->acts.p);
  CK(cudaGetLastError());
  net->train_n = n;
  return SRMG_OK;
}

// Backward from the output gradient held in net->dz0 (n samples of the last forward).
int cnn_bwd(srmg_cnn *net, int n) {
  srmg_ctx *ctx = net->err_ctx;
  const int grid = cnn_grid(net, n);
  __nv_bfloat16 *acts = (__nv_bfloat16 *)net->acts.p;
  __nv_bfloat16 *dzc = (__nv_bfloat16 *)net->dz0.p, *dzn = (__nv_bfloat16 *)net->dz1.p;
  for (int l = kL - 1; l >= 0; --l) {
    k_cnn_dw<<<grid, kDwThreads, sizeof(DwSmem), net->stream>>>(l, dzc, acts, n, (float *)net->dwp.p,
                                                                (float *)net->dbp.p);
    k_cnn_reduce<<<16, 256, 0, net->stream>>>(l, (const float *)net->dwp.p, (const float *)net->dbp.p, grid,
                                              net->grad);
    if (l > 0) {
      k_cnn_dx<<<grid, kThreads, sizeof(FwdSmem), net->stream>>>(l, dzc, net->wt, acts, dzn, n);
      std::swap(dzc, dzn);
    }
  }
  CK(cudaGetLastError());
  return SRMG_OK;
}

// Forward + loss + backward: gradient (master layout) in net->grad, loss partials.
int cnn_grad(srmg_cnn *net, const __nv_bfloat16 *x, const float *t, const int *ir0, float lambda, int geom, int n,
             double *loss) {
  srmg_ctx *ctx = net->err_ctx;
  RC(cnn_fwd_train(net, x, n));
  const int lg = std::min(1024, std::max(1, (n * kNP + 255) / 256));
  k_cnn_loss<<<lg, 256, 0, net->stream>>>((const float *)net->y.p, t, x, ir0, ir0 ? lambda : 0.f, geom, n,
                                          (__nv_bfloat16 *)net->dz0.p, (double *)net->lossp.p);
  RC(cnn_bwd(net, n));
  if (loss) {
    std::vector<double> lp(lg);
    CK(cudaMemcpyAsync(lp.data(), net->lossp.p, lg * sizeof(double), cudaMemcpyDeviceToHost, net->stream));
    CK(cudaStreamSynchronize(net->stream));
    double s = 0.0;
    for (double v : lp) s += v;
    *loss = s;
  }
  return SRMG_OK;
}

}  // namespace

extern "C" int srmg_cnn_nparams(void) { return nparams(); }

extern "C" int srmg_cnn_create(srmg_cnn **out, int device, uint64_t seed) {
  if (!out) return SRMG_ERR_BADARG;
  *out = nullptr;
  srmg_ctx *ctx = nullptr;
  int rc = srmg_create(&ctx, 2, 16, 2, device);
  if (rc) return rc;
  srmg_cnn *net = new srmg_cnn();
  net->device = device;
  net->err_ctx = ctx;
  net->stream = ctx->stream;
  cudaDeviceGetAttribute(&net->nsm, cudaDevAttrMultiProcessorCount, device);
  const int np = nparams();
  // He initialisation (normal, std sqrt(2 / fan_in)) from a splitmix64 stream, biases 0
  std::vector<float> h(np, 0.f);
  uint64_t st = seed ^ 0x9E3779B97F4A7C15ull;
  auto next = [&]() {
    uint64_t z = (st += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
  };
  for (int l = 0; l < kL; ++l) {
    const double sd = std::sqrt(2.0 / (9.0 * cin(l))) * (l == kL - 1 ? 0.1 : 1.0);
    for (int i = 0; i < 9 * cout(l) * cin(l); ++i) {
      const double u1 = std::max(next(), 1e-300), u2 = next();
      h[woff(l) + i] = (float)(sd * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2));
    }
  }
  auto dalloc = [&](void **p, size_t b) { return cudaMalloc(p, b) == cudaSuccess; };
  if (!dalloc((void **)&net->master, np * 4) || !dalloc((void **)&net->grad, np * 4) ||
      !dalloc((void **)&net->adam_m, np * 4) || !dalloc((void **)&net->adam_v, np * 4) ||
      !dalloc((void **)&net->wpk, kWElems * 2) || !dalloc((void **)&net->wt, kWElems * 2) ||
      !dalloc((void **)&net->bias, kL * kC * 4) || !dalloc((void **)&net->wtc, kTcWBytes) ||
      !dalloc((void **)&net->tc_err, sizeof(int))) {
    srmg_cnn_destroy(net);
    return SRMG_ERR_NOMEM;
  }
  // Everything on the network's stream, in order: the stream is non-blocking, so
  // nothing orders it after work on the legacy default stream (a plain cudaMemset of
  // wtc could otherwise land after the pack below and wipe it).
  bool set = cudaMemcpyAsync(net->master, h.data(), np * 4, cudaMemcpyHostToDevice, net->stream) == cudaSuccess;
  for (auto [p, b] : {std::pair<void *, size_t>{net->adam_m, np * 4}, {net->adam_v, np * 4}, {net->grad, np * 4},
                      {net->wtc, (size_t)kTcWBytes}, {net->tc_err, sizeof(int)}})
    set = set && cudaMemsetAsync(p, 0, b, net->stream) == cudaSuccess;
  if (!set) {
    srmg_cnn_destroy(net);
    return SRMG_ERR_CUDA;
  }
  if ((rc = cnn_setup_attrs(net)) || (rc = cnn_pack(net))) {
    srmg_cnn_destroy(net);
    return rc;
  }
  cudaStreamSynchronize(net->stream);
  *out = net;
  return SRMG_OK;
}

extern "C" void srmg_cnn_destroy(srmg_cnn *net) {
  if (!net) return;
  cudaSetDevice(net->device);
  cudaStreamSynchronize(net->stream);
  for (void *p : {(void *)net->master, (void *)net->grad, (void *)net->adam_m, (void *)net->adam_v, (void *)net->wpk,
                  (void *)net->wt, (void *)net->bias, (void *)net->wtc, (void *)net->tc_err})
    if (p) cudaFree(p);
  for (DevBuf *b : {&net->acts, &net->dz0, &net->dz1, &net->dwp, &net->dbp, &net->lossp, &net->y})
    if (b->p) cudaFree(b->p);
  if (net->err_ctx) srmg_destroy(net->err_ctx);
  delete net;
}

extern "C" const char *srmg_cnn_last_error(const srmg_cnn *net) {
  return net ? srmg_last_error(net->err_ctx) : "null network";
}

extern "C" int srmg_cnn_get_params(srmg_cnn *net, float *host, int n) {
  if (!net || !host || n != nparams()) return SRMG_ERR_BADARG;
  cudaSetDevice(net->device);
  srmg_ctx *ctx = net->err_ctx;
  CK(cudaMemcpyAsync(host, net->master, n * 4, cudaMemcpyDeviceToHost, net->stream));
  CK(cudaStreamSynchronize(net->stream));
  return SRMG_OK;
}

extern "C" int srmg_cnn_set_params(srmg_cnn *net, const float *host, int n) {
  if (!net || !host || n != nparams()) return SRMG_ERR_BADARG;
  cudaSetDevice(net->device);
  srmg_ctx *ctx = net->err_ctx;
  CK(cudaMemcpyAsync(net->master, host, n * 4, cudaMemcpyHostToDevice, net->stream));
  CK(cudaMemsetAsync(net->adam_m, 0, n * 4, net->stream));
  CK(cudaMemsetAsync(net->adam_v, 0, n * 4, net->stream));
  net->adam_t = 0;
  RC(cnn_pack(net));
  CK(cudaStreamSynchronize(net->stream));
  return SRMG_OK;
}

extern "C" int srmg_cnn_forward(srmg_cnn *net, const uint16_t *x, float *y, int n) {
  if (!net || !x || !y || n < 0) return SRMG_ERR_BADARG;
  if (n == 0) return SRMG_OK;
  cudaSetDevice(net->device);
  srmg_ctx *ctx = net->err_ctx;
  k_cnn_fwd<<<cnn_grid(net, n), kThreads, sizeof(FwdSmem), net->stream>>>((const __nv_bfloat16 *)x, n, net->wpk,
                                                                          net->bias, y, nullptr);
  CK(cudaGetLastError());
  return SRMG_OK;
}

extern "C" int srmg_cnn_forward_tc(srmg_cnn *net, const uint16_t *x, float *y, int n) {
  if (!net || !x || !y || n < 0) return SRMG_ERR_BADARG;
  if (n == 0) return SRMG_OK;
  cudaSetDevice(net->device);
  srmg_ctx *ctx = net->err_ctx;
  k_cnn_fwd_tc<<<cnn_grid(net, n), kTcThreads, sizeof(TcSmem), net->stream>>>((const __nv_bfloat16 *)x, n, net->wtc,
                                                                            net->bias, y, net->tc_err, nullptr);
  CK(cudaGetLastError());
  return SRMG_OK;
}

extern "C" int srmg_cnn_tc_status(srmg_cnn *net) {
  if (!net) return SRMG_ERR_BADARG;
  cudaSetDevice(net->device);
  srmg_ctx *ctx = net->err_ctx;
  int e = 0;
  CK(cudaStreamSynchronize(net->stream));
  CK(cudaMemcpy(&e, net->tc_err, sizeof(int), cudaMemcpyDeviceToHost));
  return e ? fail(ctx, SRMG_ERR_TIMEOUT, "tcgen05 forward: MMA completion wait timed out") : SRMG_OK;
}

extern "C" int srmg_cnn_use_tcgen05(srmg_cnn *net, int enable) {
  if (!net) return SRMG_ERR_BADARG;
  net->use_tc = enable != 0;
  return SRMG_OK;
}

extern "C" int srmg_cnn_gradients(srmg_cnn *net, const uint16_t *x, const float *t, const int *ir0, float lambda,
                                  int geom, int n, float *grad_host, double *loss) {
  if (!net || !x || !t || n <= 0 || lambda < 0 || geom < 0 || geom > 2) return SRMG_ERR_BADARG;
  cudaSetDevice(net->device);
  srmg_ctx *ctx = net->err_ctx;
  RC(cnn_grad(net, (const __nv_bfloat16 *)x, t, ir0, lambda, geom, n, loss));
  if (grad_host) {
    CK(cudaMemcpyAsync(grad_host, net->grad, nparams() * 4, cudaMemcpyDeviceToHost, net->stream));
    CK(cudaStreamSynchronize(net->stream));
  }
  return SRMG_OK;
}

static int cnn_adam_step(srmg_cnn *net, float lr) {
  net->adam_t++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, (float)net->adam_t), c2 = 1.f - std::pow(b2, (float)net->adam_t);
  k_cnn_adam<<<64, 256, 0, net->stream>>>(net->master, net->grad, net->adam_m, net->adam_v, nparams(), lr, b1, b2,
                                          1e-8f, c1, c2);
  return cnn_pack(net);
}

extern "C" int srmg_cnn_forward_train(srmg_cnn *net, const uint16_t *x, int n, float *y) {
  if (!net || !x || !y || n <= 0) return SRMG_ERR_BADARG;
  cudaSetDevice(net->device);
  srmg_ctx *ctx = net->err_ctx;
  RC(cnn_fwd_train(net, (const __nv_bfloat16 *)x, n));
  CK(cudaMemcpyAsync(y, net->y.p, (size_t)n * 256 * 4, cudaMemcpyDeviceToDevice, net->stream));
  CK(cudaStreamSynchronize(net->stream));
  return SRMG_OK;
}

extern "C" int srmg_cnn_backward_step(srmg_cnn *net, const float *dy, int n, float lr, float *grad_host) {
  if (!net || !dy || n <= 0 || n != net->train_n || lr < 0) return SRMG_ERR_BADARG;
  cudaSetDevice(net->device);
  srmg_ctx *ctx = net->err_ctx;
  k_cnn_dz_from_dy<<<std::min(1024, (n * kNP + 255) / 256), 256, 0, net->stream>>>(dy, n,
                                                                                   (__nv_bfloat16 *)net->dz0.p);
  RC(cnn_bwd(net, n));
  if (grad_host) {
    CK(cudaMemcpyAsync(grad_host, net->grad, nparams() * 4, cudaMemcpyDeviceToHost, net->stream));
    CK(cudaStreamSynchronize(net->stream));
  }
  if (lr > 0) RC(cnn_adam_step(net, lr));
  CK(cudaGetLastError());
  return SRMG_OK;
}

extern "C" int srmg_cnn_train_step(srmg_cnn *net, const uint16_t *x, const float *t, const int *ir0, float lambda,
                                   int geom, int n, float lr, double *loss) {
  if (!net || !x || !t || n <= 0 || !(lr > 0) || lambda < 0 || geom < 0 || geom > 2) return SRMG_ERR_BADARG;
  cudaSetDevice(net->device);
  srmg_ctx *ctx = net->err_ctx;
  RC(cnn_grad(net, (const __nv_bfloat16 *)x, t, ir0, lambda, geom, n, loss));
  RC(cnn_adam_step(net, lr));
  CK(cudaGetLastError());
  return SRMG_OK;
}

extern "C" int srmg_cnn_synchronize(srmg_cnn *net) {
  if (!net) return SRMG_ERR_BADARG;
  srmg_ctx *ctx = net->err_ctx;
  CK(cudaStreamSynchronize(net->stream));
  return SRMG_OK;
}

namespace {

int lin_field(srmg_ctx *ctx, double *d, const double *a, double ca, const double *b, double cb, const double *c,
              double cc, int64_t n) {
  k_lin_field<<<(int)std::min<int64_t>(4096, (n + 255) / 256), 256, 0, ctx->stream>>>(d, a, ca, b, cb, c, cc, n);
  return cuda_check(ctx, cudaGetLastError(), "k_lin_field");
}

// Leaf norms (sqrt of 4^-(l-1)-weighted sums over leaf cells) of up to three fields,
// or of their residuals, into out[0..nf) on the device.
int leaf_norms(srmg_ctx *ctx, const double *v0, const double *v1, const double *v2, int nf, const double *b,
               bool resid, double s, int op, double k2, int geom, double *part, double *out) {
  const int n = ctx->nleaf;
  if (n == 0) return cuda_check(ctx, cudaMemsetAsync(out, 0, nf * sizeof(double), ctx->stream), "memset");
  k_leaf_sq3<<<std::min(n, 148 * 8), 256, 0, ctx->stream>>>(v0, v1, v2, nf, b, resid, s, op, k2, geom,
                                                           WTab<double>{ctx->d_wm64, ctx->d_wp64}, ctx->d_leaf,
                                                           ctx->d_info, n, part);
  k_leaf_sq3_reduce<<<1, 1024, 0, ctx->stream>>>(part, n, nf, out);
  return cuda_check(ctx, cudaGetLastError(), "leaf norms");
}

// Samples of a tree from the input fields f (ghosts filled) and g (ghosts are filled
// here, on the copy gw unless gw == g): x, the per-sample output scale and block ids,
// with the input norms computed on the device (norms[0..1]).  No host synchronisation.
int cnn_pack_tree(srmg_ctx *ctx, const double *f, const double *g, double *gw, int64_t nblk_alloc, double s,
                  int op, double k2, int geom, const int8_t *bc, __nv_bfloat16 *x, double *scale, int *blk,
                  double *part, double *norms, int *list = nullptr, int *count = nullptr, double theta = 0.0) {
  const int64_t nval = nblk_alloc * (int64_t)kNP;
  if (gw != g) RC(lin_field(ctx, gw, g, 1.0, nullptr, 0.0, nullptr, 0.0, nval));
  const Signs sg = make_signs(bc);
  for (int l = 1; l <= ctx->nlev; l++) RC(L_fill_ghost<double>(ctx, gw, l, sg, 7));
  RC(leaf_norms(ctx, f, gw, nullptr, 2, nullptr, false, s, op, k2, geom, part, norms));
  const int n = ctx->nleaf;
  if (list) k_select_active<<<1, 1024, 0, ctx->stream>>>(part, n, theta, list, count);
  k_cnn_gather<<<(int)std::min<int64_t>(4096, ((int64_t)n * kNP + 255) / 256), 256, 0, ctx->stream>>>(
      f, gw, ctx->d_leaf, n, norms, s, x, scale, blk, list, count);
  CK(cudaGetLastError());
  return n;
}

}  // namespace

extern "C" int srmg_cnn_last_active(const srmg_ctx *ctx) { return ctx ? ctx->cnn_last_active : SRMG_ERR_BADARG; }

extern "C" int srmg_cnn_leaf_blocks(const srmg_ctx *ctx) {
  if (!ctx) return SRMG_ERR_BADARG;
  return ctx->has_tree ? ctx->nleaf : 0;
}

extern "C" int srmg_cnn_pack_dev(srmg_ctx *ctx, const double *f, const double *g, int64_t nblk_alloc, double s,
                                 int op, double k2, int geom, const int8_t bc[9], uint16_t *x, double *scale,
                                 int *blk, int max_samples) {
  RC(check_call(ctx, nblk_alloc, op, geom, bc));
  if (op == SRMG_OP_LAPLACIAN4)
    return fail(ctx, SRMG_ERR_UNSUPPORTED, "the learned warm start supports order-2 discretisations");
  if (!f || !g || !x || !scale || !blk) return fail(ctx, SRMG_ERR_BADARG, "srmg_cnn_pack_dev: null argument");
  if (max_samples < ctx->nleaf)
    return fail(ctx, SRMG_ERR_BADARG, "srmg_cnn_pack_dev: room for %d samples, the tree has %d", max_samples,
                ctx->nleaf);
  const int64_t nval = nblk_alloc * (int64_t)kNP;
  RC(ensure(ctx, ctx->cnn_work[0], nval * sizeof(double) + (3 * (size_t)ctx->nleaf + 8) * sizeof(double)));
  double *gw = (double *)ctx->cnn_work[0].p, *part = gw + nval, *norms = part + 3 * (size_t)ctx->nleaf;
  const int n = cnn_pack_tree(ctx, f, g, gw, nblk_alloc, s, op, k2, geom, bc, (__nv_bfloat16 *)x, scale, blk,
                              part, norms);
  if (n < 0) return n;
  CK(cudaStreamSynchronize(ctx->stream));
  return n;
}

extern "C" int srmg_cnn_predict_dev(srmg_ctx *ctx, srmg_cnn *net, double *u, const double *b, const double *b1,
                                    const double *phi2, const double *b2, int64_t nblk_alloc, double s, int op,
                                    double k2, int geom, const int8_t bc[9], int *which, double *resid) {
  RC(check_call(ctx, nblk_alloc, op, geom, bc));
  if (op == SRMG_OP_LAPLACIAN4)
    return fail(ctx, SRMG_ERR_UNSUPPORTED, "the learned warm start supports order-2 discretisations");
  if (!net || !u || !b || !b1 || !phi2 || !b2) return fail(ctx, SRMG_ERR_BADARG, "srmg_cnn_predict_dev: null argument");
  if (net->device != ctx->device) return fail(ctx, SRMG_ERR_BADARG, "network and context on different devices");
  const int n = ctx->nleaf;
  const int64_t nval = nblk_alloc * (int64_t)kNP;
  // work: f = u - phi2 (previous correction), g = b - 2 b1 + b2 (ghosts filled in place),
  // the extrapolated and the learned candidates, per-block partials and norms
  RC(ensure(ctx, ctx->cnn_work[1], (4 * (size_t)nval + 3 * (size_t)n + 16) * sizeof(double) + (n + 8) * sizeof(int)));
  double *f = (double *)ctx->cnn_work[1].p, *g = f + nval, *ext = g + nval, *lrn = ext + nval;
  double *part = lrn + nval, *norms = part + 3 * (size_t)n;  // norms[0..1] inputs, [2..4] residuals
  int *pick = (int *)(norms + 8), *count = pick + 1, *list = pick + 2;
  // x: [n][400][2] bf16; y: [n][256] float; scale: [n] double; blk: [n] int
  const size_t xb = (size_t)n * kNP * 2 * sizeof(__nv_bfloat16), yb = (size_t)n * 256 * sizeof(float),
               sb = (size_t)n * sizeof(double), bb = (size_t)n * sizeof(int);
  RC(ensure(ctx, ctx->cnn_work[2], xb + yb + sb + bb + 64));
  char *w = (char *)ctx->cnn_work[2].p;
  __nv_bfloat16 *x = (__nv_bfloat16 *)w;
  float *y = (float *)(w + ((xb + 15) & ~size_t(15)));
  double *scale = (double *)((char *)y + ((yb + 15) & ~size_t(15)));
  int *blk = (int *)((char *)scale + ((sb + 15) & ~size_t(15)));
  const int grid = (int)std::min<int64_t>(4096, (nval + 255) / 256);
  k_predict_prep<<<grid, 256, 0, ctx->stream>>>(u, phi2, b, b1, b2, f, g, ext, lrn, nval);
  CK(cudaGetLastError());
  // the network runs on the active blocks (g energy >= theta * the largest); the others
  // keep the extrapolation
  const double theta = ctx->cnn_active_ppm * 1e-6;
  const bool sel = ctx->cnn_active_ppm > 0;
  const int got = cnn_pack_tree(ctx, f, g, g, nblk_alloc, s, op, k2, geom, bc, x, scale, blk, part, norms,
                                sel ? list : nullptr, sel ? count : nullptr, theta);
  if (got < 0) return got;
  if (net->use_tc)
    k_cnn_fwd_tc<<<cnn_grid(net, n), kTcThreads, sizeof(TcSmem), ctx->stream>>>(x, n, net->wtc, net->bias, y,
                                                                                net->tc_err, sel ? count : nullptr);
  else
    k_cnn_fwd<<<cnn_grid(net, n), kThreads, sizeof(FwdSmem), ctx->stream>>>(x, n, net->wpk, net->bias, y, nullptr,
                                                                            sel ? count : nullptr);
  CK(cudaGetLastError());
  k_cnn_scatter<<<(int)std::min<int64_t>(4096, ((int64_t)n * 256 + 255) / 256), 256, 0, ctx->stream>>>(
      lrn, ext, y, scale, ctx->d_leaf, n, sel ? list : nullptr, sel ? count : nullptr);
  // composite-grid functions of their leaves, ghosts filled
  const Signs sg = make_signs(bc);
  for (double *v : {ext, lrn}) {
    for (int l = ctx->nlev; l >= 2; l--) RC(L_restrict<double>(ctx, v, l));
    for (int l = 1; l <= ctx->nlev; l++) RC(L_fill_ghost<double>(ctx, v, l, sg, 7));
  }
  // residual norms of the three candidates; keep the smallest (device-side)
  RC(leaf_norms(ctx, u, ext, lrn, 3, b, true, s, op, k2, geom, part, norms + 2));
  k_predict_select<<<grid, 256, 0, ctx->stream>>>(u, ext, lrn, norms + 2, pick, nval);
  CK(cudaGetLastError());
  if (which || resid) {
    double h[3];
    int hp[2] = {0, n};
    CK(cudaMemcpyAsync(h, norms + 2, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(hp, pick, (sel ? 2 : 1) * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (which) *which = hp[0];
    ctx->cnn_last_active = sel ? hp[1] : n;
    if (resid)
      for (int j = 0; j < 3; j++) resid[j] = h[j];
  }
  return SRMG_OK;
}
