// srmg_freebc.cu -- free boundary conditions on the radial boundary (FreeBC,
// src/freebc.jl, after Malagon-Romero 2018), on the device.
//
// derivs! (src/streamer.jl:320) solves the homogeneous potential uh with the same
// right-hand side and calls freebc!(q1, uh, ...), which adds boundary sources to q1;
// after the main solve, fill_ghost_free! (src/streamer.jl:348) adds the boundary
// values to u's first ghost layer before the field is evaluated.  The transform in
// between works on the outer column at the finest level `level`:
//   u1 = outer valid cells of uh / h_l (getouter!, src/freebc.jl:108-140)
//   b  = DST-III(f .* DST-II(u1)) * h / 2^(level-1) / 2          (src/freebc.jl:93-102)
// with FFTW's unnormalised RODFT10 (DST-II) and RODFT01 (DST-III):
//   DST-II:  Y_k = 2 sum_{j=0}^{n-1} X_j sin(pi (2j+1)(k+1) / (2n))
//   DST-III: Y_k = (-1)^k X_{n-1} + 2 sum_{j=0}^{n-2} X_j sin(pi (j+1)(2k+1) / (2n)).
// When n is a power of two (n = 16 2^(level-1) rootsize: rootsize a power of two along
// the other dimension, the usual (1, 1) root included) both transforms go through one
// complex FFT of length n each, O(n log n): DST-II(x)[k] = DCT-II(x')[n-1-k] with
// x'_j = (-1)^j x_j, and DCT-II through Makhoul's reordering v = (x_0, x_2, ..., x_3,
// x_1) and C_k = 2 Re(e^{-i pi k / 2n} V_k); DST-III(X)[k] = (-1)^k DCT-III(X'')[k] with
// X''_j = X_{n-1-j}, and DCT-III through the inverse reordering of an unnormalised
// inverse FFT of W^{-k} (X''_k - i X''_{n-k}).  For n <= 8192 the gather, both FFTs
// (radix-2 stages, two per pass over shared memory) and the steps between them run in
// one CTA in shared memory; above, a
// four-step n = n1 n2 split (n2 column FFTs with twiddles, then n1 row FFTs) per
// transform, twiddles from a table of e^{-2 pi i k / n}.  Other n run as direct
// sums, one CTA per output in a fixed order, with the sine of every argument from a
// table of sin(pi t / (2n)), t = 0..4n-1 (the integer argument reduced exactly modulo
// 4n).  f, the transform's kernel (modified Bessel functions of the domain's aspect),
// is computed by the caller as FreeBC does and handed over once (srmg_freebc_set).
#include <cmath>

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

namespace {

constexpr int64_t kFreeMaxN = 1 << 17;  // transform length limit (direct sums are O(n^2))
constexpr int kDstThreads = 256;

// Local 0-based (x, y) of a cell `a` cells along `dim` and `o` along the other dimension.
__device__ __forceinline__ int cell_off(int dim, int a, int o) { return dim == 1 ? a + kS * o : o + kS * a; }

__global__ void k_sin_table(double *tab, int64_t n) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < 4 * n; t += (int64_t)gridDim.x * blockDim.x)
    tab[t] = sinpi((double)t / (double)(2 * n));
}

// One position of the outer column: the element of u that getouter! (src/freebc.jl:108-140)
// reads for it -- levels walked in increasing order, so the finest level at the outer
// extent that covers the position wins -- and that level, or off = -1 where no block
// covers it (the column stays zero there).  Built on the host once per tree.
struct FbcSrc {
  long long off;
  int level;
  int pad;
};

// getouter!'s value at position j: u / h_l, h_l = h / 2^(l-1).
__device__ __forceinline__ double outer_value(const FbcSrc *__restrict__ src, const double *__restrict__ u, double h,
                                              int64_t j) {
  const FbcSrc sj = src[j];
  if (sj.off < 0) return 0.0;
  return u[sj.off] / (h / (double)((int64_t)1 << (sj.level - 1)));
}

// u1 = getouter! over every level, one launch (direct-sum path).
__global__ void k_fbc_gather(double *__restrict__ u1, const FbcSrc *__restrict__ src, const double *__restrict__ u,
                             double h, int64_t n) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
    u1[j] = outer_value(src, u, h, j);
}

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double sh[kDstThreads / 32];
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x < 32) {
    r = threadIdx.x < kDstThreads / 32 ? sh[threadIdx.x] : 0.0;
    for (int off = 16; off > 0; off >>= 1) r += __shfl_xor_sync(0xffffffffu, r, off);
  }
  return r;  // valid in thread 0
}

// ---- FFT path (n a power of two) ----------------------------------------------------

constexpr int kFftMaxLocal = 8192;  // one CTA's shared-memory FFT (128 KB of complex doubles)
constexpr int kFftThreads = 512;

__global__ void k_twiddles(double2 *tw, int64_t n) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    double sn, cs;
    sincospi(-2.0 * (double)k / (double)n, &sn, &cs);  // e^{-2 pi i k / n}
    tw[k] = make_double2(cs, sn);
  }
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// `count` forward FFTs of length len (a power of two, <= kFftMaxLocal), one per CTA
// pass: element j of transform t is in[t * in_t + j * in_j]; output k goes to
// out[t * out_t + k * out_k], multiplied by tw[(t * k * tw_mul) mod n] when tw_mul > 0
// (the four-step twiddles).  The table tw holds e^{-2 pi i k / n}; a length-len
// transform uses every (n / len)-th entry.  Iterative radix-2, bit-reversed load.
__global__ void __launch_bounds__(kFftThreads) k_fft(double2 *__restrict__ out, const double2 *__restrict__ in,
                                                     const double2 *__restrict__ tw, int64_t n, int len, int logl,
                                                     int count, int64_t in_t, int64_t in_j, int64_t out_t,
                                                     int64_t out_k, int64_t tw_mul) {
  extern __shared__ double2 sbuf[];
  const int64_t stride_n = n / len;
  for (int t = blockIdx.x; t < count; t += gridDim.x) {
    for (int j = threadIdx.x; j < len; j += blockDim.x) {
      const int r = (int)(__brev((unsigned)j) >> (32 - logl));
      sbuf[r] = in[t * in_t + j * in_j];
    }
    __syncthreads();
    for (int half = 1; half < len; half <<= 1) {
      const int64_t tstep = stride_n * (len / (2 * half));
      for (int idx = threadIdx.x; idx < len / 2; idx += blockDim.x) {
        const int pos = idx & (half - 1), i = (idx - pos) * 2 + pos;
        const double2 w = tw[pos * tstep];
        const double2 a = sbuf[i], b = cmul(sbuf[i + half], w);
        sbuf[i] = make_double2(a.x + b.x, a.y + b.y);
        sbuf[i + half] = make_double2(a.x - b.x, a.y - b.y);
      }
      __syncthreads();
    }
    for (int k = threadIdx.x; k < len; k += blockDim.x) {
      double2 v = sbuf[k];
      if (tw_mul > 0) v = cmul(v, tw[((int64_t)t * k * tw_mul) % n]);
      out[t * out_t + k * out_k] = v;
    }
    __syncthreads();
  }
}

// The length-n forward FFT of `a` into `b` (a is left modified), one or two launches.
int fft_forward(srmg_ctx *ctx, double2 *b, double2 *a, double2 *tmp, const double2 *tw, int64_t n) {
  int logn = 0;
  while (((int64_t)1 << logn) < n) ++logn;
  if (n <= kFftMaxLocal) {
    k_fft<<<1, kFftThreads, n * sizeof(double2), ctx->stream>>>(b, a, tw, n, (int)n, logn, 1, 0, 1, 0, 1, 0);
    ctx->launches++;
    return SRMG_OK;
  }
  // four-step: j = j1 + n1 j2, k = k2 + n2 k1
  const int l2 = logn / 2, l1 = logn - l2;
  const int n1 = 1 << l1, n2 = 1 << l2;
  // step 1: for every j1, the FFT over j2 (stride n1), times W_n^{j1 k2}, into tmp[j1 + n1 k2]
  k_fft<<<std::min(n1, 148 * 4), kFftThreads, n2 * sizeof(double2), ctx->stream>>>(tmp, a, tw, n, n2, l2, n1, 1,
                                                                                  n1, 1, n1, 1);
  // step 2: for every k2, the FFT over j1 (contiguous), into b[k2 + n2 k1]
  k_fft<<<std::min(n2, 148 * 4), kFftThreads, n1 * sizeof(double2), ctx->stream>>>(b, tmp, tw, n, n1, l1, n2, n1,
                                                                                  1, 1, n2, 0);
  ctx->launches += 2;
  return SRMG_OK;
}

// DST-II, step 1: the Makhoul position of x_j in v (x'_j = (-1)^j x_j; v = (x'_0, x'_2,
// ..., x'_3, x'_1)) and its sign.
__device__ __forceinline__ int64_t makhoul_pos(int64_t j, int64_t n) { return (j & 1) ? n - 1 - (j >> 1) : (j >> 1); }

// getouter! and the reordering in one launch (four-step FFT path): v[pos(j)] = +-u1_j.
__global__ void k_fbc_gather_pre(double2 *__restrict__ v, const FbcSrc *__restrict__ src, const double *__restrict__ u,
                                 double h, int64_t n) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
    const double x = outer_value(src, u, h, j);
    v[makhoul_pos(j, n)] = make_double2((j & 1) ? -x : x, 0.0);
  }
}

// The half-angle table: hw[m] = (cos, sin)(pi m / 2n), m = 0..n, from sincospi once
// per srmg_freebc_set (the transforms read it instead of evaluating sincospi).
__global__ void k_half_twiddles(double2 *hw, int64_t n) {
  for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m <= n; m += (int64_t)gridDim.x * blockDim.x) {
    double sn, cs;
    sincospi((double)m / (double)(2 * n), &sn, &cs);
    hw[m] = make_double2(cs, sn);
  }
}

// DST-II, step 2, at m: C[m] = 2 Re(e^{-i pi m / 2n} V[m]) = 2 (Re V cos + Im V sin),
// the DCT-II of x' (y_k = C[n-1-k] is the DST-II); hm = hw[m].  Every product and sum
// rounded on its own.
__device__ __forceinline__ double dct2_at(double2 z, double2 hm) {
  return 2.0 * __dadd_rn(__dmul_rn(z.x, hm.x), __dmul_rn(z.y, hm.y));
}

// The DST-III input at m from the DST-II output: X_j = f_j y_j (rounded once) reversed,
// X''_m = X_{n-1-m} = f_{n-1-m} C[m], X''_{n-m} = f_{m-1} C[n-m] (X''_n = 0), and
// V'[m] = e^{+i pi m / 2n} (X''_m - i X''_{n-m}), conjugated for the inverse transform
// done as a forward FFT: (cos xm + sin xnm) - i (sin xm - cos xnm); hm = hw[m].
__device__ __forceinline__ double2 dst3_in(double xm, double xnm, double2 hm) {
  return make_double2(__dadd_rn(__dmul_rn(hm.x, xm), __dmul_rn(hm.y, xnm)),
                      -__dadd_rn(__dmul_rn(hm.y, xm), -__dmul_rn(hm.x, xnm)));
}

// DST-II step 2 and the DST-III input over all m (four-step FFT path).  With y_out the
// DST-II output is kept.
__global__ void k_dst_mid(double2 *__restrict__ vp, double *__restrict__ y_out, const double2 *__restrict__ V,
                          const double *__restrict__ f, const double2 *__restrict__ hw, int64_t n) {
  for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < n; m += (int64_t)gridDim.x * blockDim.x) {
    const double2 hm = hw[m];
    const double cm = dct2_at(V[m], hm);
    if (y_out) y_out[n - 1 - m] = cm;
    const double xm = __dmul_rn(f[n - 1 - m], cm);
    const double xnm = m == 0 ? 0.0 : __dmul_rn(f[m - 1], dct2_at(V[n - m], hw[n - m]));
    vp[m] = dst3_in(xm, xnm, hm);
  }
}

// DST-III, last step: the unnormalised inverse FFT is conj(FFT(conj V')): w = conj of
// the forward result; y[2j] = Re w[j], y[2j+1] = Re w[n-1-j]; DST-III[k] = (-1)^k y[k];
// b[k] = DST-III[k] h / 2^(level-1) / 2.
__global__ void k_dst3_post(double *__restrict__ b, const double2 *__restrict__ w, int64_t n, double h, double p2) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n / 2; j += (int64_t)gridDim.x * blockDim.x) {
    const double ye = w[j].x, yo = w[n - 1 - j].x;  // Re(conj z) = Re z
    b[2 * j] = ye * h / p2 / 2.0;                   // (-1)^(2j) = 1
    b[2 * j + 1] = -yo * h / p2 / 2.0;
  }
}

// ---- the whole transform in one CTA (n a power of two, n <= kFftMaxLocal) -----------

constexpr int kLocalThreads = 1024;

// Shared-memory index of element i: one pad element after every eight, so that the
// power-of-two strides of the butterflies and of the twiddle reads fall on different
// banks (16-byte elements, a quarter-warp of 8 threads per 128-byte wavefront).
__device__ __forceinline__ int spad(int i) { return i + (i >> 3); }

// Decimation in time: a' = a + w c, c' = a - w c.
__device__ __forceinline__ void bfly_dit(double2 &a, double2 &c, double2 w) {
  const double2 t = cmul(c, w);
  c = make_double2(a.x - t.x, a.y - t.y);
  a = make_double2(a.x + t.x, a.y + t.y);
}

// Decimation in frequency: a' = a + c, c' = (a - c) w.
__device__ __forceinline__ void bfly_dif(double2 &a, double2 &c, double2 w) {
  const double2 d = make_double2(a.x - c.x, a.y - c.y);
  a = make_double2(a.x + c.x, a.y + c.y);
  c = cmul(d, w);
}

// In-place radix-2 FFTs over buf (padded, spad) with the twiddles W^k = e^{-2 pi i k / n},
// k < n / 2, in shared memory (padded), two stages per pass over shared memory.
// Decimation in frequency takes natural order to bit-reversed order: stages
// half = n/2, n/4, ..., 1, a thread holding e_q = g + pos + q H/2 (q = 0..3, g a
// multiple of 2H, pos < H/2) for the stage pair (H, H/2): (e0, e2) with W_{2H}^pos,
// (e1, e3) with W_{2H}^(pos + H/2), then (e0, e1) and (e2, e3) with W_H^pos.
__device__ __forceinline__ void local_fft_dif(double2 *buf, const double2 *stw, int n, int logn) {
  int H = n / 2;
  for (; H >= 2; H >>= 2) {
    const int q = H / 2, t1 = n / (2 * H), t2 = n / H;
    for (int idx = threadIdx.x; idx < n / 4; idx += blockDim.x) {
      const int pos = idx & (q - 1), e0 = (idx - pos) * 4 + pos;
      double2 a0 = buf[spad(e0)], a1 = buf[spad(e0 + q)], a2 = buf[spad(e0 + 2 * q)], a3 = buf[spad(e0 + 3 * q)];
      bfly_dif(a0, a2, stw[spad(pos * t1)]);
      bfly_dif(a1, a3, stw[spad((pos + q) * t1)]);
      const double2 w2 = stw[spad(pos * t2)];
      bfly_dif(a0, a1, w2);
      bfly_dif(a2, a3, w2);
      buf[spad(e0)] = a0;
      buf[spad(e0 + q)] = a1;
      buf[spad(e0 + 2 * q)] = a2;
      buf[spad(e0 + 3 * q)] = a3;
    }
    __syncthreads();
  }
  if (H == 1) {  // an odd stage count ends with one radix-2 stage (twiddle 1)
    for (int idx = threadIdx.x; idx < n / 2; idx += blockDim.x) {
      double2 a = buf[spad(2 * idx)], c = buf[spad(2 * idx + 1)];
      bfly_dif(a, c, stw[0]);
      buf[spad(2 * idx)] = a;
      buf[spad(2 * idx + 1)] = c;
    }
    __syncthreads();
  }
}

// Decimation in time takes bit-reversed order to natural order: stages half = 1, 2,
// ..., n/2 (the butterflies of k_fft), a thread holding g + pos + {0, h, 2h, 3h} (g a
// multiple of 4h, pos < h) for the stage pair (h, 2h): (0, h) and (2h, 3h) with
// W_{2h}^pos, then (0, 2h) with W_{4h}^pos and (h, 3h) with W_{4h}^(pos + h).
__device__ __forceinline__ void local_fft_dit(double2 *buf, const double2 *stw, int n, int logn) {
  int half = 1;
  if (logn & 1) {  // one radix-2 stage first when the stage count is odd
    for (int idx = threadIdx.x; idx < n / 2; idx += blockDim.x) {
      double2 a = buf[spad(2 * idx)], c = buf[spad(2 * idx + 1)];
      bfly_dit(a, c, stw[0]);
      buf[spad(2 * idx)] = a;
      buf[spad(2 * idx + 1)] = c;
    }
    __syncthreads();
    half = 2;
  }
  for (; half < n; half <<= 2) {
    const int t1 = n / (2 * half), t2 = n / (4 * half);
    for (int idx = threadIdx.x; idx < n / 4; idx += blockDim.x) {
      const int pos = idx & (half - 1), i = (idx - pos) * 4 + pos;
      double2 a0 = buf[spad(i)], a1 = buf[spad(i + half)], a2 = buf[spad(i + 2 * half)],
              a3 = buf[spad(i + 3 * half)];
      const double2 w1 = stw[spad(pos * t1)];
      bfly_dit(a0, a1, w1);
      bfly_dit(a2, a3, w1);
      bfly_dit(a0, a2, stw[spad(pos * t2)]);
      bfly_dit(a1, a3, stw[spad((pos + half) * t2)]);
      buf[spad(i)] = a0;
      buf[spad(i + half)] = a1;
      buf[spad(i + 2 * half)] = a2;
      buf[spad(i + 3 * half)] = a3;
    }
    __syncthreads();
  }
}

// Dynamic shared memory of k_dst_local: n + n/8 padded complex values and n/2 + n/16
// padded twiddles (27 n bytes, 216 KB at n = 8192).
constexpr int local_smem_bytes(int n) { return (int)sizeof(double2) * (n + n / 8 + n / 2 + n / 16); }

// b = DST-III(f .* DST-II(getouter!(u))) h / 2^(level-1) / 2 in one CTA.  The gather
// and the Makhoul reordering load the first FFT's input in natural order; that FFT
// (decimation in frequency) leaves V in bit-reversed order, so the DST-III input of the
// pair (m, n - m) -- formed in place by one thread -- lands exactly where the second FFT
// (decimation in time) wants it, at the bit-reversed positions of m and n - m; that FFT
// leaves natural order for the output reordering.  No permutation pass.
__global__ void __launch_bounds__(kLocalThreads, 1)
    k_dst_local(double *__restrict__ b, const FbcSrc *__restrict__ src, const double *__restrict__ u, double h,
                const double2 *__restrict__ tw, const double2 *__restrict__ hw, const double *__restrict__ f, int n,
                int logn, double p2) {
  extern __shared__ double2 sm[];
  double2 *buf = sm, *stw = sm + spad(n);
  for (int k = threadIdx.x; k < n / 2; k += blockDim.x) stw[spad(k)] = tw[k];
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    const double x = outer_value(src, u, h, j);
    buf[spad((int)makhoul_pos(j, n))] = make_double2((j & 1) ? -x : x, 0.0);
  }
  __syncthreads();
  local_fft_dif(buf, stw, n, logn);
  auto brev = [&](int i) { return (int)(__brev((unsigned)i) >> (32 - logn)); };
  for (int m = threadIdx.x; m <= n / 2; m += blockDim.x) {
    const int mm = n - m;  // the partner position (m = 0 has none, m = n / 2 is its own)
    const int am = spad(brev(m));
    const double2 hm = hw[m];
    const double cm = dct2_at(buf[am], hm);
    if (m == 0) {
      buf[am] = dst3_in(__dmul_rn(f[n - 1], cm), 0.0, hm);
      continue;
    }
    const int amm = spad(brev(mm));
    const double2 hmm = hw[mm];
    const double cmm = dct2_at(buf[amm], hmm);
    const double2 vm = dst3_in(__dmul_rn(f[n - 1 - m], cm), __dmul_rn(f[m - 1], cmm), hm);
    if (mm != m) buf[amm] = dst3_in(__dmul_rn(f[n - 1 - mm], cmm), __dmul_rn(f[mm - 1], cm), hmm);
    buf[am] = vm;
  }
  __syncthreads();
  local_fft_dit(buf, stw, n, logn);
  for (int j = threadIdx.x; j < n / 2; j += blockDim.x) {
    const double ye = buf[spad(j)].x, yo = buf[spad(n - 1 - j)].x;  // as k_dst3_post
    b[2 * j] = ye * h / p2 / 2.0;
    b[2 * j + 1] = -yo * h / p2 / 2.0;
  }
}

// y = DST-II(x).  The table index (2j + 1)(k + 1) mod 4n advances by a fixed step per
// iteration of a thread, reduced by one conditional subtraction (4n < 2^31).
__global__ void __launch_bounds__(kDstThreads) k_dst2(double *__restrict__ y, const double *__restrict__ x,
                                                      const double *__restrict__ tab, int64_t n) {
  const int m4 = (int)(4 * n);
  for (int64_t k = blockIdx.x; k < n; k += gridDim.x) {
    double acc = 0.0;
    int t = (int)(((2 * (int64_t)threadIdx.x + 1) * (k + 1)) % m4);
    const int step = (int)((2 * (int64_t)kDstThreads * (k + 1)) % m4);
    for (int64_t j = threadIdx.x; j < n; j += kDstThreads) {
      acc += x[j] * tab[t];
      t += step;
      if (t >= m4) t -= m4;
    }
    const double s = block_sum(acc);
    if (threadIdx.x == 0) y[k] = 2.0 * s;
    __syncthreads();
  }
}

// b = DST-III(f .* a) * h / 2^(level-1) / 2, the product f a rounded once per element
__global__ void __launch_bounds__(kDstThreads) k_dst3_scale(double *__restrict__ b, const double *__restrict__ a,
                                                            const double *__restrict__ f,
                                                            const double *__restrict__ tab, int64_t n, double h,
                                                            double p2) {
  const int m4 = (int)(4 * n);
  for (int64_t k = blockIdx.x; k < n; k += gridDim.x) {
    double acc = 0.0;
    int t = (int)(((int64_t)threadIdx.x + 1) * (2 * k + 1) % m4);
    const int step = (int)((int64_t)kDstThreads * (2 * k + 1) % m4);
    for (int64_t j = threadIdx.x; j < n - 1; j += kDstThreads) {
      acc += (f[j] * a[j]) * tab[t];
      t += step;
      if (t >= m4) t -= m4;
    }
    const double s = block_sum(acc);
    if (threadIdx.x == 0) {
      const double last = f[n - 1] * a[n - 1];
      const double yk = ((k & 1) ? -last : last) + 2.0 * s;
      b[k] = yk * h / p2 / 2.0;
    }
    __syncthreads();
  }
}

__device__ __forceinline__ double seg_mean(const double *b, int64_t first, int64_t count) {
  double v = 0.0;
  for (int64_t m = 0; m < count; ++m) v = __dadd_rn(v, b[first + m]);
  return v / (double)count;
}

// factor(CylindricalGeometry{D}, J, delta) with delta along D (src/geometry.jl:27-29)
__device__ __forceinline__ double cyl_factor(int64_t J) { return fabs(1.0 + 1.0 / (double)(2 * J - 1)); }

// setouter! (src/freebc.jl:157-219) over every level in one launch: one thread per cell
// of the outer valid column of each listed block (the blocks at the level's outer
// extent, or with a boundary face at +dim).  The thread adds the boundary source
// (src/freebc.jl:157-176) when the block's +dim face is a boundary, then -- for the
// first and last cell of the column -- the refinement-boundary corrections that land
// on it (src/freebc.jl:178-219), walking the connectivity's direction order (`order`
// lists face codes: 0..3 star faces, 4..7 the corners).  Each cell belongs to one
// block and one thread, so its additions happen in the reference's order: the level's
// boundary sources before its refinement corrections, those in direction order.
__global__ void k_setouter_all(double *__restrict__ q, const double *__restrict__ b, const LevelView *__restrict__ lvs,
                               const int2 *__restrict__ ent, int nent, int dim, int level, long long root_dim,
                               double s, int4 order_lo, int4 order_hi, int norder) {
  const int order[8] = {order_lo.x, order_lo.y, order_lo.z, order_lo.w, order_hi.x, order_hi.y, order_hi.z, order_hi.w};
  const int fidx = dim == 1 ? 1 : 3;
  const int64_t total = (int64_t)nent * kM;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int e = (int)(t / kM), i = (int)(t % kM);
    const int l = ent[e].x, bi = ent[e].y;
    const LevelView &lv = lvs[l - 1];
    const int4 bk = lv.blocks[bi];
    const int cd = dim == 1 ? bk.y : bk.z, co = dim == 1 ? bk.z : bk.y;
    const int64_t fl = (int64_t)1 << (l - 1);
    const double sl = s / (double)(fl * fl);
    const int64_t p = (int64_t)1 << (level - l);
    const int64_t Jd = (int64_t)kM * (cd - 1) + kM;
    if (lv.faces[4 * bi + fidx].x == FACE_BOUNDARY) {
      const int64_t i0 = (int64_t)(co - 1) * kM;
      const double bmean = seg_mean(b, p * (i0 + i), p);
      double *qc = q + (int64_t)bk.x * kSS + cell_off(dim, kG + kM - 1, kG + i);
      *qc = *qc + 2.0 * cyl_factor(Jd) * bmean / sl;
    }
    if ((i != 0 && i != kM - 1) || cd != (int)(root_dim << (l - 1))) continue;
    for (int r = 0; r < norder; ++r) {
      const int code = order[r];
      int type, fr, fz;
      if (code < 4) {
        type = lv.faces[4 * bi + code].x;
        fr = code == 0 ? -1 : code == 1 ? 1 : 0;
        fz = code == 2 ? -1 : code == 3 ? 1 : 0;
      } else {
        const int qd = code - 4;
        type = lv.cfaces ? lv.cfaces[4 * bi + qd].x : FACE_NONE;
        fr = 2 * (qd & 1) - 1;
        fz = 2 * (qd >> 1) - 1;
      }
      if (type != FACE_REFBND) continue;
      const int dir = dim == 1 ? fz : fr;  // the face's component along the other dimension
      const int i1 = dir == -1 ? kG + 1 : kM + kG;  // 1-based index along the other dimension
      if (i1 - 1 - kG != i) continue;                // another cell's correction
      const int64_t j = (int64_t)(co - 1) * kM + i1 - kG;
      const int64_t J1d = (Jd - 1) / 2 + 1;
      // 0-based first element: dir = 1 reads b[p j + 1 : p (j + 2)], otherwise
      // b[p (j - 3) : p (j - 1) - 1] (1-based, as written in the reference)
      const int64_t first = dir == 1 ? p * j : p * (j - 3) - 1;
      const double bmean = seg_mean(b, first, 2 * p);
      double *qc = q + (int64_t)bk.x * kSS + cell_off(dim, kG + kM - 1, i1 - 1);
      *qc = *qc + 2.0 * 0.25 * cyl_factor(J1d) * bmean / sl;
    }
  }
}

// fill_ghost_free! of one level (src/freebc.jl:224-243)
__global__ void k_fill_ghost_free(double *__restrict__ u, const double *__restrict__ b, LevelView lv, int dim,
                                  int kext, int p) {
  const int64_t total = (int64_t)lv.nblk * kM;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int bi = (int)(t / kM), i = (int)(t % kM);
    const int4 bk = lv.blocks[bi];
    const int cd = dim == 1 ? bk.y : bk.z, co = dim == 1 ? bk.z : bk.y;
    if (cd != kext) continue;
    const int64_t i0 = (int64_t)(co - 1) * kM;
    const double bmean = seg_mean(b, p * (i0 + i), p);
    double *uc = u + (int64_t)bk.x * kSS + cell_off(dim, kG + kM, kG + i);
    *uc = *uc + 2.0 * bmean;
  }
}

int gridfor(int64_t work, int threads) {
  const int64_t g = (work + threads - 1) / threads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 8));
}

// The context's free-boundary buffer: f [n], the sine table [4n], u1 [n], b [n] (7n
// doubles), and for the FFT path the twiddles [n complex] and three complex work arrays
// [n complex each] (8n doubles), then the half-angle table [n + 1 complex]: 17n + 2
// doubles in all.
constexpr int64_t kFbcDoubles = 7 + 2 * (1 + 3) + 2;
static_assert(kFbcDoubles == 17, "free-boundary buffer layout");
double *fbc_f(srmg_ctx *ctx) { return (double *)ctx->fbc.p; }
double *fbc_tab(srmg_ctx *ctx) { return fbc_f(ctx) + ctx->fbc_n; }
double *fbc_u1(srmg_ctx *ctx) { return fbc_tab(ctx) + 4 * ctx->fbc_n; }
double *fbc_b(srmg_ctx *ctx) { return fbc_u1(ctx) + ctx->fbc_n; }
double2 *fbc_tw(srmg_ctx *ctx) { return (double2 *)(fbc_b(ctx) + ctx->fbc_n); }
double2 *fbc_work(srmg_ctx *ctx, int k) { return fbc_tw(ctx) + (1 + k) * ctx->fbc_n; }
double2 *fbc_hw(srmg_ctx *ctx) { return fbc_work(ctx, 3); }
bool fbc_pow2(int64_t n) { return n >= 2 && (n & (n - 1)) == 0; }

// Levels the boundary work visits, and the checks freebc! makes.
int fbc_ready(srmg_ctx *ctx, int64_t nblk_alloc, const char *who) {
  RC(check_call(ctx, nblk_alloc, 0, 0, nullptr));
  if (ctx->fbc_n <= 0) return fail(ctx, SRMG_ERR_BADARG, "%s: call srmg_freebc_set first", who);
  if (ctx->nitems != 1) return fail(ctx, SRMG_ERR_UNSUPPORTED, "%s: one tree per context", who);
  if (ctx->D != 2) return fail(ctx, SRMG_ERR_UNSUPPORTED, "%s: two-dimensional trees only", who);
  for (int l = ctx->fbc_level + 1; l <= ctx->nlev; ++l)
    if (ctx->nblk_host[l - 1] > 0)
      return fail(ctx, SRMG_ERR_BADARG, "%s: the tree has level %d above the free-boundary level %d", who, l,
                  ctx->fbc_level);
  return SRMG_OK;
}

// The extent of level l along `dim`, in blocks (tree[l].domain, src/blocklayer.jl:111-115).
int extent(srmg_ctx *ctx, int l, int dim) { return (int)(ctx->fbc_root[dim - 1] << (l - 1)); }

// Host checks on the uploaded tree: every block lies inside the level's extent given by
// rootsize (so the gathers and means index inside b), and every refinement correction
// reads inside b (Julia would throw a BoundsError there), with the same index
// arithmetic as k_setouter_all.
int check_tree_fits(srmg_ctx *ctx) {
  const int dim = ctx->fbc_dim, od = dim == 1 ? 2 : 1;
  const int L = std::min(ctx->fbc_level, ctx->htree.nlev);
  for (int l = 1; l <= L; ++l) {
    const int kext = extent(ctx, l, dim), kexo = extent(ctx, l, od);
    const int64_t p = (int64_t)1 << (ctx->fbc_level - l);
    std::vector<int> cd(ctx->htree.max_blk + 1, 0), co(ctx->htree.max_blk + 1, 0);
    for (const srmg_pair &pr : ctx->htree.pairs[l - 1]) {
      if (pr.coord[dim - 1] > kext || pr.coord[od - 1] > kexo)
        return fail(ctx, SRMG_ERR_BADARG, "freebc: block %lld of level %d lies outside the rootsize extent",
                    (long long)pr.blk, l);
      cd[pr.blk] = (int)pr.coord[dim - 1];
      co[pr.blk] = (int)pr.coord[od - 1];
    }
    for (const srmg_refbnd &e : ctx->htree.rb[l - 1]) {
      if (cd[e.fine] != kext) continue;
      const int dir = (int)e.face[od - 1];
      const int i1 = dir == -1 ? kG + 1 : kM + kG;
      const int64_t j = (int64_t)(co[e.fine] - 1) * kM + i1 - kG;
      const int64_t first = dir == 1 ? p * j : p * (j - 3) - 1;
      if (first < 0 || first + 2 * p > ctx->fbc_n)
        return fail(ctx, SRMG_ERR_BADTREE, "freebc: refinement correction of block %lld reads outside b",
                    (long long)e.fine);
    }
  }
  return SRMG_OK;
}


// The tables of srmg_freebc_dev for the current tree and free-boundary setting, built
// once (check_tree_fits included): the outer-column source of every transform position
// (getouter!'s level loop run on the host), the device level views, and the (level,
// index) of every block at its level's outer extent or with a boundary face at +dim.
int fbc_build(srmg_ctx *ctx) {
  if (ctx->fbc_built) return SRMG_OK;
  RC(check_tree_fits(ctx));
  const int dim = ctx->fbc_dim, od = dim == 1 ? 2 : 1, level = ctx->fbc_level;
  const int64_t n = ctx->fbc_n;
  const int L = std::min(level, ctx->nlev);
  std::vector<FbcSrc> src((size_t)n, FbcSrc{-1, 0, 0});
  std::vector<LevelView> lvs((size_t)std::max(L, 1));
  std::vector<int2> ent;
  for (int l = 1; l <= L; ++l) {
    lvs[l - 1] = ctx->lv[l - 1].view(l);
    const int kext = extent(ctx, l, dim);
    const int64_t p = (int64_t)1 << (level - l);
    const auto &pairs = ctx->htree.pairs[l - 1];
    std::vector<char> at_bnd(pairs.size(), 0);
    std::vector<int> idx(ctx->htree.max_blk + 1, -1);
    for (size_t bi = 0; bi < pairs.size(); ++bi) idx[pairs[bi].blk] = (int)bi;
    for (const srmg_boundary &e : ctx->htree.bd[l - 1])
      if (e.face[dim - 1] == 1 && e.face[od - 1] == 0 && e.block >= 1 && e.block <= ctx->htree.max_blk &&
          idx[e.block] >= 0)
        at_bnd[idx[e.block]] = 1;
    for (size_t bi = 0; bi < pairs.size(); ++bi) {
      const srmg_pair &pr = pairs[bi];
      const bool outer = pr.coord[dim - 1] == kext;
      if (outer || at_bnd[bi]) ent.push_back(make_int2(l, (int)bi));
      if (!outer) continue;
      if (pr.coord[od - 1] < 1)
        return fail(ctx, SRMG_ERR_BADARG, "freebc: block %lld of level %d has a coordinate below 1",
                    (long long)pr.blk, l);
      const int64_t i0 = (pr.coord[od - 1] - 1) * kM;
      for (int i = 0; i < kM; ++i) {
        const long long off = (long long)(pr.blk - 1) * kSS +
                              (dim == 1 ? (kG + kM - 1) + kS * (kG + i) : (kG + i) + kS * (kG + kM - 1));
        for (int64_t m = 0; m < p; ++m) src[(size_t)(p * (i0 + i) + m)] = FbcSrc{off, l, 0};
      }
    }
  }
  const size_t b_src = src.size() * sizeof(FbcSrc);
  const size_t o_lvs = (b_src + 255) & ~size_t(255);
  const size_t o_ent = (o_lvs + lvs.size() * sizeof(LevelView) + 255) & ~size_t(255);
  const size_t total = o_ent + std::max<size_t>(ent.size(), 1) * sizeof(int2);
  RC(ensure(ctx, ctx->fbc_tabs, total));
  char *d = (char *)ctx->fbc_tabs.p;
  // on the context's stream (pageable sources, staged before each call returns)
  CK(cudaMemcpyAsync(d, src.data(), b_src, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(d + o_lvs, lvs.data(), lvs.size() * sizeof(LevelView), cudaMemcpyHostToDevice, ctx->stream));
  if (!ent.empty())
    CK(cudaMemcpyAsync(d + o_ent, ent.data(), ent.size() * sizeof(int2), cudaMemcpyHostToDevice, ctx->stream));
  ctx->fbc_off_lvs = o_lvs;
  ctx->fbc_off_ent = o_ent;
  ctx->fbc_nent = (int)ent.size();
  ctx->fbc_built = true;
  return SRMG_OK;
}

const FbcSrc *fbc_src(srmg_ctx *ctx) { return (const FbcSrc *)ctx->fbc_tabs.p; }
const LevelView *fbc_lvs(srmg_ctx *ctx) { return (const LevelView *)((char *)ctx->fbc_tabs.p + ctx->fbc_off_lvs); }
const int2 *fbc_ent(srmg_ctx *ctx) { return (const int2 *)((char *)ctx->fbc_tabs.p + ctx->fbc_off_ent); }

}  // namespace

extern "C" int srmg_freebc_set(srmg_ctx *ctx, int dim, int level, const int64_t rootsize[2], const double *f,
                               int64_t n) {
  if (!ctx) return SRMG_ERR_BADARG;
  if (dim != 1 && dim != 2) return fail(ctx, SRMG_ERR_UNSUPPORTED, "srmg_freebc_set: dim must be 1 or 2");
  if (level < 1 || level > 30 || !rootsize || rootsize[0] < 1 || rootsize[1] < 1 || !f)
    return fail(ctx, SRMG_ERR_BADARG, "srmg_freebc_set: bad arguments");
  const int od = dim == 1 ? 2 : 1;
  const int64_t want = rootsize[od - 1] * ((int64_t)1 << (level - 1)) * kM;
  if (n != want)
    return fail(ctx, SRMG_ERR_BADARG, "srmg_freebc_set: n = %lld, FreeBC has %lld", (long long)n, (long long)want);
  if (n > kFreeMaxN)
    return fail(ctx, SRMG_ERR_UNSUPPORTED, "srmg_freebc_set: transform length %lld above %lld", (long long)n,
                (long long)kFreeMaxN);
  cudaSetDevice(ctx->device);
  RC(ensure(ctx, ctx->fbc, ((size_t)kFbcDoubles * n + 2) * sizeof(double)));
  ctx->fbc_n = n;
  ctx->fbc_dim = dim;
  ctx->fbc_level = level;
  ctx->fbc_root[0] = rootsize[0];
  ctx->fbc_root[1] = rootsize[1];
  ctx->fbc_built = false;
  CK(cudaMemcpyAsync(fbc_f(ctx), f, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  k_sin_table<<<gridfor(4 * n, 256), 256, 0, ctx->stream>>>(fbc_tab(ctx), n);
  ctx->launches++;
  if (fbc_pow2(n)) {
    // the FFT kernel holds up to kFftMaxLocal complex doubles in dynamic shared memory
    CK(cudaFuncSetAttribute(k_fft, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)(kFftMaxLocal * sizeof(double2))));
    // k_dst_local: the padded transform and twiddles
    CK(cudaFuncSetAttribute(k_dst_local, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            local_smem_bytes(kFftMaxLocal)));
    k_twiddles<<<gridfor(n, 256), 256, 0, ctx->stream>>>(fbc_tw(ctx), n);
    k_half_twiddles<<<gridfor(n + 1, 256), 256, 0, ctx->stream>>>(fbc_hw(ctx), n);
    ctx->launches += 2;
  }
  CK(cudaMemsetAsync(fbc_b(ctx), 0, n * sizeof(double), ctx->stream));
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  return SRMG_OK;
}

extern "C" int srmg_freebc_dev(srmg_ctx *ctx, double *q, const double *u, int64_t nblk_alloc, double h, double s,
                               double *b_out) {
  RC(fbc_ready(ctx, nblk_alloc, "srmg_freebc"));
  if (!q || !u) return fail(ctx, SRMG_ERR_BADARG, "srmg_freebc: null field");
  if (!(h > 0.0) || !std::isfinite(h) || !std::isfinite(s) || s == 0.0)
    return fail(ctx, SRMG_ERR_BADARG, "srmg_freebc: bad h or s");
  RC(fbc_build(ctx));
  const int dim = ctx->fbc_dim, level = ctx->fbc_level;
  const int64_t n = ctx->fbc_n;
  double *u1 = fbc_u1(ctx), *b = fbc_b(ctx), *am = b;  // DST-II output shares b's storage until the end
  const double p2 = (double)((int64_t)1 << (level - 1));
  if (fbc_pow2(n) && !ctx->fbc_direct && n <= kFftMaxLocal) {
    // gather, DST-II, times f, DST-III: one CTA
    int logn = 0;
    while (((int64_t)1 << logn) < n) ++logn;
    k_dst_local<<<1, kLocalThreads, local_smem_bytes((int)n), ctx->stream>>>(b, fbc_src(ctx), u, h, fbc_tw(ctx), fbc_hw(ctx), fbc_f(ctx), (int)n,
                                                          logn, p2);
    ctx->launches++;
  } else if (fbc_pow2(n) && !ctx->fbc_direct) {
    double2 *w0 = fbc_work(ctx, 0), *w1 = fbc_work(ctx, 1), *w2 = fbc_work(ctx, 2);
    k_fbc_gather_pre<<<gridfor(n, 256), 256, 0, ctx->stream>>>(w0, fbc_src(ctx), u, h, n);
    RC(fft_forward(ctx, w1, w0, w2, fbc_tw(ctx), n));
    k_dst_mid<<<gridfor(n, 256), 256, 0, ctx->stream>>>(w0, nullptr, w1, fbc_f(ctx), fbc_hw(ctx), n);
    RC(fft_forward(ctx, w1, w0, w2, fbc_tw(ctx), n));
    k_dst3_post<<<gridfor(n / 2, 256), 256, 0, ctx->stream>>>(b, w1, n, h, p2);
    ctx->launches += 3;
  } else {
    k_fbc_gather<<<gridfor(n, 256), 256, 0, ctx->stream>>>(u1, fbc_src(ctx), u, h, n);
    const int g = (int)std::min<int64_t>(n, 148 * 16);
    k_dst2<<<g, kDstThreads, 0, ctx->stream>>>(am, u1, fbc_tab(ctx), n);
    // DST-III reads am and writes b: keep them apart (u1 is free again)
    CK(cudaMemcpyAsync(u1, am, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    k_dst3_scale<<<g, kDstThreads, 0, ctx->stream>>>(b, u1, fbc_f(ctx), fbc_tab(ctx), n, h, p2);
    ctx->launches += 3;
  }
  const int order_star[4] = {0, 1, 2, 3};                 // StarStencil order (src/stencil.jl:16-32)
  const int order_box[8] = {4, 2, 5, 0, 1, 6, 3, 7};      // BoxStencil order (src/stencil.jl:34-90)
  const int *ord = ctx->has_corners ? order_box : order_star;
  const int nord = ctx->has_corners ? 8 : 4;
  const int4 olo = make_int4(ord[0], ord[1], ord[2], ord[3]);
  const int4 ohi = nord == 8 ? make_int4(ord[4], ord[5], ord[6], ord[7]) : make_int4(0, 0, 0, 0);
  if (ctx->fbc_nent > 0) {
    k_setouter_all<<<gridfor((int64_t)ctx->fbc_nent * kM, 128), 128, 0, ctx->stream>>>(
        q, b, fbc_lvs(ctx), fbc_ent(ctx), ctx->fbc_nent, dim, level, (long long)ctx->fbc_root[dim - 1], s, olo, ohi,
        nord);
    ctx->launches++;
  }
  if (b_out) CK(cudaMemcpyAsync(b_out, b, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  CK(cudaGetLastError());
  return SRMG_OK;
}

extern "C" int srmg_fill_ghost_free_dev(srmg_ctx *ctx, double *u, int64_t nblk_alloc, int level) {
  RC(fbc_ready(ctx, nblk_alloc, "srmg_fill_ghost_free"));
  if (!u || level < 1 || level > ctx->nlev) return fail(ctx, SRMG_ERR_BADARG, "srmg_fill_ghost_free: bad level");
  if (level > ctx->fbc_level) return SRMG_OK;
  const int nb = ctx->nblk_host[level - 1];
  if (nb) {
    k_fill_ghost_free<<<gridfor((int64_t)nb * kM, 256), 256, 0, ctx->stream>>>(
        u, fbc_b(ctx), ctx->lv[level - 1].view(level), ctx->fbc_dim, extent(ctx, level, ctx->fbc_dim),
        1 << (ctx->fbc_level - level));
    ctx->launches++;
  }
  CK(cudaGetLastError());
  return SRMG_OK;
}

// Host-array variants (the ccall boundary).
extern "C" int srmg_freebc(srmg_ctx *ctx, double *q, const double *u, int64_t nblk_alloc, double h, double s,
                           double *b_out) {
  RC(fbc_ready(ctx, nblk_alloc, "srmg_freebc"));
  if (!q || !u) return fail(ctx, SRMG_ERR_BADARG, "srmg_freebc: null field");
  double *dq, *du;
  RC(stage_in(ctx, 0, q, nblk_alloc, &dq));
  RC(stage_in(ctx, 1, u, nblk_alloc, &du));
  RC(srmg_freebc_dev(ctx, dq, du, nblk_alloc, h, s, nullptr));
  RC(stage_out(ctx, q, dq, nblk_alloc));
  if (b_out) CK(cudaMemcpyAsync(b_out, fbc_b(ctx), ctx->fbc_n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return SRMG_OK;
}

extern "C" int srmg_fill_ghost_free(srmg_ctx *ctx, double *u, int64_t nblk_alloc, int level) {
  RC(fbc_ready(ctx, nblk_alloc, "srmg_fill_ghost_free"));
  if (!u) return fail(ctx, SRMG_ERR_BADARG, "srmg_fill_ghost_free: null field");
  double *du;
  RC(stage_in(ctx, 0, u, nblk_alloc, &du));
  RC(srmg_fill_ghost_free_dev(ctx, du, nblk_alloc, level));
  RC(stage_out(ctx, u, du, nblk_alloc));
  CK(cudaStreamSynchronize(ctx->stream));
  return SRMG_OK;
}
