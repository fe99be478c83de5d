// Pieces shared by the modality kernels built on the register FFT: launch shapes, the
// FP64 block reduction of loss partials, and generic 2-D transform passes between a
// natural row-major array and the tiled frame layout [tile][row][16].
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <stdint.h>

#include "ptx_pairfft.cuh"
#include "ptx_regfft.cuh"

namespace ptx {

constexpr float kEpsF32 = 1.1920928955078125e-07f;  // torch.finfo(float32).eps
constexpr int kColsPerCta = 8;                        // columns per column-pass CTA

// Copy the N-element row `src` (float2, 8-byte aligned) into `dst` with 16-byte cp.async
// that bypasses L1, element c landing at dst[c + s], s = 1 when src sits 8 bytes past a
// 16-byte boundary (dst must be 16-byte aligned and hold N + 2 elements).  A shifted row
// copies its first and last elements singly so no access leaves the row.  Thread t of the
// T threads of a line copies chunks t + T i; the caller commits, waits and then meets the
// other lanes at a barrier before reading.
template <int N>
__device__ __forceinline__ void copy_row_shifted(float2* dst, const float2* src, int s, int t, uint64_t pol) {
  using S = RegShape<N>;
  if (s == 0) {
#pragma unroll
    for (int i = 0; i < S::N1 / 2; ++i) {
      const int c = 2 * (t + S::T * i);
      cp_async16_hint(dst + c, src + c, pol);
    }
  } else {
#pragma unroll
    for (int i = 0; i < S::N1 / 2; ++i) {
      const int c = 1 + 2 * (t + S::T * i);
      if (c + 1 < N) cp_async16_hint(dst + c + 1, src + c, pol);
    }
    if (t == 0) cp_async8_hint(dst + 1, src, pol);
    if (t == S::T - 1) cp_async8_hint(dst + N, src + N - 1, pol);
  }
}
// 8-byte offset of p from a 16-byte boundary, in float2 elements (0 or 1)
__device__ __forceinline__ int half_shift(const float2* p) {
  return static_cast<int>((reinterpret_cast<uintptr_t>(p) >> 3) & 1);
}

template <int N>
struct RowPass {
  static constexpr int T = RegShape<N>::T;
  static constexpr int LP = row_line_pitch<N>();
  // rows per CTA (a whole number of warps)
  __host__ static int lines(int threads, int rows) {
    int l = threads / T;
    if (l < 1) l = 1;
    const int quantum = T >= 32 ? 1 : 32 / T;
    const int need = ((rows + quantum - 1) / quantum) * quantum;
    return l < need ? l : need;
  }
  __host__ static int smem(int lines) { return lines * LP * (int)sizeof(float2); }
  // exchange buffers plus one prefetched row of N complex values per line
  __host__ static int smem_with_row(int lines) { return lines * (LP + N) * (int)sizeof(float2); }
};

template <int N>
struct ColPass {
  static constexpr int T = RegShape<N>::T;
  static constexpr int LP = col_line_pitch<N>();
  static constexpr int kThreads = kColsPerCta * T;
  static constexpr int kMeasOffsetBytes = ((kColsPerCta * LP * (int)sizeof(float2)) + 15) / 16 * 16;
  static constexpr int kSmemBytes = kMeasOffsetBytes + N * kColsPerCta * (int)sizeof(uint16_t);
};

// ---- observed-amplitude decode table -------------------------------------------------
// lut[c] = sqrtf(float(c) * scale) for every uint16 count c: built once per sweep with the
// same two IEEE operations the per-element decode would use, then read by the epilogues
// (a cached load instead of a square root per element).
constexpr int kLutEntries = 65536;
constexpr size_t kLutBytes = kLutEntries * sizeof(float);

static __global__ void decode_lut_kernel(float* __restrict__ lut, float scale) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < kLutEntries) lut[c] = sqrtf(static_cast<float>(c) * scale);
}

// One launch for everything a sweep resets before its passes: zero two gradient arrays
// (n_a and n_b complex elements), the FP64 loss and the error word, and (lut non-null)
// build the count-decode table.  Grid-stride; any grid size works.
static __global__ void sweep_prologue_kernel(float2* __restrict__ zero_a, size_t n_a, float2* __restrict__ zero_b,
                                             size_t n_b, double* __restrict__ loss, unsigned* __restrict__ err,
                                             float* __restrict__ lut, float scale) {
  pdl_wait();
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t i0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const float2 z = make_float2(0.f, 0.f);
  for (size_t i = i0; i < n_a; i += stride) zero_a[i] = z;
  for (size_t i = i0; i < n_b; i += stride) zero_b[i] = z;
  if (lut) {
    for (size_t c = i0; c < (size_t)kLutEntries; c += stride) lut[c] = sqrtf(static_cast<float>(c) * scale);
  }
  if (i0 == 0) {
    if (loss) *loss = 0.0;
    if (err) *err = 0u;
  }
}

// Grid of sweep_prologue_kernel: about 8 elements per thread, at most 4 waves of 256-thread CTAs.
inline unsigned prologue_blocks(size_t elements, int sms) {
  const size_t want = (elements / 8 + 255) / 256;
  return static_cast<unsigned>(std::max<size_t>(1, std::min<size_t>(want, (size_t)sms * 8 * 4)));
}

// 1/sqrt(s), s > 0: the rsqrtf estimate refined by one Newton-Raphson step for the
// reciprocal square root, y <- y (3 - s y^2) / 2.
__device__ __forceinline__ float rsqrt_nr(float s) {
  const float y = rsqrtf(s);
  return y * fmaf(-0.5f * s, y * y, 1.5f);
}

// |z| and 1 / max(|z|, eps) from one reciprocal square root.
__device__ __forceinline__ void abs_and_inv(float2 z, float eps, float& a, float& inv) {
  const float s2 = cabs2(z);
  const float r = rsqrt_nr(fmaxf(s2, 1e-37f));
  a = s2 * r;
  inv = (a >= eps) ? r : 1.0f / eps;
}

// Sum a per-thread FP64 partial over the block and add it (times `scale`) to *out.
// Every thread of the block must call it; blocks that are not whole warps take the
// shared-memory atomic route (a full-mask shuffle needs all 32 lanes).  Calls may follow one
// another (the staging array is free again when a call returns).
__device__ __forceinline__ void block_add_double(double v, double scale, double* out) {
  __shared__ double red[32];
  const int tid = threadIdx.x;
  if ((blockDim.x & 31) == 0) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((tid & 31) == 0) red[tid >> 5] = v;
    __syncthreads();
    if (tid < 32) {
      const int nw = blockDim.x >> 5;
      double w = (tid < nw) ? red[tid] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
      if (tid == 0) atomicAdd(out, w * scale);
    }
    __syncthreads();  // red is read: a following call may write it
  } else {
    if (tid == 0) red[0] = 0.0;
    __syncthreads();
    atomicAdd(&red[0], v);
    __syncthreads();
    if (tid == 0) atomicAdd(out, red[0] * scale);
  }
}

// ---------------------------------------------------------------------------------------
// Generic 2-D transform passes (unnormalised; INV selects the sign)
// ---------------------------------------------------------------------------------------

// Row pass: in [H][N] natural -> row DFT -> tiled [N/16][H][16].
template <int N, bool INV>
__global__ void __launch_bounds__(256, 2) fft2_rows_kernel(const float2* __restrict__ in, int H,
                                                            float2* __restrict__ tiled,
                                                            const float2* __restrict__ tw, int lines) {
  pdl_wait();
  using S = RegShape<N>;
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x;
  const int l = tid / S::T;
  const int t = tid - l * S::T;
  const int r = blockIdx.x * lines + l;
  const bool row_ok = r < H;
  float2 v[S::N1];
#pragma unroll
  for (int j = 0; j < S::N1; ++j) v[j] = row_ok ? in[(size_t)r * N + t + S::T * j] : make_float2(0.f, 0.f);
  reg_fft<N, INV, false>(v, sm + l * RowPass<N>::LP, t, tw);
  if (row_ok) {
#pragma unroll
    for (int m = 0; m < S::N1; ++m) {
      const int kc = t + S::T * m;
      tiled[((size_t)(kc / kTile) * H + r) * kTile + (kc % kTile)] = v[m];
    }
  }
}

// Column pass: tiled [tiles][N][16] -> column DFT -> out [N][W] natural, times `scale`.
template <int N, bool INV>
__global__ void __launch_bounds__(256, 2) fft2_cols_kernel(const float2* __restrict__ tiled, int W,
                                                            float2* __restrict__ out, float scale,
                                                            const float2* __restrict__ tw) {
  pdl_wait();
  using S = RegShape<N>;
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x;
  const int c = tid % kColsPerCta;
  const int t = tid / kColsPerCta;
  constexpr int kSubs = kTile / kColsPerCta;
  const int ct = blockIdx.x / kSubs;
  const int c0 = ct * kTile + (blockIdx.x - ct * kSubs) * kColsPerCta;
  const int kc = c0 + c;
  const bool col_ok = kc < W;
  const float2* tile = tiled + (size_t)ct * N * kTile + (c0 - ct * kTile);
  float2 v[S::N1];
#pragma unroll
  for (int j = 0; j < S::N1; ++j) v[j] = col_ok ? tile[(t + S::T * j) * kTile + c] : make_float2(0.f, 0.f);
  reg_fft<N, INV, true>(v, sm + c * ColPass<N>::LP, t, tw);
  if (col_ok) {
#pragma unroll
    for (int m = 0; m < S::N1; ++m) out[(size_t)(t + S::T * m) * W + kc] = cscale(v[m], scale);
  }
}

// ---- column pass of a fused sweep on the two-line packed-FP32x2 FFT ------------------
// A CTA owns one 16-column tile of one frame of the tiled scratch [frame][tile][row][16];
// thread (p, t) transforms the column pair (2p, 2p+1) of the tile, both columns in
// lock-step (ptx_pairfft.cuh), so every butterfly, twiddle product and epilogue operation is
// one packed instruction for two columns.  A column pair is one 16-byte load / store per
// row (a warp covers four whole 128-byte tile rows).  The sequence per column: DFT in the
// FIRST_INV direction, scale by `norm`, amplitude-loss epilogue against the counts
// (decoded through `lut`; SHIFTED: the counts are stored fftshifted in both axes), the
// DFT in the other direction, store in place.  The tile's counts arrive by cp.async while
// the first transform runs; the twiddle table sits in shared memory as broadcast pairs.
template <int N>
struct ColPairCfg {
  static constexpr int kPairs = kTile / 2;
  static constexpr int LP4 = RegShape<N>::BUF + 1;  // odd float4 pitch: quarter-warps conflict-free
  static constexpr int kThreads = kPairs * RegShape<N>::T;
  static constexpr int kExchBytes = kPairs * LP4 * (int)sizeof(float4);
  static constexpr int kTwBytes = N * (int)sizeof(float4);
  static constexpr int kMeasBytes = N * kTile * (int)sizeof(uint16_t);
  static constexpr int kSmemBytes = kExchBytes + kTwBytes + kMeasBytes;
};

// UNIT_NORM: `norm` is 1 (the epilogue drops the scaling); FULL: `width` is a multiple of
// the tile, so every column pair exists and the per-column masks go.
// Up to 256-point columns a CTA fits 128 registers per thread and 47 KB of shared memory, so
// four CTAs share an SM (16 warps); longer columns keep two (512) or one (1024).
template <int N>
constexpr int col_pair_min_blocks() {
  return ColPairCfg<N>::kThreads > 128 ? 1 : (N <= 256 ? 4 : 2);
}

template <int N, bool FIRST_INV, bool SHIFTED, bool UNIT_NORM = false, bool FULL = false>
__global__ void __launch_bounds__(ColPairCfg<N>::kThreads, col_pair_min_blocks<N>()) cols_sweep_pair(
    float2* __restrict__ scratch, int width, int frame0, const float2* __restrict__ tw,
    const uint16_t* __restrict__ measured, const float* __restrict__ lut, float norm, float grad_scale,
    double inv_numel, double* __restrict__ loss) {
  pdl_wait();
  using S = RegShape<N>;
  using Cfg = ColPairCfg<N>;
  extern __shared__ float4 sm4[];
  float4* tw4 = sm4 + Cfg::kPairs * Cfg::LP4;
  uint16_t* meas_s = reinterpret_cast<uint16_t*>(tw4 + N);
  const int tid = threadIdx.x;
  const int p = tid % Cfg::kPairs;
  const int t = tid / Cfg::kPairs;
  const int ct = blockIdx.x;
  const int f = blockIdx.y;
  const int c0 = ct * kTile;
  const bool okA = FULL || c0 + 2 * p < width;
  const bool okB = FULL || c0 + 2 * p + 1 < width;
  float2* tile = scratch + ((size_t)f * num_tiles(width) + ct) * N * kTile + 2 * p;
  const size_t g = (size_t)frame0 + f;
  float4* buf = sm4 + p * Cfg::LP4;
  constexpr int kRowOff = SHIFTED ? N / 2 : 0;
  const int col_off = SHIFTED ? width / 2 : 0;

  // counts of rows kr of the tile -> meas_s[kr][16]
  int ic0 = c0 + col_off;
  if (ic0 >= width) ic0 -= width;
  const bool fast = (width % (2 * kTile) == 0) && ((reinterpret_cast<uintptr_t>(measured) & 15) == 0);
  if (fast) {
    for (int i = tid; i < 2 * N; i += blockDim.x) {
      const int kr = i >> 1, h = (i & 1) * 8;
      const int ir = (kr + kRowOff) & (N - 1);
      cp_async16(meas_s + kr * kTile + h, measured + (g * N + ir) * width + ic0 + h);
    }
    cp_async_commit();
  } else {
    for (int i = tid; i < N * kTile; i += blockDim.x) {
      const int kr = i / kTile, cc = i - kr * kTile;
      const int ir = (kr + kRowOff) & (N - 1);
      int icc = c0 + cc + col_off;
      if (icc >= width) icc -= width;
      meas_s[i] = (c0 + cc < width) ? measured[(g * N + ir) * width + icc] : 0;
    }
  }
  for (int i = tid; i < N; i += blockDim.x) {
    const float2 w = __ldg(&tw[i]);
    tw4[i] = make_float4(w.x, w.x, w.y, w.y);
  }
  const uint64_t pol = policy_evict_first();
  CPair v[S::N1];
#pragma unroll
  for (int j = 0; j < S::N1; ++j) {
    float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
    if (okA) q = ld_stream4(tile + (t + S::T * j) * kTile, pol);
    if (!okB) q.z = q.w = 0.f;
    v[j] = {make_float2(q.x, q.z), make_float2(q.y, q.w)};
  }
  __syncthreads();  // twiddle table
  pair_fft<N, FIRST_INV, true>(v, buf, t, tw4);
  cp_async_wait_all();
  __syncthreads();
  float2 part = make_float2(0.f, 0.f);  // squared residuals of the two columns
  const float2 gs = f2(grad_scale);
  const float2 nrm = f2(norm);
#pragma unroll
  for (int m = 0; m < S::N1; ++m) {
    const int kr = t + S::T * m;
    const CPair F = UNIT_NORM ? v[m] : CPair{mul2(v[m].re, nrm), mul2(v[m].im, nrm)};
    const float2 s2 = fma2(F.re, F.re, mul2(F.im, F.im));
    // rsqrt_nr on both lanes, its Newton-Raphson step in packed form (the same IEEE operations)
    const float2 sc2 = make_float2(fmaxf(s2.x, 1e-37f), fmaxf(s2.y, 1e-37f));
    const float2 y0 = make_float2(rsqrtf(sc2.x), rsqrtf(sc2.y));
    const float2 r = mul2(y0, fma2(mul2(f2(-0.5f), sc2), mul2(y0, y0), f2(1.5f)));
    const float2 a = mul2(s2, r);
    const float2 inv =
        make_float2(a.x >= kEpsF32 ? r.x : 1.0f / kEpsF32, a.y >= kEpsF32 ? r.y : 1.0f / kEpsF32);
    const uint32_t cnt = *reinterpret_cast<const uint32_t*>(meas_s + kr * kTile + 2 * p);
    const float2 y = make_float2(okA ? __ldg(&lut[cnt & 0xffffu]) : 0.f, okB ? __ldg(&lut[cnt >> 16]) : 0.f);
    float2 rr = sub2(a, y);
    rr = make_float2(okA ? rr.x : 0.f, okB ? rr.y : 0.f);
    part = fma2(rr, rr, part);
    const float2 sc = mul2(mul2(gs, rr), inv);
    v[m] = {mul2(F.re, sc), mul2(F.im, sc)};
  }
  pair_fft<N, !FIRST_INV, true>(v, buf, t, tw4);
  if (okA) {
#pragma unroll
    for (int m = 0; m < S::N1; ++m) {
      *reinterpret_cast<float4*>(tile + (t + S::T * m) * kTile) =
          make_float4(v[m].re.x, v[m].im.x, v[m].re.y, v[m].im.y);
    }
  }
  block_add_double(static_cast<double>(part.x) + static_cast<double>(part.y), inv_numel, loss);
}

}  // namespace ptx
