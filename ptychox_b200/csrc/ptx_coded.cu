// Coded and near-field ptychography: forward, adjoint and the fused sweep.
//
// Math (python/ptychoX/coded/ops.py:136-171; near-field = transfer_1 = 1, the MATLAB
// sequence fwd_adPtychoX_nearf.cu:58-114 without the first transfer function):
//   O^ = fft2(O);  x_b = ifft2(O^ T1 R_b)     R_b = exp(2 pi i (dx_b fx + dy_b fy))
//   s_b = ifft2(fft2(x_b M) T2);  A_b = sqrt(avgpool_ds |s_b|^2)
// Adjoint (the vector-Jacobian product autograd takes through that forward; step order as
// in coded_kernel.cu:347-424):
//   g_s = g / (A ds^2) s;  g_a = ifft2(fft2(g_s) conj(T2));  grad_M += g_a conj(x)
//   g_X = fft2(g_a conj(M)) / n;  grad_O^ += g_X conj(T1 R_b);  grad_O = n ifft2(grad_O^)
//
// With unnormalised transforms D (forward) and D* (inverse), every 2-D transform is a
// row pass and a column pass, and consecutive 1-D transforms along the same axis with a
// pointwise step between them share one pass.  Seven passes per frame:
//   1 col: load O^ T1 R_b, inverse column DFT                                  -> frame
//   2 row: inverse row DFT, x = ./n (stored), a = x M, forward row DFT          -> frame
//   3 col: forward column DFT, x T2, inverse column DFT                         -> frame
//   4 row: inverse row DFT, s = ./n, RMS pool, FP64 loss, g_s, forward row DFT  -> frame
//   5 col: forward column DFT, x conj(T2)/n, inverse column DFT                 -> frame
//   6 row: inverse row DFT (g_a), grad_M += g_a conj(x) in registers,
//          g_a conj(M), forward row DFT                                         -> frame
//   7 col: forward column DFT, /n, grad_O^ += . conj(T1 R_b) (float2 atomics)
// O^ = D(O) before the frames and grad_O = D*(grad_O^) after them use the generic 2-D
// passes.  The phase ramp's argument is reduced exactly in FP32 (FMA two-product and
// integer rounding) before sincospif, so the ramp is accurate to ~1 ulp of a turn.  Field
// sides that are {2,3,5}-smooth but not powers of two run the same passes on the mixed-radix
// kernels of ptx_mixcoded.cuh through the same workspace layout.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>

#include "ptx_internal.h"
#include "ptx_passes.cuh"

namespace ptx {
namespace {

constexpr size_t kHdr = 256;
enum CodedMode { kCodedSweep = 0, kCodedForward = 1, kCodedBackward = 2 };
constexpr float kAmpFloor = 1e-30f;  // keeps g / A finite when a pooled amplitude is exactly 0

// exp(2 pi i (dx fx + dy fy)) for signed integer frequencies fx, fy.
__device__ __forceinline__ float2 shift_ramp(float dx, float dy, int fx, int fy) {
  const float ffx = static_cast<float>(fx), ffy = static_cast<float>(fy);
  const float px = dx * ffx, py = dy * ffy;
  const float ex = fmaf(dx, ffx, -px), ey = fmaf(dy, ffy, -py);  // exact product remainders
  const float t = (px - rintf(px)) + (py - rintf(py)) + (ex + ey);  // turns, |t| < ~1
  float s, c;
  sincospif(2.0f * t, &s, &c);
  return make_float2(c, s);
}

__device__ __forceinline__ int signed_freq(int k, int n) { return k < n / 2 ? k : k - n; }

// ---- column passes ---------------------------------------------------------------------
// STAGE 1: load O^ T1 R, inverse DFT.  STAGE 3: forward DFT, x T2 (or conj(T2)/n when
// CONJ), inverse DFT.  STAGE 7: forward DFT, /n, grad_O^ += . conj(T1 R).
template <int STAGE, bool CONJ, int N>
__global__ void __launch_bounds__(256, 2) coded_cols(
    float2* __restrict__ scratch, const float2* __restrict__ ospec, const float2* __restrict__ t1,
    const float2* __restrict__ t2, const float* __restrict__ shifts, float inv_n, float2* __restrict__ grad_ospec,
    const float2* __restrict__ tw, double* __restrict__ grad_shifts) {
  using S = RegShape<N>;
  using CP = ColPass<N>;
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x;
  const int c = tid % kColsPerCta;
  const int t = tid / kColsPerCta;
  constexpr int kSubs = kTile / kColsPerCta;
  constexpr int kTiles = (N + kTile - 1) / kTile;
  const int ct = blockIdx.x / kSubs;
  const int c0 = ct * kTile + (blockIdx.x - ct * kSubs) * kColsPerCta;
  const int f = blockIdx.y;
  const int kc = c0 + c;
  const bool col_ok = kc < N;
  float2* tile = scratch + ((size_t)f * kTiles + ct) * N * kTile + (c0 - ct * kTile);
  float2* buf = sm + c * CP::LP;
  float2 v[S::N1];
  const float dx = (STAGE == 1 || STAGE == 7) ? shifts[2 * f] : 0.f;
  const float dy = (STAGE == 1 || STAGE == 7) ? shifts[2 * f + 1] : 0.f;
  const int fx = signed_freq(kc, N);

  if (STAGE == 1) {
#pragma unroll
    for (int j = 0; j < S::N1; ++j) {
      const int kr = t + S::T * j;
      float2 w = make_float2(0.f, 0.f);
      if (col_ok) {
        const size_t idx = (size_t)kr * N + kc;
        w = cmul(ospec[idx], shift_ramp(dx, dy, fx, signed_freq(kr, N)));
        if (t1) w = cmul(w, t1[idx]);
      }
      v[j] = w;
    }
    reg_fft<N, true, true>(v, buf, t, tw);
  } else {
#pragma unroll
    for (int j = 0; j < S::N1; ++j) v[j] = col_ok ? tile[(t + S::T * j) * kTile + c] : make_float2(0.f, 0.f);
    reg_fft<N, false, true>(v, buf, t, tw);
    if (STAGE == 3) {
#pragma unroll
      for (int m = 0; m < S::N1; ++m) {
        const int kr = t + S::T * m;
        if (col_ok) {
          const float2 h = t2[(size_t)kr * N + kc];
          v[m] = CONJ ? cscale(cmulc(v[m], h), inv_n) : cmul(v[m], h);
        }
      }
      reg_fft<N, true, true>(v, buf, t, tw);
    } else {  // STAGE 7
      // with grad_shifts: dL/d(dx, dy) += -2 pi sum (fx, fy) Im(conj(G) u), G = v / n the
      // gradient of u = O^ T1 R (the ramp is the only place the shifts enter)
      float sx = 0.f, sy = 0.f;
      if (col_ok) {
#pragma unroll
        for (int m = 0; m < S::N1; ++m) {
          const int kr = t + S::T * m;
          const size_t idx = (size_t)kr * N + kc;
          float2 w = shift_ramp(dx, dy, fx, signed_freq(kr, N));
          if (t1) w = cmul(w, t1[idx]);
          const float2 G = cscale(v[m], inv_n);
          atomicAdd(&grad_ospec[idx], cmulc(G, w));
          if (grad_shifts) {
            const float2 u = cmul(ospec[idx], w);
            const float im = fmaf(G.x, u.y, -G.y * u.x);  // Im(conj(G) u)
            sx = fmaf(static_cast<float>(fx), im, sx);
            sy = fmaf(static_cast<float>(signed_freq(kr, N)), im, sy);
          }
        }
      }
      if (grad_shifts) {
        constexpr double kTwoPi = 6.283185307179586476925286766559;
        block_add_double(static_cast<double>(sx), -kTwoPi, &grad_shifts[2 * f]);
        block_add_double(static_cast<double>(sy), -kTwoPi, &grad_shifts[2 * f + 1]);
      }
      return;
    }
  }
  if (col_ok) {
#pragma unroll
    for (int m = 0; m < S::N1; ++m) tile[(t + S::T * m) * kTile + c] = v[m];
  }
}

// Stage 3 on the two-line packed FFT: a CTA owns one 16-column tile of one frame; thread
// (p, t) transforms the column pair (2p, 2p+1) in lock-step (forward DFT, x T2 or
// conj(T2)/n, inverse DFT).  One 16-byte load / store per row and column pair.
template <bool CONJ, int N>
__global__ void __launch_bounds__(ColPairCfg<N>::kThreads, ColPairCfg<N>::kThreads <= 128 ? 2 : 1) coded_cols_filter_pair(
    float2* __restrict__ scratch, const float2* __restrict__ t2, float inv_n, const float2* __restrict__ tw) {
  using S = RegShape<N>;
  using Cfg = ColPairCfg<N>;
  constexpr int kTiles = (N + kTile - 1) / kTile;
  extern __shared__ float4 sm4[];
  float4* tw4 = sm4 + Cfg::kPairs * Cfg::LP4;
  const int tid = threadIdx.x;
  const int p = tid % Cfg::kPairs;
  const int t = tid / Cfg::kPairs;
  const int ct = blockIdx.x;
  const int f = blockIdx.y;
  const int c = ct * kTile + 2 * p;  // line A column (line B: c + 1; N is a multiple of 16)
  float2* tile = scratch + ((size_t)f * kTiles + ct) * N * kTile + 2 * p;
  float4* buf = sm4 + p * Cfg::LP4;
  for (int i = tid; i < N; i += blockDim.x) {
    const float2 w = __ldg(&tw[i]);
    tw4[i] = make_float4(w.x, w.x, w.y, w.y);
  }
  const uint64_t pol = policy_evict_first();
  CPair v[S::N1];
#pragma unroll
  for (int j = 0; j < S::N1; ++j) {
    const float4 q = ld_stream4(tile + (t + S::T * j) * kTile, pol);
    v[j] = {make_float2(q.x, q.z), make_float2(q.y, q.w)};
  }
  __syncthreads();  // twiddle table
  pair_fft<N, false, true>(v, buf, t, tw4);
  const float2 sc = f2(inv_n);
#pragma unroll
  for (int m = 0; m < S::N1; ++m) {
    const int kr = t + S::T * m;
    const float4 q = __ldg(reinterpret_cast<const float4*>(t2 + (size_t)kr * N + c));
    const float2 hre = make_float2(q.x, q.z), him = make_float2(q.y, q.w);
    const CPair a = v[m];
    if (CONJ) {  // cscale(cmulc(a, h), inv_n)
      v[m] = {mul2(fma2(a.re, hre, mul2(a.im, him)), sc), mul2(fma2(a.im, hre, mul2(a.re, neg2(him))), sc)};
    } else {  // cmul(a, h)
      v[m] = {fma2(a.re, hre, mul2(a.im, neg2(him))), fma2(a.re, him, mul2(a.im, hre))};
    }
  }
  pair_fft<N, true, true>(v, buf, t, tw4);
#pragma unroll
  for (int m = 0; m < S::N1; ++m) {
    *reinterpret_cast<float4*>(tile + (t + S::T * m) * kTile) = make_float4(v[m].re.x, v[m].im.x, v[m].re.y, v[m].im.y);
  }
}

// ---- row passes ------------------------------------------------------------------------

template <int N>
__device__ __forceinline__ void load_frame_row(const float2* __restrict__ scratch, int f, int r,
                                               float2 (&v)[RegShape<N>::N1], int t) {
  using S = RegShape<N>;
  constexpr int kTiles = (N + kTile - 1) / kTile;
  const float2* base = scratch + (size_t)f * kTiles * N * kTile + (size_t)r * kTile;
#pragma unroll
  for (int j = 0; j < S::N1; ++j) {
    const int c = t + S::T * j;
    v[j] = base[(size_t)(c / kTile) * N * kTile + (c % kTile)];
  }
}

// Frame row r of frame f loaded straight into registers with loads that do not allocate in
// L1 (the frames stream through once per pass; L1 is left to the twiddles and masks).
template <int N>
__device__ __forceinline__ void load_frame_row_stream(const float2* __restrict__ scratch, int f, int r,
                                                      float2 (&v)[RegShape<N>::N1], int t, uint64_t pol) {
  using S = RegShape<N>;
  constexpr int kTiles = (N + kTile - 1) / kTile;
  const float2* base = scratch + (size_t)f * kTiles * N * kTile + (size_t)r * kTile;
#pragma unroll
  for (int j = 0; j < S::N1; ++j) {
    const int c = t + S::T * j;
    const float4 q = ld_stream4(base + (size_t)(c / kTile) * N * kTile + (c % kTile) - (c & 1), pol);
    v[j] = (c & 1) ? make_float2(q.z, q.w) : make_float2(q.x, q.y);
  }
}
// Frame row r of frame f into the line buffer `dst` (element c at dst[c]) by 16-byte
// cp.async that bypasses L1; thread t of the line's T threads copies chunks t + T i, so the
// line meets at a warp barrier after the wait before reading.
template <int N>
__device__ __forceinline__ void prefetch_frame_row(float2* dst, const float2* __restrict__ scratch, int f, int r,
                                                   int t, uint64_t pol) {
  using S = RegShape<N>;
  constexpr int kTiles = (N + kTile - 1) / kTile;
  const float2* base = scratch + (size_t)f * kTiles * N * kTile + (size_t)r * kTile;
#pragma unroll
  for (int i = 0; i < S::N1 / 2; ++i) {
    const int c = 2 * (t + S::T * i);
    cp_async16_hint(dst + c, base + (size_t)(c / kTile) * N * kTile + (c % kTile), pol);
  }
  cp_async_commit();
}

template <int N>
__device__ __forceinline__ void store_frame_row(float2* __restrict__ scratch, int f, int r,
                                                const float2 (&v)[RegShape<N>::N1], int t) {
  using S = RegShape<N>;
  constexpr int kTiles = (N + kTile - 1) / kTile;
  float2* base = scratch + (size_t)f * kTiles * N * kTile + (size_t)r * kTile;
#pragma unroll
  for (int m = 0; m < S::N1; ++m) {
    const int c = t + S::T * m;
    base[(size_t)(c / kTile) * N * kTile + (c % kTile)] = v[m];
  }
}

// Shared memory of the persistent coded row passes, per line: the exchange / landing line
// (BP), then `rows` further rows of N values (mask row; x row); per CTA the twiddle table
// laid out by thread.
template <int N>
struct CodedRowCfg {
  static constexpr int BP = RowPass<N>::LP > N ? RowPass<N>::LP : N;
  static_assert(BP % 2 == 0, "16-byte landing lines");
  static int smem(int lines, int rows) { return (lines * (BP + rows * N) + N) * (int)sizeof(float2); }
};

// Pass 2: inverse row DFT, x = ./n (stored), a = x M, forward row DFT.  Work units are
// (row group, frame) pairs in row-group-major order over one wave of resident CTAs (CTA b
// takes the contiguous units [u0, u1)); the mask rows of the current row group and the
// twiddle table sit in shared memory, and the next unit's frame row is requested by
// cp.async as soon as this unit's transforms have released the line buffer.
template <int N>
__global__ void __launch_bounds__(128, 3) coded_rows_mask(float2* __restrict__ scratch,
                                                          const float2* __restrict__ mask,
                                                          float2* __restrict__ xstore, float inv_n, int nframes,
                                                          int rowgroups, const float2* __restrict__ tw, int lines) {
  using S = RegShape<N>;
  using Cfg = CodedRowCfg<N>;
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x;
  const int l = tid / S::T;
  const int t = tid - l * S::T;
  const long long units = (long long)rowgroups * nframes;
  const long long u0 = units * blockIdx.x / gridDim.x;
  const long long u1 = units * (blockIdx.x + 1) / gridDim.x;
  if (u0 >= u1) return;
  int g = static_cast<int>(u0 / nframes);
  int f = static_cast<int>(u0 - (long long)g * nframes);
  float2* buf = sm + l * Cfg::BP;
  float2* mbuf = sm + lines * Cfg::BP + l * N;
  float2* tws = sm + lines * (Cfg::BP + N);
  load_twiddles_by_thread<N>(tws, tw);
  __syncthreads();
  const uint64_t pol_first = policy_evict_first();
  int r = g * lines + l;
  if (r < N) prefetch_frame_row<N>(buf, scratch, f, r, t, pol_first);
  bool new_group = true;
  for (long long u = u0; u < u1; ++u) {
    const bool row_ok = r < N;
    if (new_group && row_ok) {
#pragma unroll
      for (int m = 0; m < S::N1; ++m) mbuf[t + S::T * m] = __ldg(&mask[(size_t)r * N + t + S::T * m]);
    }
    new_group = false;
    cp_async_wait_all();
    __syncwarp();
    float2 v[S::N1];
#pragma unroll
    for (int j = 0; j < S::N1; ++j) v[j] = row_ok ? buf[t + S::T * j] : make_float2(0.f, 0.f);
    __syncwarp();
    reg_fft<N, true, false, true>(v, buf, t, tws);
    float2* xrow = xstore + ((size_t)f * N + (row_ok ? r : 0)) * N;
#pragma unroll
    for (int m = 0; m < S::N1; ++m) {
      const int c = t + S::T * m;
      const float2 x = cscale(v[m], inv_n);
      if (row_ok) xrow[c] = x;
      v[m] = cmul(x, mbuf[c]);
    }
    reg_fft<N, false, false, true>(v, buf, t, tws);
    const bool more = u + 1 < u1;
    int gn = g, fn = f + 1;
    if (fn == nframes) {
      gn = g + 1;
      fn = 0;
    }
    const int rn = gn * lines + l;
    if (more && rn < N) prefetch_frame_row<N>(buf, scratch, fn, rn, t, pol_first);
    if (row_ok) store_frame_row<N>(scratch, f, r, v, t);
    if (gn != g) new_group = true;
    g = gn;
    f = fn;
    r = rn;
  }
}

// Pass 4.  kCodedSweep: inverse row DFT, s = ./n, RMS pool over ds x ds, FP64 loss,
// g_s = gA / (A ds^2) s, forward row DFT.  kCodedForward: inverse row DFT, write s and
// the pooled amplitude.  kCodedBackward: g_s from saved s, amplitude and grad_output,
// forward row DFT.  A CTA owns `lines` consecutive rows, a multiple of ds.
template <int MODE, int N>
__global__ void __launch_bounds__(256, 2) coded_rows_pool(
    float2* __restrict__ scratch, int ds, int frame0, float inv_n, const uint16_t* __restrict__ measured,
    float scale, float grad_scale, double inv_numel, double* __restrict__ loss, float2* __restrict__ sensor,
    float* __restrict__ amplitude, const float* __restrict__ grad_output, const float2* __restrict__ tw,
    int lines) {
  using S = RegShape<N>;
  extern __shared__ float2 sm[];
  float* pool = reinterpret_cast<float*>(sm + lines * RowPass<N>::LP);  // [lines][N] |s|^2, then factors
  float2* tws = reinterpret_cast<float2*>(pool + lines * N);             // twiddles by thread
  load_twiddles_by_thread<N>(tws, tw);
  __syncthreads();
  const int tid = threadIdx.x;
  const int l = tid / S::T;
  const int t = tid - l * S::T;
  const int r0 = blockIdx.x * lines;
  const int r = r0 + l;
  const int f = blockIdx.y;
  const size_t g = (size_t)frame0 + f;
  const int lw = N / ds;  // pooled width
  float2 v[S::N1];
  if (MODE == kCodedBackward) {
    const float2* srow = sensor + (g * N + r) * N;
    const float* arow = amplitude + (g * lw + r / ds) * lw;
    const float* grow = grad_output + (g * lw + r / ds) * lw;
#pragma unroll
    for (int m = 0; m < S::N1; ++m) {
      const int c = t + S::T * m;
      const float a = fmaxf(arow[c / ds], kAmpFloor);
      v[m] = cscale(srow[c], grow[c / ds] / (a * static_cast<float>(ds * ds)));
    }
  } else {
    load_frame_row_stream<N>(scratch, f, r, v, t, policy_evict_first());
    reg_fft<N, true, false, true>(v, sm + l * RowPass<N>::LP, t, tws);
#pragma unroll
    for (int m = 0; m < S::N1; ++m) {
      v[m] = cscale(v[m], inv_n);
      pool[l * N + t + S::T * m] = cabs2(v[m]);
    }
    __syncthreads();
    // pooled values of this CTA: (lines/ds) x lw, one per thread-iteration
    const int nb = (lines / ds) * lw;
    double acc = 0.0;
    for (int q = tid; q < nb; q += blockDim.x) {
      const int py = q / lw, px = q - py * lw;
      float sum = 0.f;
      for (int yy = 0; yy < ds; ++yy)
        for (int xx = 0; xx < ds; ++xx) sum += pool[(py * ds + yy) * N + px * ds + xx];
      const float a = sqrtf(fmaxf(sum / static_cast<float>(ds * ds), 0.f));
      const size_t oidx = (g * lw + r0 / ds + py) * lw + px;
      if (MODE == kCodedForward) {
        amplitude[oidx] = a;
      } else {
        const float y = sqrtf(static_cast<float>(measured[oidx]) * scale);
        const float d = a - y;
        acc += static_cast<double>(d) * static_cast<double>(d);
        // store the factor gA / (A ds^2) at the block's first pixel
        pool[(py * ds) * N + px * ds] = grad_scale * d / (fmaxf(a, kAmpFloor) * static_cast<float>(ds * ds));
      }
    }
    if (MODE == kCodedForward) {
      float2* srow = sensor + (g * N + r) * N;
#pragma unroll
      for (int m = 0; m < S::N1; ++m) srow[t + S::T * m] = v[m];
      return;
    }
    block_add_double(acc, inv_numel, loss);  // synchronises the block
#pragma unroll
    for (int m = 0; m < S::N1; ++m) {
      const int c = t + S::T * m;
      v[m] = cscale(v[m], pool[((l / ds) * ds) * N + (c / ds) * ds]);
    }
  }
  reg_fft<N, false, false, true>(v, sm + l * RowPass<N>::LP, t, tws);
  store_frame_row<N>(scratch, f, r, v, t);
}

// Pass 6: inverse row DFT (g_a), grad_M += g_a conj(x) in registers over the CTA's frames,
// g_a conj(M), forward row DFT.
template <int N>
__global__ void __launch_bounds__(128, 2) coded_rows_grad_mask(
    float2* __restrict__ scratch, const float2* __restrict__ mask, const float2* __restrict__ xstore, int nframes,
    int rowgroups, float2* __restrict__ grad_mask, const float2* __restrict__ tw, int lines) {
  using S = RegShape<N>;
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x;
  const int l = tid / S::T;
  const int t = tid - l * S::T;
  // (row group, frame) units in row-group-major order; the grid is one wave of resident
  // CTAs and CTA b takes the contiguous units [u0, u1)
  const long long units = (long long)rowgroups * nframes;
  const long long u0 = units * blockIdx.x / gridDim.x;
  const long long u1 = units * (blockIdx.x + 1) / gridDim.x;
  if (u0 >= u1) return;
  int g = static_cast<int>(u0 / nframes);
  int f = static_cast<int>(u0 - (long long)g * nframes);
  using Cfg = CodedRowCfg<N>;
  float2* buf = sm + l * Cfg::BP;
  float2* xbuf = sm + lines * Cfg::BP + l * 2 * N;
  float2* mbuf = xbuf + N;
  float2* tws = sm + lines * (Cfg::BP + 2 * N);
  load_twiddles_by_thread<N>(tws, tw);
  __syncthreads();
  const uint64_t pol_first = policy_evict_first();
  float2 acc[S::N1];
#pragma unroll
  for (int m = 0; m < S::N1; ++m) acc[m] = make_float2(0.f, 0.f);
  bool new_group = true;
  for (long long u = u0; u < u1; ++u) {
    const int r = g * lines + l;
    const bool row_ok = r < N;
    const int rr = row_ok ? r : 0;
    if (new_group && row_ok) {
#pragma unroll
      for (int m = 0; m < S::N1; ++m) mbuf[t + S::T * m] = __ldg(&mask[(size_t)r * N + t + S::T * m]);
    }
    new_group = false;
    const float2* xrow = xstore + ((size_t)f * N + rr) * N;
    prefetch_frame_row<N>(buf, scratch, f, rr, t, pol_first);
#pragma unroll
    for (int i = 0; i < S::N1 / 2; ++i) {
      const int c = 2 * (t + S::T * i);
      cp_async16_hint(xbuf + c, xrow + c, pol_first);
    }
    cp_async_commit();
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");  // the frame row
    __syncwarp();
    float2 v[S::N1];
#pragma unroll
    for (int j = 0; j < S::N1; ++j) v[j] = buf[t + S::T * j];
    __syncwarp();
    reg_fft<N, true, false, true>(v, buf, t, tws);
    cp_async_wait_all();  // the x row
    __syncwarp();
#pragma unroll
    for (int m = 0; m < S::N1; ++m) {
      const int c = t + S::T * m;
      acc[m] = cadd(acc[m], cmulc(v[m], xbuf[c]));
      v[m] = cmulc(v[m], mbuf[c]);
    }
    reg_fft<N, false, false, true>(v, buf, t, tws);
    if (row_ok) store_frame_row<N>(scratch, f, r, v, t);
    int gn = g, fn = f + 1;
    if (fn == nframes) {
      gn = g + 1;
      fn = 0;
    }
    if (u + 1 == u1 || gn != g) {
      new_group = true;
      // leaving this row group: fold its mask-gradient partial sums into grad_mask
      if (row_ok) {
#pragma unroll
        for (int m = 0; m < S::N1; ++m) {
          atomicAdd(&grad_mask[(size_t)r * N + t + S::T * m], acc[m]);
          acc[m] = make_float2(0.f, 0.f);
        }
      }
    }
    g = gn;
    f = fn;
  }
}

// ---- finite-difference data loss ---------------------------------------------------------
// fd_loss of train_coded.py:101-107 on the pooled amplitudes A [batch, h, w] against the
// decoded counts Y = sqrt(I scale): D = A - Y, dx = D(y, x+1) - D, dy = D(y+1, x) - D
// (periodic), loss = sum sqrt(dx^2 + dy^2 + 1e-5) (isotropic) or sum |dx| + |dy|, and
// dL/dA = -(ux + uy)(y, x) + ux(y, x-1) + uy(y-1, x) with (ux, uy) = (dx, dy) / m or the
// signs.  One thread per pixel; the 7-point neighbourhood of D is re-derived from A and I.
__device__ __forceinline__ float fd_diff(const float* __restrict__ amp, const uint16_t* __restrict__ meas,
                                         size_t base, int h, int w, int y, int x, float scale) {
  y = y < 0 ? y + h : (y >= h ? y - h : y);
  x = x < 0 ? x + w : (x >= w ? x - w : x);
  const size_t i = base + (size_t)y * w + x;
  return amp[i] - sqrtf(static_cast<float>(meas[i]) * scale);
}

__device__ __forceinline__ void fd_unit(float dx, float dy, bool isotropic, float& ux, float& uy, float& m) {
  if (isotropic) {
    m = sqrtf(fmaf(dx, dx, fmaf(dy, dy, 1e-5f)));
    ux = dx / m;
    uy = dy / m;
  } else {
    m = fabsf(dx) + fabsf(dy);
    ux = dx > 0.f ? 1.f : (dx < 0.f ? -1.f : 0.f);
    uy = dy > 0.f ? 1.f : (dy < 0.f ? -1.f : 0.f);
  }
}

__global__ void __launch_bounds__(256) fd_loss_kernel(const float* __restrict__ amp, const uint16_t* __restrict__ meas,
                                                      float scale, long long total, int h, int w, int isotropic,
                                                      float* __restrict__ grad_amp, double* __restrict__ loss) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double part = 0.0;
  if (i < total) {
    const long long hw = (long long)h * w;
    const long long b = i / hw;
    const int y = static_cast<int>((i - b * hw) / w);
    const int x = static_cast<int>(i - b * hw - (long long)y * w);
    const size_t base = (size_t)(b * hw);
    const bool iso = isotropic != 0;
    const float d = fd_diff(amp, meas, base, h, w, y, x, scale);
    const float dr = fd_diff(amp, meas, base, h, w, y, x + 1, scale);
    const float dd = fd_diff(amp, meas, base, h, w, y + 1, x, scale);
    const float dl = fd_diff(amp, meas, base, h, w, y, x - 1, scale);
    const float ddl = fd_diff(amp, meas, base, h, w, y + 1, x - 1, scale);
    const float du = fd_diff(amp, meas, base, h, w, y - 1, x, scale);
    const float dur = fd_diff(amp, meas, base, h, w, y - 1, x + 1, scale);
    float ux, uy, m, uxl, uyl, ml, uxu, uyu, mu;
    fd_unit(dr - d, dd - d, iso, ux, uy, m);           // this pixel's term
    fd_unit(d - dl, ddl - dl, iso, uxl, uyl, ml);      // left neighbour's term
    fd_unit(dur - du, d - du, iso, uxu, uyu, mu);      // upper neighbour's term
    grad_amp[i] = -(ux + uy) + uxl + uyu;
    part = static_cast<double>(m);
  }
  block_add_double(part, 1.0, loss);
}

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------

struct CodedGeom {
  int n, ds, batch;
  LinePlan plan;
  const MixCodedOps* mix;  // non-null: the mixed-radix passes (side not a power of two)
  const MixFpmOps* mfft;   // their 2-D transforms of the object spectrum
  size_t field_bytes;
  int chunk;
  float2* ospec;
  float2* gospec;
  float2* tmp;
  float2* xstore;
  float2* frames;
};

// A field n x n in natural layout, and one in the tiled frame layout [tile][row][16] (the
// same when 16 divides n).
size_t field_bytes_of(int n) { return (size_t)n * n * sizeof(float2); }
size_t tiled_bytes_of(int n) { return (size_t)num_tiles(n) * kTile * n * sizeof(float2); }
// object spectrum and its gradient (natural), the 2-D transforms' temporary (tiled)
size_t coded_fixed_bytes(int n) { return kHdr + 2 * field_bytes_of(n) + tiled_bytes_of(n); }

int coded_lines(int n) {
  int lines = 0;
  dispatch_pow2(n, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    lines = RowPass<N>::lines(256, N);
  });
  return lines;
}

int coded_check(int n, int ds, const void* a, const void* b, const void* t2, const float* shifts, int batch, void* ws,
                size_t ws_bytes, bool need_xstore, CodedGeom* g) {
  if (!a || !b || !t2 || (!shifts && batch > 0) || !ws) return set_error(PTX_ERR_INVALID_ARGUMENT, "null pointer argument");
  if (batch < 0) return set_error(PTX_ERR_INVALID_ARGUMENT, "negative batch");
  if (reinterpret_cast<uintptr_t>(ws) & 255) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "workspace must start on a 256-byte boundary");
  }
  const bool pow2 = is_pow2_len(n) && n >= 16;
  g->mix = pow2 ? nullptr : mix_coded_ops(n);
  g->mfft = pow2 ? nullptr : mix_fpm_ops(n);
  if (!pow2 && !(g->mix && g->mfft)) {
    return set_error(PTX_ERR_UNSUPPORTED_SIZE, "coded field side must be 2^a 3^b 5^c in [16, 1024] (got %d)", n);
  }
  if (pow2) {
    const int lines = coded_lines(n);
    if (ds < 1 || n % ds != 0 || lines % ds != 0) {
      return set_error(PTX_ERR_UNSUPPORTED_SIZE, "downsample %d must divide %d and %d", ds, n, lines);
    }
  } else if (ds < 1 || n % ds != 0) {
    return set_error(PTX_ERR_UNSUPPORTED_SIZE, "downsample %d must divide %d", ds, n);
  }
  g->n = n; g->ds = ds; g->batch = batch;
  if (int st = get_line_plan(n, &g->plan)) return st;
  if (!pow2 && !g->plan.mix_twt) return set_error(PTX_ERR_UNSUPPORTED_SIZE, "no mixed-radix twiddle tables for %d", n);
  g->field_bytes = field_bytes_of(n);
  const size_t tiled = tiled_bytes_of(n);
  const size_t fixed = coded_fixed_bytes(n);
  const size_t per = tiled + (need_xstore ? g->field_bytes : 0);  // a frame and its stored x
  if (ws_bytes < fixed + per) {
    return set_error(PTX_ERR_WORKSPACE, "workspace of %zu bytes is smaller than the %zu bytes needed", ws_bytes,
                     fixed + per);
  }
  // frames per chunk: what the workspace holds, at most the batch and 65535 (a grid dimension)
  g->chunk = static_cast<int>(std::min<size_t>({(ws_bytes - fixed) / per, (size_t)std::max(batch, 1), (size_t)65535}));
  char* p = static_cast<char*>(ws) + kHdr;
  g->ospec = reinterpret_cast<float2*>(p);
  g->gospec = reinterpret_cast<float2*>(p + g->field_bytes);
  g->tmp = reinterpret_cast<float2*>(p + 2 * g->field_bytes);
  g->frames = reinterpret_cast<float2*>(p + 2 * g->field_bytes + tiled);
  g->xstore = need_xstore ? reinterpret_cast<float2*>(p + 2 * g->field_bytes + tiled + (size_t)g->chunk * tiled)
                          : nullptr;
  if (g->mix) {
    int st = g->mix->prepare(ds);
    if (!st) st = g->mfft->prepare();
    return st;
  }
  const int lines = coded_lines(n);
  int st = PTX_OK;
  dispatch_pow2(n, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    const int rs = RowPass<N>::smem(lines);
    const int lines128 = RowPass<N>::lines(128, N);
    const int pool = rs + lines * N * (int)sizeof(float) + N * (int)sizeof(float2);
    const int cs = kColsPerCta * ColPass<N>::LP * (int)sizeof(float2);
    if (!st) st = ensure_smem((const void*)fft2_rows_kernel<N, false>, rs);
    if (!st) st = ensure_smem((const void*)fft2_rows_kernel<N, true>, rs);
    if (!st) st = ensure_smem((const void*)fft2_cols_kernel<N, false>, cs);
    if (!st) st = ensure_smem((const void*)fft2_cols_kernel<N, true>, cs);
    if (!st) st = ensure_smem((const void*)coded_cols<1, false, N>, cs);
    if (!st) st = ensure_smem((const void*)coded_cols<3, false, N>, cs);
    if (!st) st = ensure_smem((const void*)coded_cols<3, true, N>, cs);
    if (!st) st = ensure_smem((const void*)coded_cols_filter_pair<false, N>, ColPairCfg<N>::kExchBytes + ColPairCfg<N>::kTwBytes);
    if (!st) st = ensure_smem((const void*)coded_cols_filter_pair<true, N>, ColPairCfg<N>::kExchBytes + ColPairCfg<N>::kTwBytes);
    if (!st) st = ensure_smem((const void*)coded_cols<7, false, N>, cs);
    if (!st) st = ensure_smem((const void*)coded_rows_mask<N>, CodedRowCfg<N>::smem(lines128, 1));
    if (!st) st = ensure_smem((const void*)coded_rows_pool<kCodedSweep, N>, pool);
    if (!st) st = ensure_smem((const void*)coded_rows_pool<kCodedForward, N>, pool);
    if (!st) st = ensure_smem((const void*)coded_rows_pool<kCodedBackward, N>, pool);
    if (!st) st = ensure_smem((const void*)coded_rows_grad_mask<N>, CodedRowCfg<N>::smem(lines128, 2));
  });
  return st;
}

// Arguments of the mixed-radix passes common to all of them; callers fill in the rest.
MixCodedArgs mix_args(const CodedGeom& g, int nf, float inv_n) {
  MixCodedArgs a{};
  a.scratch = g.frames;
  a.ospec = g.ospec;
  a.inv_n = inv_n;
  a.grad_ospec = g.gospec;
  a.twt = g.plan.mix_twt;
  a.twi = g.plan.mix_twi;
  a.ds = g.ds;
  a.nframes = nf;
  return a;
}

template <bool INV>
void launch_fft2(const CodedGeom& g, const float2* in, int n, float2* out, float2* tmp, const LinePlan& p,
                 cudaStream_t s) {
  if (g.mix) {
    prof_begin(kFft2Rows, s);
    g.mfft->fft2_rows(INV, in, n, tmp, p.mix_twt, s);
    prof_end(kFft2Rows, s);
    prof_begin(kFft2Cols, s);
    g.mfft->fft2_cols(INV, tmp, n, out, 1.0f, p.mix_twt, s);
    prof_end(kFft2Cols, s);
    return;
  }
  dispatch_pow2(n, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    const int lines = RowPass<N>::lines(256, N);
    prof_begin(kFft2Rows, s);
    fft2_rows_kernel<N, INV><<<(N + lines - 1) / lines, lines * RowPass<N>::T, RowPass<N>::smem(lines), s>>>(
        in, N, tmp, p.tw, lines);
    prof_end(kFft2Rows, s);
    prof_begin(kFft2Cols, s);
    fft2_cols_kernel<N, INV><<<num_tiles(N) * (kTile / kColsPerCta), ColPass<N>::kThreads,
                               kColsPerCta * ColPass<N>::LP * (int)sizeof(float2), s>>>(tmp, N, out, 1.0f, p.tw);
    prof_end(kFft2Cols, s);
  });
}

template <int STAGE, bool CONJ>
void launch_cols(const CodedGeom& g, int nf, const float2* t1, const float2* t2, const float* shifts,
                 cudaStream_t s, double* grad_shifts = nullptr) {
  const float inv_n = 1.0f / static_cast<float>((double)g.n * g.n);
  prof_begin(kCodedCols, s);
  if (g.mix) {
    MixCodedArgs a = mix_args(g, nf, inv_n);
    a.t1 = t1;
    a.t2 = t2;
    a.shifts = shifts;
    a.grad_shifts = STAGE == 7 ? grad_shifts : nullptr;
    g.mix->cols(STAGE, CONJ, a, s);
    prof_end(kCodedCols, s);
    return;
  }
  dispatch_pow2(g.n, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    if constexpr (STAGE == 3) {
      // the paired kernel reads T2 two columns at a time (16-byte loads)
      if ((reinterpret_cast<uintptr_t>(t2) & 15) == 0) {
        using C = ColPairCfg<N>;
        dim3 grid(num_tiles(N), nf);
        coded_cols_filter_pair<CONJ, N><<<grid, C::kThreads, C::kExchBytes + C::kTwBytes, s>>>(g.frames, t2, inv_n,
                                                                                             g.plan.tw);
        return;
      }
    }
    dim3 grid(num_tiles(N) * (kTile / kColsPerCta), nf);
    coded_cols<STAGE, CONJ, N><<<grid, ColPass<N>::kThreads, kColsPerCta * ColPass<N>::LP * (int)sizeof(float2), s>>>(
        g.frames, g.ospec, t1, t2, shifts, inv_n, g.gospec, g.plan.tw, STAGE == 7 ? grad_shifts : nullptr);
  });
  prof_end(kCodedCols, s);
}

void launch_rows_mask(const CodedGeom& g, int nf, const float2* mask, float2* xstore, cudaStream_t s) {
  const float inv_n = 1.0f / static_cast<float>((double)g.n * g.n);
  prof_begin(kCodedRows, s);
  if (g.mix) {
    MixCodedArgs a = mix_args(g, nf, inv_n);
    a.mask = mask;
    a.xstore = xstore;
    g.mix->rows_mask(a, s);
    prof_end(kCodedRows, s);
    return;
  }
  dispatch_pow2(g.n, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    const int lines = RowPass<N>::lines(128, N);
    const int rowgroups = (N + lines - 1) / lines;
    const int threads = lines * RowPass<N>::T, smem = CodedRowCfg<N>::smem(lines, 1);
    const int grid = persistent_grid((const void*)coded_rows_mask<N>, threads, smem, (long long)rowgroups * nf);
    coded_rows_mask<N><<<grid, threads, smem, s>>>(g.frames, mask, xstore, inv_n, nf, rowgroups, g.plan.tw, lines);
  });
  prof_end(kCodedRows, s);
}

template <int MODE>
void launch_rows_pool(const CodedGeom& g, int frame0, int nf, const uint16_t* measured, float scale,
                      float grad_scale, double inv_numel, double* loss, float2* sensor, float* amplitude,
                      const float* grad_output, cudaStream_t s) {
  const float inv_n = 1.0f / static_cast<float>((double)g.n * g.n);
  prof_begin(kCodedRows, s);
  if (g.mix) {
    MixCodedArgs a = mix_args(g, nf, inv_n);
    a.frame0 = frame0;
    a.measured = measured;
    a.scale = scale;
    a.grad_scale = grad_scale;
    a.inv_numel = inv_numel;
    a.loss = loss;
    a.sensor = sensor;
    a.amplitude = amplitude;
    a.grad_output = grad_output;
    g.mix->rows_pool(MODE == kCodedSweep ? kMixColSweep : MODE == kCodedForward ? kMixColForward : kMixColBackward,
                     a, s);
    prof_end(kCodedRows, s);
    return;
  }
  dispatch_pow2(g.n, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    const int lines = RowPass<N>::lines(256, N);
    dim3 grid((N + lines - 1) / lines, nf);
    const int smem = RowPass<N>::smem(lines) + lines * N * (int)sizeof(float) + N * (int)sizeof(float2);
    coded_rows_pool<MODE, N><<<grid, lines * RowPass<N>::T, smem, s>>>(g.frames, g.ds, frame0, inv_n, measured, scale,
                                                                       grad_scale, inv_numel, loss, sensor, amplitude,
                                                                       grad_output, g.plan.tw, lines);
  });
  prof_end(kCodedRows, s);
}

void launch_rows_grad_mask(const CodedGeom& g, int nf, const float2* mask, const float2* xstore, float2* grad_mask,
                           cudaStream_t s) {
  prof_begin(kCodedRows, s);
  if (g.mix) {
    MixCodedArgs a = mix_args(g, nf, 1.0f / static_cast<float>((double)g.n * g.n));
    a.mask = mask;
    a.xstore = const_cast<float2*>(xstore);
    a.grad_mask = grad_mask;
    g.mix->rows_grad_mask(a, s);
    prof_end(kCodedRows, s);
    return;
  }
  dispatch_pow2(g.n, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    const int lines = RowPass<N>::lines(128, N);
    const int rowgroups = (N + lines - 1) / lines;
    const int threads = lines * RowPass<N>::T, smem = CodedRowCfg<N>::smem(lines, 2);
    const int grid = persistent_grid((const void*)coded_rows_grad_mask<N>, threads, smem, (long long)rowgroups * nf);
    coded_rows_grad_mask<N><<<grid, threads, smem, s>>>(g.frames, mask, xstore, nf, rowgroups, grad_mask, g.plan.tw,
                                                        lines);
  });
  prof_end(kCodedRows, s);
}

// The adjoint passes 4 (backward part) to 7 for one chunk, given g_s already in the frames.
void adjoint_tail(const CodedGeom& g, int nf, const float2* mask, const float2* t1, const float2* t2,
                  const float* shifts, const float2* xstore, float2* grad_mask, cudaStream_t s,
                  double* grad_shifts = nullptr) {
  launch_cols<3, true>(g, nf, t1, t2, shifts, s);
  launch_rows_grad_mask(g, nf, mask, xstore, grad_mask, s);
  launch_cols<7, false>(g, nf, t1, t2, shifts, s, grad_shifts);
}

}  // namespace
}  // namespace ptx

using namespace ptx;

namespace ptx {
namespace {
int coded_backward_impl(const float* grad_output, const float* x_forward, const float* sensor, const float* amplitude,
                        const float* coded_surface, const float* transfer_1, const float* transfer_2, int n,
                        const float* shifts_xy, int batch, int downsample, float* grad_object, float* grad_coded,
                        void* workspace, size_t workspace_bytes, void* stream, double* grad_shifts) {
  CodedGeom g;
  if (int st = coded_check(n, downsample, coded_surface, coded_surface, transfer_2, shifts_xy, batch, workspace,
                           workspace_bytes, false, &g)) {
    return st;
  }
  if (((!grad_output || !x_forward || !sensor || !amplitude) && batch > 0) || !grad_object || !grad_coded) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "null pointer argument");
  }
  if (reinterpret_cast<uintptr_t>(x_forward) & 15) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "x_forward must be 16-byte aligned");
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const float2* T1 = reinterpret_cast<const float2*>(transfer_1);
  const float2* T2 = reinterpret_cast<const float2*>(transfer_2);
  const float2* M = reinterpret_cast<const float2*>(coded_surface);
  cudaMemsetAsync(g.gospec, 0, g.field_bytes, s);
  cudaMemsetAsync(grad_coded, 0, g.field_bytes, s);
  for (int b0 = 0; b0 < batch; b0 += g.chunk) {
    const int nf = std::min(g.chunk, batch - b0);
    launch_rows_pool<kCodedBackward>(g, b0, nf, nullptr, 0.f, 0.f, 0.0, nullptr,
                                     const_cast<float2*>(reinterpret_cast<const float2*>(sensor)),
                                     const_cast<float*>(amplitude), grad_output, s);
    adjoint_tail(g, nf, M, T1, T2, shifts_xy + 2 * (size_t)b0,
                 reinterpret_cast<const float2*>(x_forward) + (size_t)b0 * n * n,
                 reinterpret_cast<float2*>(grad_coded), s, grad_shifts ? grad_shifts + 2 * (size_t)b0 : nullptr);
  }
  launch_fft2<true>(g, g.gospec, n, reinterpret_cast<float2*>(grad_object), g.tmp, g.plan, s);
  return cuda_status(cudaGetLastError(), "ptx_coded_backward launch");
}

}  // namespace
}  // namespace ptx

extern "C" {

size_t ptx_coded_workspace_bytes(int n, int batch) {
  if (n <= 0) return 0;
  const size_t per = tiled_bytes_of(n) + field_bytes_of(n);  // a frame and its stored x
  const size_t frames = std::max<size_t>(1, std::min<size_t>((size_t)std::max(batch, 1), (4096ull << 20) / per));
  return coded_fixed_bytes(n) + frames * per;
}

int ptx_coded_forward(const float* object, const float* coded_surface, const float* transfer_1, const float* transfer_2,
                      int n, const float* shifts_xy, int batch, int downsample, float* x_forward, float* sensor,
                      float* amplitude, void* workspace, size_t workspace_bytes, void* stream) {
  CodedGeom g;
  if (int st = coded_check(n, downsample, object, coded_surface, transfer_2, shifts_xy, batch, workspace,
                           workspace_bytes, false, &g)) {
    return st;
  }
  if ((!x_forward || !sensor || !amplitude) && batch > 0) return set_error(PTX_ERR_INVALID_ARGUMENT, "null output");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const float2* T1 = reinterpret_cast<const float2*>(transfer_1);
  const float2* T2 = reinterpret_cast<const float2*>(transfer_2);
  const float2* M = reinterpret_cast<const float2*>(coded_surface);
  launch_fft2<false>(g, reinterpret_cast<const float2*>(object), n, g.ospec, g.tmp, g.plan, s);
  for (int b0 = 0; b0 < batch; b0 += g.chunk) {
    const int nf = std::min(g.chunk, batch - b0);
    const float* sh = shifts_xy + 2 * (size_t)b0;
    launch_cols<1, false>(g, nf, T1, T2, sh, s);
    launch_rows_mask(g, nf, M, reinterpret_cast<float2*>(x_forward) + (size_t)b0 * n * n, s);
    launch_cols<3, false>(g, nf, T1, T2, sh, s);
    launch_rows_pool<kCodedForward>(g, b0, nf, nullptr, 0.f, 0.f, 0.0, nullptr, reinterpret_cast<float2*>(sensor),
                                    amplitude, nullptr, s);
  }
  return cuda_status(cudaGetLastError(), "ptx_coded_forward launch");
}

int ptx_coded_backward(const float* grad_output, const float* x_forward, const float* sensor, const float* amplitude,
                       const float* coded_surface, const float* transfer_1, const float* transfer_2, int n,
                       const float* shifts_xy, int batch, int downsample, float* grad_object, float* grad_coded,
                       void* workspace, size_t workspace_bytes, void* stream) {
  return coded_backward_impl(grad_output, x_forward, sensor, amplitude, coded_surface, transfer_1, transfer_2, n,
                             shifts_xy, batch, downsample, grad_object, grad_coded, workspace, workspace_bytes, stream,
                             nullptr);
}

static int coded_sweep_mse(const float* object, const float* coded_surface, const float* transfer_1,
                           const float* transfer_2, int n, const float* shifts_xy, int batch, int downsample,
                           const uint16_t* measured, float scale, double* loss, float* grad_object, float* grad_coded,
                           double* grad_shifts, void* workspace, size_t workspace_bytes, void* stream) {
  CodedGeom g;
  if (int st = coded_check(n, downsample, object, coded_surface, transfer_2, shifts_xy, batch, workspace,
                           workspace_bytes, true, &g)) {
    return st;
  }
  if ((!measured && batch > 0) || !loss || !grad_object || !grad_coded) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "null pointer argument");
  }
  if (!(scale > 0.f)) return set_error(PTX_ERR_INVALID_ARGUMENT, "scale must be positive");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const float2* T1 = reinterpret_cast<const float2*>(transfer_1);
  const float2* T2 = reinterpret_cast<const float2*>(transfer_2);
  const float2* M = reinterpret_cast<const float2*>(coded_surface);
  {
    const size_t nf = g.field_bytes / sizeof(float2);
    prof_begin(kMiscKernel, s);
    sweep_prologue_kernel<<<prologue_blocks(nf, sm_count()), 256, 0, s>>>(
        g.gospec, nf, reinterpret_cast<float2*>(grad_coded), nf, loss, nullptr, nullptr, 0.f);
    if (grad_shifts) cudaMemsetAsync(grad_shifts, 0, sizeof(double) * 2 * (size_t)batch, s);
    prof_end(kMiscKernel, s);
  }
  const int lw = n / downsample;
  const double numel = (double)batch * lw * lw;
  const float grad_scale = static_cast<float>(2.0 / std::max(numel, 1.0));
  launch_fft2<false>(g, reinterpret_cast<const float2*>(object), n, g.ospec, g.tmp, g.plan, s);
  for (int b0 = 0; b0 < batch; b0 += g.chunk) {
    const int nf = std::min(g.chunk, batch - b0);
    const float* sh = shifts_xy + 2 * (size_t)b0;
    launch_cols<1, false>(g, nf, T1, T2, sh, s);
    launch_rows_mask(g, nf, M, g.xstore, s);
    launch_cols<3, false>(g, nf, T1, T2, sh, s);
    launch_rows_pool<kCodedSweep>(g, b0, nf, measured, scale, grad_scale, 1.0 / std::max(numel, 1.0), loss, nullptr,
                                  nullptr, nullptr, s);
    adjoint_tail(g, nf, M, T1, T2, sh, g.xstore, reinterpret_cast<float2*>(grad_coded), s,
                 grad_shifts ? grad_shifts + 2 * (size_t)b0 : nullptr);
  }
  launch_fft2<true>(g, g.gospec, n, reinterpret_cast<float2*>(grad_object), g.tmp, g.plan, s);
  return cuda_status(cudaGetLastError(), "ptx_coded_sweep launch");
}


int ptx_coded_sweep(const float* object, const float* coded_surface, const float* transfer_1, const float* transfer_2,
                    int n, const float* shifts_xy, int batch, int downsample, const uint16_t* measured, float scale,
                    double* loss, float* grad_object, float* grad_coded, void* workspace, size_t workspace_bytes,
                    void* stream) {
  return coded_sweep_mse(object, coded_surface, transfer_1, transfer_2, n, shifts_xy, batch, downsample, measured,
                         scale, loss, grad_object, grad_coded, nullptr, workspace, workspace_bytes, stream);
}

size_t ptx_coded_fd_workspace_bytes(int n, int batch, int downsample) {
  if (n <= 0 || batch < 0 || downsample <= 0) return 0;
  const size_t b = (size_t)std::max(batch, 1);
  const size_t field = (size_t)n * n * sizeof(float2);
  const size_t pooled = (size_t)(n / downsample) * (n / downsample) * sizeof(float);
  auto up = [](size_t x) { return (x + 255) / 256 * 256; };
  return 2 * up(b * field) + 2 * up(b * pooled) + ptx_coded_workspace_bytes(n, batch);
}

static int coded_sweep_fd(const float* object, const float* coded_surface, const float* transfer_1,
                          const float* transfer_2, int n, const float* shifts_xy, int batch, int downsample,
                          const uint16_t* measured, float scale, int isotropic, double* loss, float* grad_object,
                          float* grad_coded, double* grad_shifts, void* workspace, size_t workspace_bytes,
                          void* stream) {
  if (!loss || !grad_object || !grad_coded || !workspace || (!measured && batch > 0)) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "null pointer argument");
  }
  if (n <= 0 || downsample <= 0 || batch < 0) return set_error(PTX_ERR_INVALID_ARGUMENT, "non-positive shape");
  if (!(scale > 0.f)) return set_error(PTX_ERR_INVALID_ARGUMENT, "scale must be positive");
  if (reinterpret_cast<uintptr_t>(workspace) & 255) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "workspace must start on a 256-byte boundary");
  }
  const size_t need = ptx_coded_fd_workspace_bytes(n, batch, downsample);
  if (workspace_bytes < need) {
    return set_error(PTX_ERR_WORKSPACE, "workspace of %zu bytes is smaller than the %zu bytes needed",
                     workspace_bytes, need);
  }
  // workspace: x fields | sensor fields | pooled amplitudes | dL/dA | forward/backward frames
  auto up = [](size_t x) { return (x + 255) / 256 * 256; };
  const size_t b = (size_t)std::max(batch, 1);
  const size_t field = (size_t)n * n * sizeof(float2);
  const int h = n / downsample;
  const size_t pooled = (size_t)h * h * sizeof(float);
  char* p = static_cast<char*>(workspace);
  float* xf = reinterpret_cast<float*>(p);
  p += up(b * field);
  float* sensor = reinterpret_cast<float*>(p);
  p += up(b * field);
  float* amp = reinterpret_cast<float*>(p);
  p += up(b * pooled);
  float* gamp = reinterpret_cast<float*>(p);
  p += up(b * pooled);
  const size_t inner = workspace_bytes - static_cast<size_t>(p - static_cast<char*>(workspace));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (int st = ptx_coded_forward(object, coded_surface, transfer_1, transfer_2, n, shifts_xy, batch, downsample, xf,
                                 sensor, amp, p, inner, stream)) {
    return st;
  }
  cudaMemsetAsync(loss, 0, sizeof(double), s);
  const long long total = (long long)batch * h * h;
  if (total > 0) {
    prof_begin(kMiscKernel, s);
    fd_loss_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(amp, measured, scale, total, h, h,
                                                                            isotropic, gamp, loss);
    prof_end(kMiscKernel, s);
  }
  // the backward reuses the forward's region of the workspace, whose object spectrum the
  // shift gradient reads
  if (grad_shifts) cudaMemsetAsync(grad_shifts, 0, sizeof(double) * 2 * (size_t)batch, s);
  return coded_backward_impl(gamp, xf, sensor, amp, coded_surface, transfer_1, transfer_2, n, shifts_xy, batch,
                             downsample, grad_object, grad_coded, p, inner, stream, grad_shifts);
}

int ptx_coded_sweep_fd(const float* object, const float* coded_surface, const float* transfer_1,
                       const float* transfer_2, int n, const float* shifts_xy, int batch, int downsample,
                       const uint16_t* measured, float scale, int isotropic, double* loss, float* grad_object,
                       float* grad_coded, void* workspace, size_t workspace_bytes, void* stream) {
  return coded_sweep_fd(object, coded_surface, transfer_1, transfer_2, n, shifts_xy, batch, downsample, measured,
                        scale, isotropic, loss, grad_object, grad_coded, nullptr, workspace, workspace_bytes, stream);
}

size_t ptx_coded_sweep_ex_workspace_bytes(int n, int batch, int downsample, int loss_kind) {
  return loss_kind == PTX_LOSS_MSE ? ptx_coded_workspace_bytes(n, batch)
                                   : ptx_coded_fd_workspace_bytes(n, batch, downsample);
}

int ptx_coded_sweep_ex(const float* object, const float* coded_surface, const float* transfer_1,
                       const float* transfer_2, int n, const float* shifts_xy, int batch, int downsample,
                       const uint16_t* measured, float scale, int loss_kind, double* loss, float* grad_object,
                       float* grad_coded, double* grad_shifts, void* workspace, size_t workspace_bytes, void* stream) {
  switch (loss_kind) {
    case PTX_LOSS_MSE:
      return coded_sweep_mse(object, coded_surface, transfer_1, transfer_2, n, shifts_xy, batch, downsample,
                             measured, scale, loss, grad_object, grad_coded, grad_shifts, workspace, workspace_bytes,
                             stream);
    case PTX_LOSS_FD_ISOTROPIC:
    case PTX_LOSS_FD_ANISOTROPIC:
      return coded_sweep_fd(object, coded_surface, transfer_1, transfer_2, n, shifts_xy, batch, downsample,
                            measured, scale, loss_kind == PTX_LOSS_FD_ISOTROPIC ? 1 : 0, loss, grad_object,
                            grad_coded, grad_shifts, workspace, workspace_bytes, stream);
    default:
      return set_error(PTX_ERR_INVALID_ARGUMENT, "unknown loss kind %d", loss_kind);
  }
}

}  // extern "C"
