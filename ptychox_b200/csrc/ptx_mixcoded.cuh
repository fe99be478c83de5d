// Coded and near-field ptychography passes for field sides that are {2,3,5}-smooth but not
// powers of two, on the mixed-radix register FFT (ptx_mixfft.cuh).
//
// Same math, seven-pass structure and workspace layout as the power-of-two coded kernels
// (ptx_coded.cu; python/ptychoX/coded/ops.py:136-171, the adjoint in the step order of
// coded_kernel.cu:347-424).  Row passes that run two transforms (2, 4, 6) take the line from
// the space layout to the frequency layout with the inverse DFT, apply their pointwise step
// there (where thread u < A holds spatial columns u + A k) and return with the forward DFT;
// single-transform column passes (1, 7) store or consume the frequency layout directly.
// Signed frequencies follow numpy's fftfreq for odd sides too (k <= (n - 1) / 2 is
// non-negative).  The mask gradient of pass 6 is added per frame with float2 atomics: in the
// frequency layout a thread holds B spatial columns of its row, too many to keep partial sums
// in registers across frames.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <stdint.h>

#include "ptx_mix.cuh"

namespace ptx {
namespace mixcoded {

using mixk::ColCfg;
using mixk::RowCfg;

constexpr float kAmpFloor = 1e-30f;  // keeps g / A finite when a pooled amplitude is exactly 0

// numpy fftfreq(n) * n: k for k <= (n - 1) / 2, k - n above
__device__ __forceinline__ int signed_freq(int k, int n) { return k <= (n - 1) / 2 ? k : k - n; }

// exp(2 pi i (dx fx + dy fy)) for signed integer frequencies fx, fy: the argument reduced
// exactly in FP32 (FMA two-product remainders, integer turns removed) before sincospif.
__device__ __forceinline__ float2 shift_ramp(float dx, float dy, int fx, int fy) {
  const float ffx = static_cast<float>(fx), ffy = static_cast<float>(fy);
  const float px = dx * ffx, py = dy * ffy;
  const float ex = fmaf(dx, ffx, -px), ey = fmaf(dy, ffy, -py);
  const float t = (px - rintf(px)) + (py - rintf(py)) + (ex + ey);
  float s, c;
  sincospif(2.0f * t, &s, &c);
  return make_float2(c, s);
}

template <int N>
__device__ __forceinline__ size_t frame_elem(int f, int r, int c) {
  return ((size_t)f * num_tiles(N) + c / kTile) * N * kTile + (size_t)r * kTile + (c % kTile);
}

// ---- column passes: grid (tiles * 16 / C, frames) ------------------------------------------
// STAGE 1: load O^ T1 R, inverse column DFT, store.  STAGE 3: forward DFT, x T2 (CONJ: x
// conj(T2) / n), inverse DFT, store.  STAGE 7: forward DFT, / n, grad_O^ += . conj(T1 R)
// (float2 atomics) and, with grad_shifts, dL/d(dx, dy) += -2 pi sum (fx, fy) Im(conj(G) u).
template <int STAGE, bool CONJ, int N>
__global__ void __launch_bounds__(ColCfg<N>::THREADS) mix_coded_cols(MixCodedArgs a) {
  using Cfg = ColCfg<N>;
  constexpr int A = Cfg::A, B = Cfg::B, C = Cfg::C;
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x;
  const int t = tid / C;
  const int c = tid - t * C;
  constexpr int kSubs = kTile / C;
  const int ct = blockIdx.x / kSubs;
  const int c0 = ct * kTile + (blockIdx.x - ct * kSubs) * C;
  const int f = blockIdx.y;
  const int kc = c0 + c;
  const bool col_ok = kc < N;
  float2* tile = a.scratch + ((size_t)f * num_tiles(N) + ct) * N * kTile + (c0 - ct * kTile);
  float2* buf = sm + c;
  const float dx = (STAGE == 1 || STAGE == 7) ? a.shifts[2 * f] : 0.f;
  const float dy = (STAGE == 1 || STAGE == 7) ? a.shifts[2 * f + 1] : 0.f;
  const int fx = signed_freq(kc, N);
  float2 y[A];
  if (STAGE == 1) {
#pragma unroll
    for (int j = 0; j < A; ++j) {
      const int kr = t + B * j;
      float2 w = make_float2(0.f, 0.f);
      if (col_ok) {
        const size_t idx = (size_t)kr * N + kc;
        w = cmul(a.ospec[idx], shift_ramp(dx, dy, fx, signed_freq(kr, N)));
        if (a.t1) w = cmul(w, a.t1[idx]);
      }
      y[j] = w;
    }
    mix::fwd_step1<N, Cfg::RS, C, true>(y, buf, t, a.twt);
  } else {
#pragma unroll
    for (int j = 0; j < A; ++j) y[j] = col_ok ? tile[(t + B * j) * kTile + c] : make_float2(0.f, 0.f);
    mix::fwd_step1<N, Cfg::RS, C, false>(y, buf, t, a.twt);
  }
  __syncthreads();
  float2 z[B];
  if (STAGE == 1) {
    if (t < A && col_ok) {
      mix::fwd_step2<N, Cfg::RS, C, true>(z, buf, t);
#pragma unroll
      for (int k = 0; k < B; ++k) tile[(t + A * k) * kTile + c] = z[k];
    }
    return;
  }
  if (t < A) mix::fwd_step2<N, Cfg::RS, C, false>(z, buf, t);
  if (STAGE == 3) {
    if (t < A) {
#pragma unroll
      for (int k = 0; k < B; ++k) {
        const int kr = t + A * k;
        if (col_ok) {
          const float2 h = a.t2[(size_t)kr * N + kc];
          z[k] = CONJ ? cscale(cmulc(z[k], h), a.inv_n) : cmul(z[k], h);
        }
      }
      // thread u wrote and reads only row u of the exchange buffer since the barrier
      mix::inv_step1<N, Cfg::RS, C, true>(z, buf, t, a.twi);
    }
    __syncthreads();
    mix::inv_step2<N, Cfg::RS, C, true>(y, buf, t);
    if (col_ok) {
#pragma unroll
      for (int j = 0; j < A; ++j) tile[(t + B * j) * kTile + c] = y[j];
    }
    return;
  }
  // STAGE 7
  float sx = 0.f, sy = 0.f;
  if (t < A && col_ok) {
#pragma unroll
    for (int k = 0; k < B; ++k) {
      const int kr = t + A * k;
      const size_t idx = (size_t)kr * N + kc;
      const int fy = signed_freq(kr, N);
      float2 w = shift_ramp(dx, dy, fx, fy);
      if (a.t1) w = cmul(w, a.t1[idx]);
      const float2 G = cscale(z[k], a.inv_n);
      atomicAdd(&a.grad_ospec[idx], cmulc(G, w));
      if (a.grad_shifts) {
        const float2 u = cmul(a.ospec[idx], w);
        const float im = fmaf(G.x, u.y, -G.y * u.x);  // Im(conj(G) u)
        sx = fmaf(static_cast<float>(fx), im, sx);
        sy = fmaf(static_cast<float>(fy), im, sy);
      }
    }
  }
  if (a.grad_shifts) {
    constexpr double kTwoPi = 6.283185307179586476925286766559;
    block_add_double(static_cast<double>(sx), -kTwoPi, &a.grad_shifts[2 * f]);
    block_add_double(static_cast<double>(sy), -kTwoPi, &a.grad_shifts[2 * f + 1]);
  }
}

// ---- pass 2: grid (frames, row groups of `lines` rows) -------------------------------------
// inverse row DFT, x = . / n (stored to xstore), a = x M, forward row DFT.
template <int N>
__global__ void __launch_bounds__(RowCfg<N>::THREADS) mix_coded_rows_mask(MixCodedArgs a, int lines) {
  using Cfg = RowCfg<N>;
  constexpr int A = Cfg::A, B = Cfg::B;
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x;
  const int l = tid / B;
  const int t = tid - l * B;
  const int f = blockIdx.x;
  const int r = blockIdx.y * lines + l;
  const bool row_ok = r < N;
  float2* buf = sm + l * Cfg::BUF;
  float2 y[A];
#pragma unroll
  for (int j = 0; j < A; ++j) y[j] = row_ok ? a.scratch[frame_elem<N>(f, r, t + B * j)] : make_float2(0.f, 0.f);
  mix::fwd_step1<N, Cfg::P, 1, true>(y, buf, t, a.twt);
  __syncthreads();
  if (t < A) {
    float2 z[B];
    mix::fwd_step2<N, Cfg::P, 1, true>(z, buf, t);
    float2* xrow = a.xstore + ((size_t)f * N + (row_ok ? r : 0)) * N;
    const float2* mrow = a.mask + (size_t)(row_ok ? r : 0) * N;
#pragma unroll
    for (int k = 0; k < B; ++k) {
      const int c = t + A * k;
      const float2 x = cscale(z[k], a.inv_n);
      if (row_ok) xrow[c] = x;
      z[k] = cmul(x, __ldg(mrow + c));
    }
    mix::inv_step1<N, Cfg::P, 1, false>(z, buf, t, a.twi);
  }
  __syncthreads();
  mix::inv_step2<N, Cfg::P, 1, false>(y, buf, t);
  if (row_ok) {
#pragma unroll
    for (int j = 0; j < A; ++j) a.scratch[frame_elem<N>(f, r, t + B * j)] = y[j];
  }
}

// ---- pass 4: grid (row groups, frames); `lines` a multiple of ds -----------------------------
// kMixColSweep: inverse row DFT, s = . / n, RMS pool over ds x ds, FP64 loss, g_s = gA / (A
// ds^2) s, forward row DFT.  kMixColForward: inverse row DFT, write s and the pooled
// amplitude.  kMixColBackward: g_s from the saved s, amplitude and grad_output, forward DFT.
template <int MODE, int N>
__global__ void __launch_bounds__(512) mix_coded_rows_pool(MixCodedArgs a, int lines) {
  using Cfg = RowCfg<N>;
  constexpr int A = Cfg::A, B = Cfg::B;
  extern __shared__ float2 sm[];
  float* pool = reinterpret_cast<float*>(sm + lines * Cfg::BUF);  // [lines][N] |s|^2, then factors
  const int tid = threadIdx.x;
  const int l = tid / B;
  const int t = tid - l * B;
  const int r0 = blockIdx.x * lines;
  const int r = r0 + l;
  const bool row_ok = r < N;
  const int f = blockIdx.y;
  const size_t g = (size_t)a.frame0 + f;
  const int ds = a.ds;
  const int lw = N / ds;
  float2* buf = sm + l * Cfg::BUF;
  float2 z[B];
  if (MODE == kMixColBackward) {
    if (t < A) {
      const int rr = row_ok ? r : 0;
      const float2* srow = a.sensor + (g * N + rr) * N;
      const float* arow = a.amplitude + (g * lw + rr / ds) * lw;
      const float* grow = a.grad_output + (g * lw + rr / ds) * lw;
#pragma unroll
      for (int k = 0; k < B; ++k) {
        const int c = t + A * k;
        const float am = fmaxf(arow[c / ds], kAmpFloor);
        z[k] = row_ok ? cscale(srow[c], grow[c / ds] / (am * static_cast<float>(ds * ds))) : make_float2(0.f, 0.f);
      }
    }
  } else {
    float2 y[A];
#pragma unroll
    for (int j = 0; j < A; ++j) y[j] = row_ok ? a.scratch[frame_elem<N>(f, r, t + B * j)] : make_float2(0.f, 0.f);
    mix::fwd_step1<N, Cfg::P, 1, true>(y, buf, t, a.twt);
    __syncthreads();
    if (t < A) {
      mix::fwd_step2<N, Cfg::P, 1, true>(z, buf, t);
#pragma unroll
      for (int k = 0; k < B; ++k) {
        z[k] = cscale(z[k], a.inv_n);
        pool[l * N + t + A * k] = cabs2(z[k]);
      }
    }
    __syncthreads();
    // pooled values of this CTA's rows: (lines / ds) x lw blocks, pooled rows below N / ds
    const int prows = min(lines / ds, lw - r0 / ds);
    const int nb = prows * lw;
    double acc = 0.0;
    for (int q = tid; q < nb; q += blockDim.x) {
      const int py = q / lw, px = q - py * lw;
      float sum = 0.f;
      for (int yy = 0; yy < ds; ++yy)
        for (int xx = 0; xx < ds; ++xx) sum += pool[(py * ds + yy) * N + px * ds + xx];
      const float am = sqrtf(fmaxf(sum / static_cast<float>(ds * ds), 0.f));
      const size_t oidx = (g * lw + r0 / ds + py) * lw + px;
      if (MODE == kMixColForward) {
        a.amplitude[oidx] = am;
      } else {
        const float yv = sqrtf(static_cast<float>(a.measured[oidx]) * a.scale);
        const float d = am - yv;
        acc += static_cast<double>(d) * static_cast<double>(d);
        // the factor gA / (A ds^2) at the block's first pixel
        pool[(py * ds) * N + px * ds] = a.grad_scale * d / (fmaxf(am, kAmpFloor) * static_cast<float>(ds * ds));
      }
    }
    if (MODE == kMixColForward) {
      if (t < A && row_ok) {
        float2* srow = a.sensor + (g * N + r) * N;
#pragma unroll
        for (int k = 0; k < B; ++k) srow[t + A * k] = z[k];
      }
      return;
    }
    block_add_double(acc, a.inv_numel, a.loss);  // synchronises the block
    if (t < A) {
#pragma unroll
      for (int k = 0; k < B; ++k) {
        const int c = t + A * k;
        z[k] = row_ok ? cscale(z[k], pool[((l / ds) * ds) * N + (c / ds) * ds]) : make_float2(0.f, 0.f);
      }
    }
  }
  if (t < A) mix::inv_step1<N, Cfg::P, 1, false>(z, buf, t, a.twi);
  __syncthreads();
  float2 y[A];
  mix::inv_step2<N, Cfg::P, 1, false>(y, buf, t);
  if (row_ok) {
#pragma unroll
    for (int j = 0; j < A; ++j) a.scratch[frame_elem<N>(f, r, t + B * j)] = y[j];
  }
}

// ---- pass 6: grid (frames, row groups) ---------------------------------------------------
// inverse row DFT (g_a), grad_M += g_a conj(x) (float2 atomics), g_a conj(M), forward DFT.
template <int N>
__global__ void __launch_bounds__(RowCfg<N>::THREADS) mix_coded_rows_grad_mask(MixCodedArgs a, int lines) {
  using Cfg = RowCfg<N>;
  constexpr int A = Cfg::A, B = Cfg::B;
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x;
  const int l = tid / B;
  const int t = tid - l * B;
  const int f = blockIdx.x;
  const int r = blockIdx.y * lines + l;
  const bool row_ok = r < N;
  float2* buf = sm + l * Cfg::BUF;
  float2 y[A];
#pragma unroll
  for (int j = 0; j < A; ++j) y[j] = row_ok ? a.scratch[frame_elem<N>(f, r, t + B * j)] : make_float2(0.f, 0.f);
  mix::fwd_step1<N, Cfg::P, 1, true>(y, buf, t, a.twt);
  __syncthreads();
  if (t < A) {
    float2 z[B];
    mix::fwd_step2<N, Cfg::P, 1, true>(z, buf, t);
    const int rr = row_ok ? r : 0;
    const float2* xrow = a.xstore + ((size_t)f * N + rr) * N;
    const float2* mrow = a.mask + (size_t)rr * N;
    float2* gmrow = a.grad_mask + (size_t)rr * N;
#pragma unroll
    for (int k = 0; k < B; ++k) {
      const int c = t + A * k;
      if (row_ok) atomicAdd(&gmrow[c], cmulc(z[k], xrow[c]));
      z[k] = cmulc(z[k], __ldg(mrow + c));
    }
    mix::inv_step1<N, Cfg::P, 1, false>(z, buf, t, a.twi);
  }
  __syncthreads();
  mix::inv_step2<N, Cfg::P, 1, false>(y, buf, t);
  if (row_ok) {
#pragma unroll
    for (int j = 0; j < A; ++j) a.scratch[frame_elem<N>(f, r, t + B * j)] = y[j];
  }
}

// ---- launchers --------------------------------------------------------------------------

template <int N>
struct Ops {
  using RC = RowCfg<N>;
  using CC = ColCfg<N>;
  static int row_lines() { return std::min(RC::LINES, N); }
  // rows per CTA of pass 4: a multiple of ds, 0 when ds rows of B threads exceed the
  // kernel's 512-thread bound
  static int pool_lines(int ds) {
    if (ds < 1 || N % ds != 0 || ds * RC::B > 512) return 0;
    return ds * std::max(1, RC::LINES / ds);
  }
  static int pool_smem(int lines) { return lines * RC::BUF * (int)sizeof(float2) + lines * N * (int)sizeof(float); }
  static int prepare(int ds) {
    const int pl = pool_lines(ds);
    if (pl == 0) return set_error(PTX_ERR_UNSUPPORTED_SIZE, "downsample %d too large for field side %d", ds, N);
    int st = ensure_smem((const void*)mix_coded_cols<1, false, N>, CC::SMEM);
    if (!st) st = ensure_smem((const void*)mix_coded_cols<3, false, N>, CC::SMEM);
    if (!st) st = ensure_smem((const void*)mix_coded_cols<3, true, N>, CC::SMEM);
    if (!st) st = ensure_smem((const void*)mix_coded_cols<7, false, N>, CC::SMEM);
    if (!st) st = ensure_smem((const void*)mix_coded_rows_mask<N>, RC::smem_forward(row_lines()));
    if (!st) st = ensure_smem((const void*)mix_coded_rows_grad_mask<N>, RC::smem_forward(row_lines()));
    if (!st) st = ensure_smem((const void*)mix_coded_rows_pool<kMixColSweep, N>, pool_smem(pl));
    if (!st) st = ensure_smem((const void*)mix_coded_rows_pool<kMixColForward, N>, pool_smem(pl));
    if (!st) st = ensure_smem((const void*)mix_coded_rows_pool<kMixColBackward, N>, pool_smem(pl));
    return st;
  }
  static void cols(int stage, bool conj, const MixCodedArgs& a, cudaStream_t s) {
    if (a.nframes <= 0) return;
    dim3 grid(num_tiles(N) * (kTile / CC::C), a.nframes);
    if (stage == 1) {
      mix_coded_cols<1, false, N><<<grid, CC::THREADS, CC::SMEM, s>>>(a);
    } else if (stage == 3) {
      if (conj) {
        mix_coded_cols<3, true, N><<<grid, CC::THREADS, CC::SMEM, s>>>(a);
      } else {
        mix_coded_cols<3, false, N><<<grid, CC::THREADS, CC::SMEM, s>>>(a);
      }
    } else {
      mix_coded_cols<7, false, N><<<grid, CC::THREADS, CC::SMEM, s>>>(a);
    }
  }
  static void rows_mask(const MixCodedArgs& a, cudaStream_t s) {
    if (a.nframes <= 0) return;
    const int lines = row_lines();
    dim3 grid(a.nframes, (N + lines - 1) / lines);
    mix_coded_rows_mask<N><<<grid, lines * RC::B, RC::smem_forward(lines), s>>>(a, lines);
  }
  static void rows_grad_mask(const MixCodedArgs& a, cudaStream_t s) {
    if (a.nframes <= 0) return;
    const int lines = row_lines();
    dim3 grid(a.nframes, (N + lines - 1) / lines);
    mix_coded_rows_grad_mask<N><<<grid, lines * RC::B, RC::smem_forward(lines), s>>>(a, lines);
  }
  static void rows_pool(int mode, const MixCodedArgs& a, cudaStream_t s) {
    if (a.nframes <= 0) return;
    const int lines = pool_lines(a.ds);
    dim3 grid((N + lines - 1) / lines, a.nframes);
    const int threads = lines * RC::B, smem = pool_smem(lines);
    if (mode == kMixColSweep) {
      mix_coded_rows_pool<kMixColSweep, N><<<grid, threads, smem, s>>>(a, lines);
    } else if (mode == kMixColForward) {
      mix_coded_rows_pool<kMixColForward, N><<<grid, threads, smem, s>>>(a, lines);
    } else {
      mix_coded_rows_pool<kMixColBackward, N><<<grid, threads, smem, s>>>(a, lines);
    }
  }
  static const MixCodedOps* table() {
    static const MixCodedOps ops{&prepare, &cols, &rows_mask, &rows_pool, &rows_grad_mask};
    return &ops;
  }
};

}  // namespace mixcoded
}  // namespace ptx
