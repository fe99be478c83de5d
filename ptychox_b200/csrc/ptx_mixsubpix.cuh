// Sub-pixel conventional passes for probe sides that are {2,3,5}-smooth but not powers of two,
// on the mixed-radix register FFT (ptx_mixfft.cuh).
//
// Same formulation, five-pass structure and workspace layout as the power-of-two sub-pixel
// kernels (ptx_subpix.cu): the window at the rounded corner shifted by the fraction with a
// Fourier phase ramp (the reference's shift_phase_ramp, python/ptychoX/coded/ops.py:157-171,
// on the patch), separably along columns and rows.  Each shift is the engine's round trip --
// space -> frequency layout with the forward DFT, the ramp at the natural frequency index
// u + A k, frequency -> space with the inverse DFT -- so the line returns to the threads and
// layout it came from.  The ramp tables hold exp(2 pi i d kf / n) / n (the inverse's 1/n
// folded in).  The row pass of the forward sweep then multiplies by the probe and stores the
// spectrum row from the frequency layout (natural spectral columns, as the loss column pass
// expects); the adjoint row pass loads it in that layout.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <math.h>
#include <stdint.h>

#include "ptx_mix.cuh"

namespace ptx {
namespace mixsp {

using mixk::ColCfg;

__device__ __forceinline__ void corner(const double* __restrict__ pos, int f, long long& x0, long long& y0) {
  x0 = static_cast<long long>(floor(pos[2 * f] + 0.5));
  y0 = static_cast<long long>(floor(pos[2 * f + 1] + 0.5));
}

__device__ __forceinline__ bool window_ok(long long x0, long long y0, int ph, int pw, int H, int W) {
  return x0 >= 0 && y0 >= 0 && x0 + pw <= W && y0 + ph <= H;
}

// Row passes: about 128 threads per CTA; per line the exchange buffer (BUF, as the
// conventional row passes lay it out), the probe row (M) and, in the adjoint, the grad_P
// partials (M).  Thread t touches only columns t + B j of the probe and partial rows.
template <int M>
struct RowCfg {
  using R = mixk::RowCfg<M>;
  static constexpr int A = R::A, B = R::B, P = R::P, BUF = R::BUF;
  static constexpr int LINES = 128 / B > 0 ? 128 / B : 1;
  static constexpr int THREADS = LINES * B;
  static int smem(int lines, bool adjoint) { return lines * (BUF + (adjoint ? 2 : 1) * M) * (int)sizeof(float2); }
};

// ---- column shift: grid (tiles * 16 / C, frames) ------------------------------------------
// GATHER: the window's columns from the object (zero for a window outside it), column DFT,
// x ramp_y, inverse DFT, stored into the tiled frame.  Otherwise: the frame's columns, column
// DFT, x conj(ramp_y), inverse DFT, added into grad_sample at the window (float2 atomics;
// windows outside the object are skipped).
template <int N, bool GATHER>
__global__ void __launch_bounds__(ColCfg<N>::THREADS) mix_subpix_cols(MixSubpixArgs a) {
  using Cfg = ColCfg<N>;
  constexpr int A = Cfg::A, B = Cfg::B, C = Cfg::C;
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x;
  const int t = tid / C;
  const int c = tid - t * C;
  constexpr int kSubs = kTile / C;
  const int ct = blockIdx.x / kSubs;
  const int c0 = ct * kTile + (blockIdx.x - ct * kSubs) * C;
  const int kc = c0 + c;
  const bool col_ok = kc < a.pw;
  const int f = blockIdx.y;
  const int g = a.frame0 + f;
  float2* tile = a.scratch + ((size_t)f * num_tiles(a.pw) + ct) * N * kTile + (c0 - ct * kTile);
  long long x0, y0;
  corner(a.pos, g, x0, y0);
  const bool ok = window_ok(x0, y0, N, a.pw, a.H, a.W);
  const float2* ry = a.ry + (size_t)g * N;
  float2* buf = sm + c;
  float2 y[A];
  if (GATHER) {
    const float2* col = a.sample + y0 * a.W + x0 + kc;
#pragma unroll
    for (int j = 0; j < A; ++j) y[j] = (ok && col_ok) ? __ldg(col + (size_t)(t + B * j) * a.W) : make_float2(0.f, 0.f);
  } else {
#pragma unroll
    for (int j = 0; j < A; ++j) y[j] = col_ok ? tile[(t + B * j) * kTile + c] : make_float2(0.f, 0.f);
  }
  mix::fwd_step1<N, Cfg::RS, C, false>(y, buf, t, a.twt_col);
  __syncthreads();
  if (t < A) {
    float2 z[B];
    mix::fwd_step2<N, Cfg::RS, C, false>(z, buf, t);
#pragma unroll
    for (int k = 0; k < B; ++k) {
      float2 w = __ldg(ry + t + A * k);
      if (!GATHER) w.y = -w.y;
      z[k] = cmul(z[k], w);
    }
    // thread u wrote and reads only row u of the exchange buffer since the barrier
    mix::inv_step1<N, Cfg::RS, C, true>(z, buf, t, a.twi_col);
  }
  __syncthreads();
  mix::inv_step2<N, Cfg::RS, C, true>(y, buf, t);
  if (GATHER) {
    if (col_ok) {
#pragma unroll
      for (int j = 0; j < A; ++j) tile[(t + B * j) * kTile + c] = y[j];
    }
  } else if (ok && col_ok) {
    float2* col = a.grad_sample + y0 * a.W + x0 + kc;
#pragma unroll
    for (int j = 0; j < A; ++j) atomicAdd(col + (size_t)(t + B * j) * a.W, y[j]);
  }
}

// ---- row passes: grid (row groups of `lines` rows, frame chunks of `fpc` frames) --------------
// FORWARD: row DFT, x ramp_x, inverse DFT (= S, stored into sbuf when STORE_S), and with
// STORE_OUT x P and the row DFT, stored from the frequency layout.  Adjoint: inverse row DFT of
// the spectrum row (= G), grad_P += G conj(S) (shared-memory partials, one float2 atomic per
// element per CTA at the end), G conj(P), row DFT, x conj(ramp_x), inverse DFT, stored.
template <int M, bool FORWARD, bool STORE_S, bool STORE_OUT>
__global__ void __launch_bounds__(RowCfg<M>::THREADS) mix_subpix_rows(MixSubpixArgs a, int lines, int fpc) {
  using Cfg = RowCfg<M>;
  constexpr int A = Cfg::A, B = Cfg::B, P = Cfg::P;
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x;
  const int l = tid / B;
  const int t = tid - l * B;
  const int r = blockIdx.x * lines + l;
  const bool row_ok = r < a.ph;
  float2* buf = sm + l * Cfg::BUF;
  float2* pbuf = sm + lines * Cfg::BUF + l * M;
  float2* acc = sm + lines * (Cfg::BUF + M) + l * M;  // adjoint only
  const int tiles = num_tiles(M);
#pragma unroll
  for (int j = 0; j < A; ++j) {
    const int cc = t + B * j;
    pbuf[cc] = row_ok ? __ldg(a.probe + (size_t)r * M + cc) : make_float2(0.f, 0.f);
    if (!FORWARD) acc[cc] = make_float2(0.f, 0.f);
  }
  const int f0 = blockIdx.y * fpc;
  const int f1 = min(a.nframes, f0 + fpc);
  for (int f = f0; f < f1; ++f) {
    const float2* rx = a.rx + (size_t)(a.frame0 + f) * M;
    const size_t row0 = (size_t)f * tiles * a.ph * kTile + (size_t)(row_ok ? r : 0) * kTile;
    auto elem = [&](int cc) { return row0 + (size_t)(cc / kTile) * a.ph * kTile + (cc % kTile); };
    float2 y[A];
    if (FORWARD) {
#pragma unroll
      for (int j = 0; j < A; ++j) y[j] = row_ok ? a.scratch[elem(t + B * j)] : make_float2(0.f, 0.f);
      mix::fwd_step1<M, P, 1, false>(y, buf, t, a.twt_row);
      __syncthreads();
      if (t < A) {
        float2 z[B];
        mix::fwd_step2<M, P, 1, false>(z, buf, t);
#pragma unroll
        for (int k = 0; k < B; ++k) z[k] = cmul(z[k], __ldg(rx + t + A * k));
        mix::inv_step1<M, P, 1, true>(z, buf, t, a.twi_row);
      }
      __syncthreads();
      mix::inv_step2<M, P, 1, true>(y, buf, t);  // S at columns t + B j
      if (STORE_S && row_ok) {
#pragma unroll
        for (int j = 0; j < A; ++j) a.sbuf[elem(t + B * j)] = y[j];
      }
      if constexpr (STORE_OUT) {
#pragma unroll
        for (int j = 0; j < A; ++j) y[j] = cmul(y[j], pbuf[t + B * j]);
        // thread t read and now writes only column t of the exchange buffer
        mix::fwd_step1<M, P, 1, false>(y, buf, t, a.twt_row);
        __syncthreads();
        if (t < A) {
          float2 z[B];
          mix::fwd_step2<M, P, 1, false>(z, buf, t);
          if (row_ok) {
#pragma unroll
            for (int k = 0; k < B; ++k) a.scratch[elem(t + A * k)] = z[k];
          }
        }
        __syncthreads();  // the rows are read before the next frame writes the buffer
      }
    } else {
      if (t < A) {
        float2 z[B];
#pragma unroll
        for (int k = 0; k < B; ++k) z[k] = row_ok ? a.scratch[elem(t + A * k)] : make_float2(0.f, 0.f);
        mix::inv_step1<M, P, 1, true>(z, buf, t, a.twi_row);
      }
      __syncthreads();
      mix::inv_step2<M, P, 1, true>(y, buf, t);  // G at columns t + B j
#pragma unroll
      for (int j = 0; j < A; ++j) {
        const int cc = t + B * j;
        const float2 s = row_ok ? a.sbuf[elem(cc)] : make_float2(0.f, 0.f);
        acc[cc] = cadd(acc[cc], cmulc(y[j], s));
        y[j] = cmulc(y[j], pbuf[cc]);
      }
      // thread t read and now writes only column t of the exchange buffer
      mix::fwd_step1<M, P, 1, false>(y, buf, t, a.twt_row);
      __syncthreads();
      if (t < A) {
        float2 z[B];
        mix::fwd_step2<M, P, 1, false>(z, buf, t);
#pragma unroll
        for (int k = 0; k < B; ++k) z[k] = cmulc(z[k], __ldg(rx + t + A * k));
        mix::inv_step1<M, P, 1, true>(z, buf, t, a.twi_row);
      }
      __syncthreads();
      mix::inv_step2<M, P, 1, true>(y, buf, t);
      if (row_ok) {
#pragma unroll
        for (int j = 0; j < A; ++j) a.scratch[elem(t + B * j)] = y[j];
      }
      __syncthreads();  // the columns are read before the next frame writes the rows
    }
  }
  if (!FORWARD && row_ok && f0 < f1) {
#pragma unroll
    for (int j = 0; j < A; ++j) {
      const int cc = t + B * j;
      atomicAdd(a.grad_probe + (size_t)r * M + cc, acc[cc]);
    }
  }
}

// ---- launchers --------------------------------------------------------------------------

template <int N>
struct Ops {
  using CC = ColCfg<N>;
  using RC = RowCfg<N>;
  template <bool F, bool S, bool O>
  static void rows_t(const MixSubpixArgs& a, cudaStream_t s) {
    const int lines = std::min(RC::LINES, a.ph);
    const int rowgroups = (a.ph + lines - 1) / lines;
    // about 8 CTAs per SM in all; each keeps its probe rows (and grad_P partials) over its frames
    const long long target = (long long)sm_count() * 8;
    int fpc = static_cast<int>(std::max<long long>(1, ((long long)rowgroups * a.nframes) / target));
    fpc = std::min(fpc, std::max(a.nframes, 1));
    dim3 grid(rowgroups, (a.nframes + fpc - 1) / fpc);
    mix_subpix_rows<N, F, S, O><<<grid, lines * RC::B, RC::smem(lines, !F), s>>>(a, lines, fpc);
  }
  static int prepare() {
    const int rs = RC::smem(RC::LINES, true);
    int st = ensure_smem((const void*)mix_subpix_cols<N, true>, CC::SMEM);
    if (!st) st = ensure_smem((const void*)mix_subpix_cols<N, false>, CC::SMEM);
    if (!st) st = ensure_smem((const void*)mix_subpix_rows<N, true, true, true>, rs);
    if (!st) st = ensure_smem((const void*)mix_subpix_rows<N, true, true, false>, rs);
    if (!st) st = ensure_smem((const void*)mix_subpix_rows<N, true, false, true>, rs);
    if (!st) st = ensure_smem((const void*)mix_subpix_rows<N, false, false, false>, rs);
    return st;
  }
  static void cols(bool gather, const MixSubpixArgs& a, cudaStream_t s) {
    if (a.nframes <= 0) return;
    dim3 grid(num_tiles(a.pw) * (kTile / CC::C), a.nframes);
    if (gather) {
      mix_subpix_cols<N, true><<<grid, CC::THREADS, CC::SMEM, s>>>(a);
    } else {
      mix_subpix_cols<N, false><<<grid, CC::THREADS, CC::SMEM, s>>>(a);
    }
  }
  static void rows(int variant, const MixSubpixArgs& a, cudaStream_t s) {
    if (a.nframes <= 0) return;
    switch (variant) {
      case kMixSubpixSweepForward: rows_t<true, true, true>(a, s); break;
      case kMixSubpixShiftOnly: rows_t<true, true, false>(a, s); break;
      case kMixSubpixForwardOnly: rows_t<true, false, true>(a, s); break;
      default: rows_t<false, false, false>(a, s); break;
    }
  }
  static const MixSubpixOps* table() {
    static const MixSubpixOps ops{&prepare, &cols, &rows};
    return &ops;
  }
};

}  // namespace mixsp
}  // namespace ptx
