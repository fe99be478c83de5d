// Fourier ptychography passes for sides that are not all powers of two, on the mixed-radix
// register FFT (ptx_mixfft.cuh), which takes every {2,3,5}-smooth length 4..1024 including
// the powers of two.
//
// Same math, pass structure and scratch layout as the power-of-two FPM kernels (ptx_fpm.cu;
// python/ptychoX/fpm/ops.py:180-183 forward, :209-221 adjoint, :113-124 windows), with
// modulo arithmetic where those use masks and the reference's shift conventions for odd
// sides: the window of LED b is S[(ly + r + H // 2) % H, (lx + c + W // 2) % W]
// (Python modulo), fftshift places window row r at frame row i with r = (i + ceil(h/2)) % h
// (columns likewise), and ifftshift maps the adjoint back through the same relation.
//   spectrum     S = fft2(O): row pass (natural -> tiled) and column pass (tiled ->
//                natural); grad_O = ifft2(grad_S) * H W the same with PLUS = true;
//   rows forward gather window x pupil at the fftshifted places (space layout), inverse
//                row DFT, store the row from the frequency layout;
//   columns      inverse column DFT, image = X / (h w), amplitude-loss epilogue against the
//                (unshifted) counts, forward column DFT back to the space layout (sweep); the
//                image and amplitude (forward); g image / |image| and the forward column DFT
//                (backward);
//   rows adjoint forward row DFT from the frequency layout, / (h w), grad_S += Gl conj(pupil)
//                (float2 atomics, wrapped), grad_pupil += Gl conj(S) in registers.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <stdint.h>

#include "ptx_mix.cuh"

namespace ptx {
namespace mixfpm {

using mixk::ColCfg;
using mixk::ld_nc_here;
using mixk::opaque_zero;
using mixk::RowCfg;

constexpr float kEps = 1.1920928955078125e-07f;  // torch.finfo(float32).eps

// v mod n in [0, n) for any sign of v (Python's %)
__device__ __forceinline__ int pymod(long long v, int n) {
  long long r = v % n;
  return static_cast<int>(r < 0 ? r + n : r);
}

// ---- 2-D transform of one image: rows (natural [H][N] -> tiled [tiles(N)][H][16]) --------
template <int N, bool PLUS>
__global__ void __launch_bounds__(RowCfg<N>::THREADS) mix_fft2_rows(const float2* __restrict__ in, int H,
                                                                     float2* __restrict__ tiled,
                                                                     const float2* __restrict__ twt, int lines) {
  pdl_wait();
  using Cfg = RowCfg<N>;
  constexpr int A = Cfg::A, B = Cfg::B;
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x;
  const int l = tid / B;
  const int t = tid - l * B;
  const int r = blockIdx.x * lines + l;
  const bool row_ok = r < H;
  float2 y[A];
#pragma unroll
  for (int j = 0; j < A; ++j) y[j] = row_ok ? in[(size_t)r * N + t + B * j] : make_float2(0.f, 0.f);
  float2* buf = sm + l * Cfg::BUF;
  mix::fwd_step1<N, Cfg::P, 1, PLUS>(y, buf, t, twt);
  __syncthreads();
  if (t < A && row_ok) {
    float2 z[B];
    mix::fwd_step2<N, Cfg::P, 1, PLUS>(z, buf, t);
#pragma unroll
    for (int k = 0; k < B; ++k) {
      const int kc = t + A * k;
      tiled[((size_t)(kc / kTile) * H + r) * kTile + (kc % kTile)] = z[k];
    }
  }
}

// ---- columns (tiled [tiles(W)][N][16] -> natural out [N][W], times `scale`) ---------------
template <int N, bool PLUS>
__global__ void __launch_bounds__(ColCfg<N>::THREADS) mix_fft2_cols(const float2* __restrict__ tiled, int W,
                                                                     float2* __restrict__ out, float scale,
                                                                     const float2* __restrict__ twt) {
  pdl_wait();
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
  const bool col_ok = kc < W;
  const float2* tile = tiled + (size_t)ct * N * kTile + (c0 - ct * kTile);
  float2 y[A];
#pragma unroll
  for (int j = 0; j < A; ++j) y[j] = col_ok ? tile[(t + B * j) * kTile + c] : make_float2(0.f, 0.f);
  mix::fwd_step1<N, Cfg::RS, C, PLUS>(y, sm + c, t, twt);
  __syncthreads();
  if (t < A && col_ok) {
    float2 z[B];
    mix::fwd_step2<N, Cfg::RS, C, PLUS>(z, sm + c, t);
#pragma unroll
    for (int k = 0; k < B; ++k) out[(size_t)(t + A * k) * W + kc] = cscale(z[k], scale);
  }
}

// ---- rows forward: grid (frames, row groups of `lines` rows) ------------------------------
template <int N>
__global__ void __launch_bounds__(RowCfg<N>::THREADS) mix_fpm_rows_forward(MixFpmRowsArgs a, int lines) {
  pdl_wait();
  using Cfg = RowCfg<N>;
  constexpr int A = Cfg::A, B = Cfg::B;
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x;
  const int l = tid / B;
  const int t = tid - l * B;
  const int f = blockIdx.x;
  const int i = blockIdx.y * lines + l;  // frame row
  const bool row_ok = i < a.lh;
  float2 y[A];
  if (row_ok) {
    const int r = (i + (a.lh + 1) / 2) % a.lh;  // window row at frame row i
    const long long lx = a.led[2 * f], ly = a.led[2 * f + 1];
    const float2* srow = a.spec + (size_t)pymod(ly + r + a.oh / 2, a.oh) * a.ow;
    const int x0 = pymod(lx + a.ow / 2, a.ow);
    const float2* prow = a.pupil + (size_t)r * N;
#pragma unroll
    for (int j = 0; j < A; ++j) {
      const int c = (t + B * j + (N + 1) / 2) % N;  // window column at frame column t + B j
      int x = x0 + c;
      if (x >= a.ow) x -= a.ow;
      y[j] = cmul(__ldg(srow + x), __ldg(prow + c));
    }
  } else {
#pragma unroll
    for (int j = 0; j < A; ++j) y[j] = make_float2(0.f, 0.f);
  }
  float2* buf = sm + l * Cfg::BUF;
  mix::fwd_step1<N, Cfg::P, 1, true>(y, buf, t, a.twt);
  __syncthreads();
  if (t < A && row_ok) {
    float2 z[B];
    mix::fwd_step2<N, Cfg::P, 1, true>(z, buf, t);
    float2* base = a.scratch + (size_t)f * num_tiles(N) * a.lh * kTile + (size_t)i * kTile;
#pragma unroll
    for (int k = 0; k < B; ++k) {
      const int kc = t + A * k;
      base[(size_t)(kc / kTile) * a.lh * kTile + (kc % kTile)] = z[k];
    }
  }
}

// ---- rows adjoint: grid (frame chunks, row groups), `fpc` frames per CTA --------------------
// The next frame's scratch row lands in shared memory by cp.async while the current frame
// scatters (as in the conventional mixed-radix adjoint); grad_pupil partials stay in
// registers across the CTA's frames.
template <int N>
__global__ void __launch_bounds__(RowCfg<N>::THREADS, 2) mix_fpm_rows_adjoint(MixFpmRowsArgs a, int lines, int fpc) {
  pdl_wait();
  using Cfg = RowCfg<N>;
  constexpr int A = Cfg::A, B = Cfg::B;
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x;
  const int l = tid / B;
  const int t = tid - l * B;
  const int i = blockIdx.y * lines + l;
  const bool row_ok = i < a.lh;
  const int r = row_ok ? (i + (a.lh + 1) / 2) % a.lh : 0;
  const int f0 = blockIdx.x * fpc;
  const int f1 = min(a.nframes, f0 + fpc);
  float2* buf = sm + l * Cfg::BUF;
  float2* twi_s = sm + lines * Cfg::BUF;
  float2* land = sm + Cfg::land_offset(lines) + l * Cfg::LAND;
  const size_t frame_stride = (size_t)num_tiles(N) * a.lh * kTile;
  const uint64_t pol_first = policy_evict_first();
  auto prefetch = [&](int f) {
    const float2* src = a.scratch + (size_t)f * frame_stride + (size_t)i * kTile;
    const int tq = t + opaque_zero();
#pragma unroll
    for (int q = 0; q < (N / 2 + B - 1) / B; ++q) {
      const int kc = 2 * (tq + B * q);
      if (kc + 1 < N) cp_async16_hint(land + kc, src + (kc / kTile) * a.lh * kTile + (kc % kTile), pol_first);
    }
    if ((N & 1) && t == 0) cp_async8_hint(land + N - 1, src + ((N - 1) / kTile) * a.lh * kTile + ((N - 1) % kTile), pol_first);
    cp_async_commit();
  };
  for (int q = tid; q < N; q += blockDim.x) twi_s[q] = __ldg(a.twi + q);
  if (row_ok && f0 < f1) prefetch(f0);
  float2 acc[A];
#pragma unroll
  for (int j = 0; j < A; ++j) acc[j] = make_float2(0.f, 0.f);
  cp_async_wait_all();
  __syncthreads();
  for (int f = f0; f < f1; ++f) {
    if (t < A && row_ok) {
      float2 z[B];
#pragma unroll
      for (int k = 0; k < B; ++k) z[k] = land[t + A * k];
      mix::inv_step1<N, Cfg::P, 1, false>(z, buf, t, twi_s);
    }
    __syncthreads();  // the exchange rows are complete and the landing line is free
    if (row_ok && f + 1 < f1) prefetch(f + 1);
    if (row_ok) {
      float2 y[A];
      mix::inv_step2<N, Cfg::P, 1, false>(y, buf, t);
      const long long lx = a.led[2 * f], ly = a.led[2 * f + 1];
      const size_t srow = (size_t)pymod(ly + r + a.oh / 2, a.oh) * a.ow;
      const int x0 = pymod(lx + a.ow / 2, a.ow);
      const int tz = t + opaque_zero();  // per-trip offsets (see opaque_zero)
      const float2* prow = a.pupil + (size_t)r * N;
#pragma unroll
      for (int j = 0; j < A; ++j) {
        const int c = (tz + B * j + (N + 1) / 2) % N;
        int x = x0 + c;
        if (x >= a.ow) x -= a.ow;
        const float2 gl = cscale(y[j], a.norm);
        atomicAdd(&a.grad_spec[srow + x], cmulc(gl, ld_nc_here(prow + c)));
        acc[j] = cadd(acc[j], cmulc(gl, __ldg(a.spec + srow + x)));
      }
    }
    cp_async_wait_all();
    __syncthreads();  // the exchange rows are read and the next landing line is complete
  }
  if (row_ok && f0 < f1) {
#pragma unroll
    for (int j = 0; j < A; ++j) {
      const int c = (t + B * j + (N + 1) / 2) % N;
      atomicAdd(&a.grad_pupil[(size_t)r * N + c], acc[j]);
    }
  }
}

// ---- columns: grid (tiles * 16 / C, frames) ---------------------------------------------
template <int MODE, int N>
__global__ void __launch_bounds__(ColCfg<N>::THREADS) mix_fpm_cols(MixFpmColsArgs a) {
  pdl_wait();
  using Cfg = ColCfg<N>;
  constexpr int A = Cfg::A, B = Cfg::B, C = Cfg::C;
  extern __shared__ float2 sm[];
  __shared__ double red_s[Cfg::THREADS / 32 + 1];
  uint16_t* meas_s = reinterpret_cast<uint16_t*>(reinterpret_cast<char*>(sm) + Cfg::MEAS_OFF);
  const int tid = threadIdx.x;
  const int t = tid / C;
  const int c = tid - t * C;
  constexpr int kSubs = kTile / C;
  const int ct = blockIdx.x / kSubs;
  const int c0 = ct * kTile + (blockIdx.x - ct * kSubs) * C;
  const int f = blockIdx.y;
  const int kc = c0 + c;
  const int lw = a.lw;
  const bool col_ok = kc < lw;
  float2* tile = a.scratch + ((size_t)f * num_tiles(lw) + ct) * N * kTile + (c0 - ct * kTile);
  const size_t g = (size_t)a.frame0 + f;
  float2* buf = sm + c;

  if (MODE == kMixColSweep) {
    // counts of image rows kr (not shifted) -> meas_s[kr * C + cc]
    const bool fast = (lw % kTile == 0) && ((reinterpret_cast<uintptr_t>(a.measured) & 15) == 0);
    if (fast) {
      for (int kr = tid; kr < N; kr += Cfg::THREADS) cp_async16(meas_s + kr * C, a.measured + (g * N + kr) * lw + c0);
      cp_async_commit();
    } else {
      for (int q = tid; q < N * C; q += Cfg::THREADS) {
        const int kr = q / C, cc = q - kr * C;
        meas_s[q] = (c0 + cc < lw) ? a.measured[(g * N + kr) * lw + c0 + cc] : 0;
      }
    }
  }

  float2 z[B];
  if (MODE != kMixColBackward) {
    float2 y[A];
#pragma unroll
    for (int j = 0; j < A; ++j) y[j] = col_ok ? tile[(t + B * j) * kTile + c] : make_float2(0.f, 0.f);
    mix::fwd_step1<N, Cfg::RS, C, true>(y, buf, t, a.twt);
    if (MODE == kMixColSweep) cp_async_wait_all();
    __syncthreads();
    if (t < A) mix::fwd_step2<N, Cfg::RS, C, true>(z, buf, t);
  }

  if (MODE == kMixColSweep) {
    float part = 0.f;
    if (t < A) {
#pragma unroll
      for (int k = 0; k < B; ++k) {
        const int kr = t + A * k;
        float2 out = make_float2(0.f, 0.f);
        if (col_ok) {
          const float2 im = cscale(z[k], a.norm);
          const float yv = __ldg(&a.lut[meas_s[kr * C + c]]);
          float am, inv;
          abs_and_inv(im, kEps, am, inv);
          const float rr = am - yv;
          part = fmaf(rr, rr, part);
          out = cscale(im, a.grad_scale * rr * inv);
        }
        z[k] = out;
      }
    }
    if constexpr (Cfg::THREADS % 32 == 0) {
      double w = static_cast<double>(part);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
      if ((tid & 31) == 0) red_s[tid >> 5] = w;
    } else {
      block_add_double(static_cast<double>(part), a.inv_numel, a.loss);
    }
  } else if (MODE == kMixColForward) {
    if (t < A && col_ok) {
#pragma unroll
      for (int k = 0; k < B; ++k) {
        const size_t idx = (g * N + t + A * k) * lw + kc;
        const float2 im = cscale(z[k], a.norm);
        if (a.image) a.image[idx] = im;
        a.amplitude[idx] = cabsf(im);
      }
    }
    return;
  } else {
    if (t < A) {
#pragma unroll
      for (int k = 0; k < B; ++k) {
        float2 out = make_float2(0.f, 0.f);
        if (col_ok) {
          const size_t idx = (g * N + t + A * k) * lw + kc;
          const float2 im = a.image[idx];
          out = cscale(im, a.grad_output[idx] / fmaxf(cabsf(im), kEps));
        }
        z[k] = out;
      }
    }
  }
  // thread u < A wrote and reads only row u of the exchange buffer since the last barrier
  if (t < A) mix::inv_step1<N, Cfg::RS, C, false>(z, buf, t, a.twi);
  __syncthreads();
  if constexpr (MODE == kMixColSweep && Cfg::THREADS % 32 == 0) {
    if (tid == 0) {
      double w = 0.0;
#pragma unroll
      for (int q = 0; q < Cfg::THREADS / 32; ++q) w += red_s[q];
      atomicAdd(a.loss, w * a.inv_numel);
    }
  }
  float2 y[A];
  mix::inv_step2<N, Cfg::RS, C, false>(y, buf, t);
  if (col_ok) {
#pragma unroll
    for (int j = 0; j < A; ++j) tile[(t + B * j) * kTile + c] = y[j];
  }
}

// ---- launchers --------------------------------------------------------------------------

template <int N>
struct Ops {
  using RC = RowCfg<N>;
  using CC = ColCfg<N>;
  static int prepare() {
    int st = ensure_smem((const void*)mix_fft2_rows<N, false>, RC::SMEM_MAX);
    if (!st) st = ensure_smem((const void*)mix_fft2_rows<N, true>, RC::SMEM_MAX);
    if (!st) st = ensure_smem((const void*)mix_fft2_cols<N, false>, CC::SMEM);
    if (!st) st = ensure_smem((const void*)mix_fft2_cols<N, true>, CC::SMEM);
    if (!st) st = ensure_smem((const void*)mix_fpm_rows_forward<N>, RC::SMEM_MAX);
    if (!st) st = ensure_smem((const void*)mix_fpm_rows_adjoint<N>, RC::SMEM_MAX);
    if (!st) st = ensure_smem((const void*)mix_fpm_cols<kMixColSweep, N>, CC::SMEM);
    if (!st) st = ensure_smem((const void*)mix_fpm_cols<kMixColForward, N>, CC::SMEM);
    if (!st) st = ensure_smem((const void*)mix_fpm_cols<kMixColBackward, N>, CC::SMEM);
    return st;
  }
  static void fft2_rows(bool plus, const float2* in, int H, float2* tiled, const float2* twt, cudaStream_t s) {
    if (H <= 0) return;
    const int lines = std::min(RC::LINES, H);
    const int grid = (H + lines - 1) / lines;
    if (plus) {
      launch_pdl(mix_fft2_rows<N, true>, grid, lines * RC::B, RC::smem_forward(lines), s, in, H, tiled, twt, lines);
    } else {
      launch_pdl(mix_fft2_rows<N, false>, grid, lines * RC::B, RC::smem_forward(lines), s, in, H, tiled, twt, lines);
    }
  }
  static void fft2_cols(bool plus, const float2* tiled, int W, float2* out, float scale, const float2* twt,
                        cudaStream_t s) {
    if (W <= 0) return;
    const int grid = num_tiles(W) * (kTile / CC::C);
    if (plus) {
      launch_pdl(mix_fft2_cols<N, true>, grid, CC::THREADS, CC::SMEM, s, tiled, W, out, scale, twt);
    } else {
      launch_pdl(mix_fft2_cols<N, false>, grid, CC::THREADS, CC::SMEM, s, tiled, W, out, scale, twt);
    }
  }
  static void rows_forward(const MixFpmRowsArgs& a, cudaStream_t s) {
    if (a.nframes <= 0) return;
    const int lines = std::min(RC::LINES, a.lh);
    dim3 grid(a.nframes, (a.lh + lines - 1) / lines);
    launch_pdl(mix_fpm_rows_forward<N>, grid, lines * RC::B, RC::smem_forward(lines), s, a, lines);
  }
  static void rows_adjoint(const MixFpmRowsArgs& a, cudaStream_t s) {
    if (a.nframes <= 0) return;
    const int lines = std::min(RC::LINES, a.lh);
    const int rowgroups = (a.lh + lines - 1) / lines;
    // (row group, frame chunk) CTAs: about 8 per SM in all
    const long long target = (long long)sm_count() * 8;
    int fpc = static_cast<int>(((long long)rowgroups * a.nframes) / std::max(target, 1LL));
    fpc = std::max(1, std::min(fpc, a.nframes));
    dim3 grid((a.nframes + fpc - 1) / fpc, rowgroups);
    launch_pdl(mix_fpm_rows_adjoint<N>, grid, lines * RC::B, RC::smem_adjoint(lines), s, a, lines, fpc);
  }
  static void cols(int mode, const MixFpmColsArgs& a, cudaStream_t s) {
    if (a.nframes <= 0) return;
    dim3 grid(num_tiles(a.lw) * (kTile / CC::C), a.nframes);
    if (mode == kMixColSweep) {
      launch_pdl(mix_fpm_cols<kMixColSweep, N>, grid, CC::THREADS, CC::SMEM, s, a);
    } else if (mode == kMixColForward) {
      launch_pdl(mix_fpm_cols<kMixColForward, N>, grid, CC::THREADS, CC::SMEM, s, a);
    } else {
      launch_pdl(mix_fpm_cols<kMixColBackward, N>, grid, CC::THREADS, CC::SMEM, s, a);
    }
  }
  static const MixFpmOps* table() {
    static const MixFpmOps ops{&prepare, &fft2_rows, &fft2_cols, &rows_forward, &rows_adjoint, &cols};
    return &ops;
  }
};

}  // namespace mixfpm
}  // namespace ptx
