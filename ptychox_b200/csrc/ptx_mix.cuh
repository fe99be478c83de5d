// Conventional sweep passes for {2,3,5}-smooth line lengths that are not powers of two, on
// the mixed-radix register FFT of ptx_mixfft.cuh (N = A * B, one shared-memory exchange).
//
// Same three passes, scratch layout ([frame][tile][row][16]) and arithmetic as the
// power-of-two kernels of the conventional operator (python/ptychoX/base/ops.py:59-67
// forward, :92-105 adjoint; the fused sweep of python/ptychoX/csrc/base_kernel.cu):
//   rows forward : gather O x P rows (space layout, x[t + B j]), forward row DFT, store
//                  the spectrum row (frequency layout, X[u + A k]) tiled;
//   columns      : column DFT, then per mode the amplitude-loss epilogue against the
//                  fftshifted counts and the inverse column DFT (sweep), the far field and
//                  amplitude (forward), or g F / max(|F|, eps) and the inverse column DFT
//                  (backward); the inverse returns the columns to the space layout;
//   rows adjoint : load the row in the frequency layout, inverse row DFT back to the space
//                  layout, scatter G conj(P) into grad_O and accumulate G conj(O) for grad_P.
// A line is held by B threads; the forward transform leaves the frequency layout in the A
// threads t < A, which the inverse takes as its input, so no pass reorders data.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <stdint.h>

#include "ptx_internal.h"
#include "ptx_mixfft.cuh"
#include "ptx_passes.cuh"

namespace ptx {
namespace mixk {

constexpr float kEps = 1.1920928955078125e-07f;  // torch.finfo(float32).eps

__device__ __forceinline__ bool window_in(long long x0, long long y0, int ph, int pw, int H, int W) {
  return x0 >= 0 && y0 >= 0 && x0 + pw <= W && y0 + ph <= H;
}

// Read-only global load that the compiler issues where it stands: the adjoint's probe reads
// are the same on every frame of its loop, and hoisting them out of the loop would hold A
// more complex values in registers for the whole pass.
__device__ __forceinline__ float2 ld_nc_here(const float2* p) {
  float2 v;
  asm volatile("ld.global.nc.v2.f32 {%0, %1}, [%2];\n" : "=f"(v.x), "=f"(v.y) : "l"(p));
  return v;
}

// 0, as a value the compiler cannot see through: offsets derived from it inside a loop are
// recomputed on each trip instead of being hoisted into registers for the whole loop.
__device__ __forceinline__ int opaque_zero() {
  int z;
  asm volatile("mov.u32 %0, 0;\n" : "=r"(z));
  return z;
}

// Row passes: LINES lines of B threads; each line's A x B exchange buffer has the odd row
// pitch P, and consecutive lines sit BUF apart with BUF = B (mod 16), so the 8-byte accesses
// of neighbouring threads of different lines fall in different bank pairs.
template <int N>
struct RowCfg {
  using S = mix::Shape<N>;
  static constexpr int A = S::A, B = S::B, P = S::P;
  static constexpr int LINES = 256 / B > 0 ? 256 / B : 1;
  static constexpr int THREADS = LINES * B;
  static constexpr int BUF = A * P + (((B - A * P) % 16) + 16) % 16;
  // adjoint landing lines: one scratch row per line, 16-byte aligned
  static constexpr int LAND = (N + 1) / 2 * 2;
  // forward: exchange buffers; adjoint: exchange buffers, the inverse twiddle table and the
  // landing lines
  static int smem_forward(int lines) { return lines * BUF * (int)sizeof(float2); }
  __host__ __device__ static constexpr int land_offset(int lines) { return (lines * BUF + N + 1) / 2 * 2; }
  static int smem_adjoint(int lines) { return (land_offset(lines) + lines * LAND) * (int)sizeof(float2); }
  static constexpr int SMEM_MAX = (land_offset(LINES) + LINES * LAND) * (int)sizeof(float2);
};

// Column pass: C columns of one frame tile per CTA, thread (t, c) at t * C + c; the C lines
// are interleaved element by element in the exchange buffer, element (u, t) of column c at
// u * RS + t * C + c, with RS = 8 (mod 16) so the two rows a half-warp touches in the second
// step fall in different bank pairs.
template <int N>
struct ColCfg {
  using S = mix::Shape<N>;
  static constexpr int A = S::A, B = S::B;
  static constexpr int C = 8;
  static constexpr int THREADS = C * B;
  static constexpr int RS = (B * C) % 16 == 0 ? B * C + 8 : B * C;
  static constexpr int BUF = A * RS;
  static constexpr int MEAS_OFF = (BUF * (int)sizeof(float2) + 15) / 16 * 16;
  static constexpr int SMEM = MEAS_OFF + N * C * (int)sizeof(uint16_t);
};

// ---- rows forward: grid (frames, row groups of `lines` rows), lines * B threads -----------
template <int N>
__global__ void __launch_bounds__(RowCfg<N>::THREADS) mix_rows_forward(MixRowsArgs a, int lines) {
  pdl_wait();
  using Cfg = RowCfg<N>;
  constexpr int A = Cfg::A, B = Cfg::B;
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x;
  const int l = tid / B;
  const int t = tid - l * B;
  const int f = blockIdx.x;
  const int r = blockIdx.y * lines + l;
  const long long x0 = a.pos[2 * f], y0 = a.pos[2 * f + 1];
  const bool ok = window_in(x0, y0, a.ph, N, a.H, a.W);
  if (!ok && tid == 0) atomicOr(a.err, 1u);
  const bool row_ok = r < a.ph;
  float2 y[A];
  if (ok && row_ok) {
    const float2* orow = a.sample + (y0 + r) * a.W + x0;
    const float2* prow = a.probe + (size_t)r * N;
#pragma unroll
    for (int j = 0; j < A; ++j) y[j] = cmul(__ldg(orow + t + B * j), __ldg(prow + t + B * j));
  } else {
#pragma unroll
    for (int j = 0; j < A; ++j) y[j] = make_float2(0.f, 0.f);
  }
  float2* buf = sm + l * Cfg::BUF;
  mix::fwd_step1<N, Cfg::P, 1>(y, buf, t, a.twt);
  __syncthreads();
  if (t < A && row_ok) {
    float2 z[B];
    mix::fwd_step2<N, Cfg::P, 1>(z, buf, t);
    float2* base = a.scratch + (size_t)f * num_tiles(N) * a.ph * kTile + (size_t)r * kTile;
#pragma unroll
    for (int k = 0; k < B; ++k) {
      const int kc = t + A * k;
      base[(size_t)(kc / kTile) * a.ph * kTile + (kc % kTile)] = z[k];
    }
  }
}

// ---- rows adjoint: grid (frame chunks, row groups), `fpc` frames per CTA -------------------
// Each line's scratch row of the next frame lands in shared memory by 16-byte cp.async (L2
// evict-first: read once) while the current frame scatters.  The grad_P partials stay in
// registers across the CTA's frames; the twiddles are read from a shared-memory copy and the
// probe through ld_nc_here, so neither is held in registers.
template <int N>
__global__ void __launch_bounds__(RowCfg<N>::THREADS, 2) mix_rows_adjoint(MixRowsArgs a, int lines, int fpc) {
  pdl_wait();
  using Cfg = RowCfg<N>;
  constexpr int A = Cfg::A, B = Cfg::B;
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x;
  const int l = tid / B;
  const int t = tid - l * B;
  const int r = blockIdx.y * lines + l;
  const bool row_ok = r < a.ph;
  const int f0 = blockIdx.x * fpc;
  const int f1 = min(a.nframes, f0 + fpc);
  float2* buf = sm + l * Cfg::BUF;
  float2* twi_s = sm + lines * Cfg::BUF;
  float2* land = sm + Cfg::land_offset(lines) + l * Cfg::LAND;
  const size_t frame_stride = (size_t)num_tiles(N) * a.ph * kTile;
  const uint64_t pol_first = policy_evict_first();
  // scratch row r of frame f -> land[0, N): pairs of elements (a tile row holds 16)
  auto prefetch = [&](int f) {
    const float2* src = a.scratch + (size_t)f * frame_stride + (size_t)r * kTile;
    const int tq = t + opaque_zero();
#pragma unroll
    for (int i = 0; i < (N / 2 + B - 1) / B; ++i) {
      const int kc = 2 * (tq + B * i);
      if (kc + 1 < N) cp_async16_hint(land + kc, src + (kc / kTile) * a.ph * kTile + (kc % kTile), pol_first);
    }
    if ((N & 1) && t == 0) cp_async8_hint(land + N - 1, src + ((N - 1) / kTile) * a.ph * kTile + ((N - 1) % kTile), pol_first);
    cp_async_commit();
  };
  for (int i = tid; i < N; i += blockDim.x) twi_s[i] = __ldg(a.twi + i);
  if (row_ok && f0 < f1) prefetch(f0);
  float2 acc[A];
#pragma unroll
  for (int j = 0; j < A; ++j) acc[j] = make_float2(0.f, 0.f);
  cp_async_wait_all();
  __syncthreads();
  for (int f = f0; f < f1; ++f) {
    const long long x0 = a.pos[2 * f], y0 = a.pos[2 * f + 1];
    const bool ok = window_in(x0, y0, a.ph, N, a.H, a.W);
    if (t < A && row_ok) {
      float2 z[B];
#pragma unroll
      for (int k = 0; k < B; ++k) z[k] = land[t + A * k];
      mix::inv_step1<N, Cfg::P, 1>(z, buf, t, twi_s);
    }
    __syncthreads();  // the exchange rows are complete and the landing line is free
    if (row_ok && f + 1 < f1) prefetch(f + 1);
    if (row_ok && ok) {
      float2 y[A];
      mix::inv_step2<N, Cfg::P, 1>(y, buf, t);
      const int tz = t + opaque_zero();  // per-trip offsets (see opaque_zero)
      const float2* orow = a.sample + (y0 + r) * a.W + x0;
      float2* grow = a.grad_sample + (y0 + r) * a.W + x0;
      const float2* prow = a.probe + (size_t)r * N;
#pragma unroll
      for (int j = 0; j < A; ++j) {
        const int c = tz + B * j;
        atomicAdd(&grow[c], cmulc(y[j], ld_nc_here(prow + c)));
        acc[j] = cadd(acc[j], cmulc(y[j], __ldg(orow + c)));
      }
    }
    cp_async_wait_all();
    __syncthreads();  // the exchange rows are read and the next landing line is complete
  }
  if (row_ok && f0 < f1) {
#pragma unroll
    for (int j = 0; j < A; ++j) atomicAdd(&a.grad_probe[(size_t)r * N + t + B * j], acc[j]);
  }
}

// ---- columns: grid (tiles * 16 / C, frames) ---------------------------------------------
template <int MODE, int N>
__global__ void __launch_bounds__(ColCfg<N>::THREADS) mix_cols(MixColsArgs a) {
  pdl_wait();
  using Cfg = ColCfg<N>;
  constexpr int A = Cfg::A, B = Cfg::B, C = Cfg::C;
  extern __shared__ float2 sm[];
  uint16_t* meas_s = reinterpret_cast<uint16_t*>(reinterpret_cast<char*>(sm) + Cfg::MEAS_OFF);
  const int tid = threadIdx.x;
  const int t = tid / C;
  const int c = tid - t * C;
  constexpr int kSubs = kTile / C;
  const int ct = blockIdx.x / kSubs;
  const int c0 = ct * kTile + (blockIdx.x - ct * kSubs) * C;  // first column of the CTA
  const int f = blockIdx.y;
  const int kc = c0 + c;
  const bool col_ok = kc < a.pw;
  const int pw = a.pw;
  float2* tile = a.scratch + ((size_t)f * num_tiles(pw) + ct) * N * kTile + (c0 - ct * kTile);
  const size_t g = (size_t)a.frame0 + f;
  float2* buf = sm + c;
  int ic = kc + pw / 2;
  if (ic >= pw) ic -= pw;

  if (MODE == kMixColSweep) {
    // counts of spectrum rows kr (unshifted order) -> meas_s[kr * C + cc]
    const bool fast = (pw % kTile == 0) && ((reinterpret_cast<uintptr_t>(a.measured) & 15) == 0);
    if (fast) {
      int ic0 = c0 + pw / 2;
      if (ic0 >= pw) ic0 -= pw;
      for (int kr = tid; kr < N; kr += Cfg::THREADS) {
        int ir = kr + N / 2;
        if (ir >= N) ir -= N;
        cp_async16(meas_s + kr * C, a.measured + (g * N + ir) * pw + ic0);
      }
      cp_async_commit();
    } else {
      for (int i = tid; i < N * C; i += Cfg::THREADS) {
        const int kr = i / C, cc = i - kr * C;
        int ir = kr + N / 2;
        if (ir >= N) ir -= N;
        int icc = c0 + cc + pw / 2;
        if (icc >= pw) icc -= pw;
        meas_s[i] = (c0 + cc < pw) ? a.measured[(g * N + ir) * pw + icc] : 0;
      }
    }
  }

  float2 z[B];
  if (MODE != kMixColBackward) {
    float2 y[A];
#pragma unroll
    for (int j = 0; j < A; ++j) y[j] = col_ok ? tile[(t + B * j) * kTile + c] : make_float2(0.f, 0.f);
    mix::fwd_step1<N, Cfg::RS, C>(y, buf, t, a.twt);
    if (MODE == kMixColSweep) cp_async_wait_all();
    __syncthreads();
    if (t < A) mix::fwd_step2<N, Cfg::RS, C>(z, buf, t);
  }

  __shared__ double red_s[Cfg::THREADS / 32 + 1];
  if (MODE == kMixColSweep) {
    float part = 0.f;
    if (t < A) {
#pragma unroll
      for (int k = 0; k < B; ++k) {
        const int kr = t + A * k;
        float2 out = make_float2(0.f, 0.f);
        if (col_ok) {
          const float yv = __ldg(&a.lut[meas_s[kr * C + c]]);
          float am, inv;
          abs_and_inv(z[k], kEps, am, inv);
          const float rr = am - yv;
          part = fmaf(rr, rr, part);
          out = cscale(z[k], a.grad_scale * rr * inv);
        }
        z[k] = out;
      }
    }
    if constexpr (Cfg::THREADS % 32 == 0) {
      // warp partials now; their sum after the barrier that the inverse transform needs anyway
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
        int ir = t + A * k + N / 2;
        if (ir >= N) ir -= N;
        const size_t idx = (g * N + ir) * pw + ic;
        if (a.far_field) a.far_field[idx] = z[k];
        a.amplitude[idx] = cabsf(z[k]);
      }
    }
    return;
  } else {
    if (t < A) {
#pragma unroll
      for (int k = 0; k < B; ++k) {
        float2 out = make_float2(0.f, 0.f);
        if (col_ok) {
          int ir = t + A * k + N / 2;
          if (ir >= N) ir -= N;
          const size_t idx = (g * N + ir) * pw + ic;
          const float2 F = a.far_field[idx];
          out = cscale(F, a.grad_output[idx] / fmaxf(cabsf(F), kEps));
        }
        z[k] = out;
      }
    }
  }
  // thread u < A wrote and reads only row u of the exchange buffer since the last barrier
  if (t < A) mix::inv_step1<N, Cfg::RS, C>(z, buf, t, a.twi);
  __syncthreads();
  if constexpr (MODE == kMixColSweep && Cfg::THREADS % 32 == 0) {
    if (tid == 0) {
      double w = 0.0;
#pragma unroll
      for (int i = 0; i < Cfg::THREADS / 32; ++i) w += red_s[i];
      atomicAdd(a.loss, w * a.inv_numel);
    }
  }
  float2 y[A];
  mix::inv_step2<N, Cfg::RS, C>(y, buf, t);
  if (col_ok) {
#pragma unroll
    for (int j = 0; j < A; ++j) tile[(t + B * j) * kTile + c] = y[j];
  }
}

// ---- launchers --------------------------------------------------------------------------

template <int N>
struct Ops {
  static int prepare() {
    int st = ensure_smem((const void*)mix_rows_forward<N>, RowCfg<N>::SMEM_MAX);
    if (!st) st = ensure_smem((const void*)mix_rows_adjoint<N>, RowCfg<N>::SMEM_MAX);
    if (!st) st = ensure_smem((const void*)mix_cols<kMixColSweep, N>, ColCfg<N>::SMEM);
    if (!st) st = ensure_smem((const void*)mix_cols<kMixColForward, N>, ColCfg<N>::SMEM);
    if (!st) st = ensure_smem((const void*)mix_cols<kMixColBackward, N>, ColCfg<N>::SMEM);
    return st;
  }
  static void rows_forward(const MixRowsArgs& a, cudaStream_t s) {
    using Cfg = RowCfg<N>;
    if (a.nframes <= 0) return;
    const int lines = std::min(Cfg::LINES, a.ph);
    dim3 grid(a.nframes, (a.ph + lines - 1) / lines);
    launch_pdl(mix_rows_forward<N>, grid, lines * Cfg::B, Cfg::smem_forward(lines), s, a, lines);
  }
  static void rows_adjoint(const MixRowsArgs& a, cudaStream_t s) {
    using Cfg = RowCfg<N>;
    if (a.nframes <= 0) return;
    const int lines = std::min(Cfg::LINES, a.ph);
    const int rowgroups = (a.ph + lines - 1) / lines;
    // (row group, frame chunk) CTAs: about 8 per SM in all
    const long long target = (long long)sm_count() * 8;
    int fpc = static_cast<int>(((long long)rowgroups * a.nframes) / std::max(target, 1LL));
    fpc = std::max(1, std::min(fpc, a.nframes));
    dim3 grid((a.nframes + fpc - 1) / fpc, rowgroups);
    launch_pdl(mix_rows_adjoint<N>, grid, lines * Cfg::B, Cfg::smem_adjoint(lines), s, a, lines, fpc);
  }
  static void cols(int mode, const MixColsArgs& a, cudaStream_t s) {
    using Cfg = ColCfg<N>;
    if (a.nframes <= 0) return;
    dim3 grid(num_tiles(a.pw) * (kTile / Cfg::C), a.nframes);
    if (mode == kMixColSweep) {
      launch_pdl(mix_cols<kMixColSweep, N>, grid, Cfg::THREADS, Cfg::SMEM, s, a);
    } else if (mode == kMixColForward) {
      launch_pdl(mix_cols<kMixColForward, N>, grid, Cfg::THREADS, Cfg::SMEM, s, a);
    } else {
      launch_pdl(mix_cols<kMixColBackward, N>, grid, Cfg::THREADS, Cfg::SMEM, s, a);
    }
  }
  static const MixOps* table() {
    static const MixOps ops{&prepare, &rows_forward, &rows_adjoint, &cols};
    return &ops;
  }
};

}  // namespace mixk
}  // namespace ptx
