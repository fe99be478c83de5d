// Conventional ptychography: forward, adjoint and the fused forward+loss+adjoint sweep.
//
// Math (python/ptychoX/base/ops.py:59-67 forward, :92-105 adjoint):
//   F_b = fft2(O[y_b:y_b+ph, x_b:x_b+pw] * P),   A_b = |fftshift(F_b)|
//   G_b = ifft2(ifftshift(g_b * F/max(|F|, eps))) * ph*pw
//   grad_O[window_b] += G_b conj(P),   grad_P += sum_b G_b conj(O_window_b)
//
// The 2-D transforms are split into a row pass and a column pass, and every pointwise
// step is fused into the pass that holds the data:
//   row pass   (gather O rows x probe rows, row DFT)                      -> scratch
//   col pass   (column DFT, |F|, residual vs sqrt(scale I), loss, phase,
//               inverse column DFT)                                        -> scratch
//   row pass   (inverse row DFT, scatter G conj(P) into grad_O with float2
//               atomics, accumulate G conj(O) for grad_P in registers)
// so exit waves and far fields never exist as separate arrays.  Scratch frames use a
// tiled layout [frame][tile][row][16] so both passes move contiguous runs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>

#include "ptx_internal.h"
#include "ptx_passes.cuh"

namespace ptx {
namespace {

constexpr size_t kHeaderBytes = 256 + kLutBytes;  // error word + padding, count-decode table
constexpr size_t kTargetScratch = 4096ull << 20;  // upper bound on workspace frames
constexpr float kEps = 1.1920928955078125e-07f;  // torch.finfo(float32).eps

enum ColMode { kColSweep = 0, kColForward = 1, kColBackward = 2 };

__device__ __forceinline__ bool window_ok(long long x0, long long y0, int ph, int pw, int H, int W) {
  return x0 >= 0 && y0 >= 0 && x0 + pw <= W && y0 + ph <= H;
}

// Row pass 1: gather O rows, multiply by the probe, forward row DFT, store tiled.
template <int NR>
__global__ void __launch_bounds__(256) base_rows_forward_rt(
    const float2* __restrict__ sample, int H, int W, const float2* __restrict__ probe, int ph, int pw,
    const int64_t* __restrict__ pos, int nframes, int frames_per_cta, float2* __restrict__ scratch,
    LinePlan plan, int lines, unsigned* __restrict__ err) {
  extern __shared__ float2 sm[];
  const int pitch = line_pitch(pw);
  const int tid = threadIdx.x;
  const int l = tid / plan.threads;
  const int t = (l < lines) ? tid - l * plan.threads : plan.threads;
  const int r0 = blockIdx.x * lines;
  const int nrows = min(lines, ph - r0);
  const int tiles = num_tiles(pw);
  const int f0 = blockIdx.y * frames_per_cta;
  const int f1 = min(nframes, f0 + frames_per_cta);
  float2* my_line = sm + min(l, lines - 1) * pitch;
  for (int f = f0; f < f1; ++f) {
    const long long x0 = pos[2 * f], y0 = pos[2 * f + 1];
    const bool ok = window_ok(x0, y0, ph, pw, H, W);
    if (!ok && tid == 0) atomicOr(err, 1u);
    for (int i = tid; i < nrows * pw; i += blockDim.x) {
      const int li = i / pw, c = i - li * pw;
      const int r = r0 + li;
      float2 v = make_float2(0.f, 0.f);
      if (ok) v = cmul(sample[(y0 + r) * W + x0 + c], __ldg(&probe[r * pw + c]));
      sm[li * pitch + c] = v;
    }
    __syncthreads();
    line_fft<NR, false>(my_line, plan, t);
    const int run = nrows * kTile;
    for (int i = tid; i < tiles * run; i += blockDim.x) {
      const int ct = i / run;
      const int rem = i - ct * run;
      const int li = rem / kTile, cc = rem - li * kTile;
      const int c = ct * kTile + cc;
      if (c < pw) scratch[(((size_t)f * tiles + ct) * ph + r0 + li) * kTile + cc] = sm[li * pitch + c];
    }
    __syncthreads();
  }
}

// Column pass.  kColSweep: column DFT, loss epilogue, inverse column DFT (in place).
// kColForward: column DFT, write fftshifted far field and amplitude.
// kColBackward: build g F/|F| from the saved far field, inverse column DFT.
template <int MODE, int NC>
__global__ void __launch_bounds__(512, 1) base_cols_rt(
    float2* __restrict__ scratch, int ph, int pw, int frame0, LinePlan plan, int cols,
    const uint16_t* __restrict__ measured, float scale, float grad_scale, double inv_numel,
    double* __restrict__ loss, float2* __restrict__ far_field, float* __restrict__ amplitude,
    const float* __restrict__ grad_output) {
  extern __shared__ float2 sm[];
  __shared__ double red[32];
  const int pitch = line_pitch(ph);
  const int tid = threadIdx.x;
  const int l = tid / plan.threads;
  const int t = (l < cols) ? tid - l * plan.threads : plan.threads;
  const int subs = kTile / cols;
  const int ct = blockIdx.x / subs;
  const int c0 = ct * kTile + (blockIdx.x - ct * subs) * cols;  // first column of this CTA
  const int f = blockIdx.y;
  const int tiles = num_tiles(pw);
  const int ncols = max(0, min(cols, pw - c0));
  float2* frame = scratch + ((size_t)f * tiles + ct) * ph * kTile + (c0 - ct * kTile);
  const size_t g = (size_t)frame0 + f;
  float2* my_line = sm + min(l, cols - 1) * pitch;
  const int hh = ph / 2, hw = pw / 2;
  const int nel = ph * cols;

  if (MODE != kColBackward) {
    for (int i = tid; i < nel; i += blockDim.x) {
      const int n = i / cols, cc = i - n * cols;
      sm[cc * pitch + n] = (cc < ncols) ? frame[n * kTile + cc] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    line_fft<NC, false>(my_line, plan, t);
  }

  if (MODE == kColSweep) {
    double acc = 0.0;
    for (int i = tid; i < nel; i += blockDim.x) {
      const int n = i / cols, cc = i - n * cols;
      if (cc >= ncols) continue;
      const int kc = c0 + cc;
      int ir = n + hh; if (ir >= ph) ir -= ph;
      int ic = kc + hw; if (ic >= pw) ic -= pw;
      const size_t idx = (g * ph + ir) * pw + ic;
      const float y = sqrtf(static_cast<float>(measured[idx]) * scale);
      const float2 F = sm[cc * pitch + n];
      const float a = cabsf(F);
      const float r = a - y;
      acc += static_cast<double>(r) * static_cast<double>(r);
      sm[cc * pitch + n] = cscale(F, grad_scale * r / fmaxf(a, kEps));
    }
    // block reduction of the FP64 loss partial
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((tid & 31) == 0) red[tid >> 5] = acc;
    __syncthreads();
    if (tid < 32) {
      const int nw = (blockDim.x + 31) >> 5;
      double v = (tid < nw) ? red[tid] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (tid == 0) atomicAdd(loss, v * inv_numel);
    }
  } else if (MODE == kColForward) {
    for (int i = tid; i < nel; i += blockDim.x) {
      const int n = i / cols, cc = i - n * cols;
      if (cc >= ncols) continue;
      const int kc = c0 + cc;
      int ir = n + hh; if (ir >= ph) ir -= ph;
      int ic = kc + hw; if (ic >= pw) ic -= pw;
      const size_t idx = (g * ph + ir) * pw + ic;
      const float2 F = sm[cc * pitch + n];
      if (far_field) far_field[idx] = F;
      amplitude[idx] = cabsf(F);
    }
    return;
  } else {  // kColBackward
    for (int i = tid; i < nel; i += blockDim.x) {
      const int n = i / cols, cc = i - n * cols;
      float2 v = make_float2(0.f, 0.f);
      if (cc < ncols) {
        const int kc = c0 + cc;
        int ir = n + hh; if (ir >= ph) ir -= ph;
        int ic = kc + hw; if (ic >= pw) ic -= pw;
        const size_t idx = (g * ph + ir) * pw + ic;
        const float2 F = far_field[idx];
        v = cscale(F, grad_output[idx] / fmaxf(cabsf(F), kEps));
      }
      sm[cc * pitch + n] = v;
    }
  }
  __syncthreads();
  line_fft<NC, true>(my_line, plan, t);
  for (int i = tid; i < nel; i += blockDim.x) {
    const int n = i / cols, cc = i - n * cols;
    if (cc < ncols) frame[n * kTile + cc] = sm[cc * pitch + n];
  }
}

// Row pass 2: inverse row DFT, scatter G conj(P) into grad_O, accumulate G conj(O).
constexpr int kOwn = kValuesPerThread;  // elements of a line owned by one thread

template <int NR>
__global__ void __launch_bounds__(256) base_rows_adjoint_rt(
    const float2* __restrict__ scratch, const float2* __restrict__ sample, int H, int W,
    const float2* __restrict__ probe, int ph, int pw, const int64_t* __restrict__ pos, int nframes,
    int frames_per_cta, float2* __restrict__ grad_sample, float2* __restrict__ grad_probe,
    LinePlan plan, int lines) {
  extern __shared__ float2 sm[];
  const int pitch = line_pitch(pw);
  const int tid = threadIdx.x;
  const int l = tid / plan.threads;
  const bool own = l < lines;
  const int t = own ? tid - l * plan.threads : plan.threads;
  const int r0 = blockIdx.x * lines;
  const int nrows = min(lines, ph - r0);
  const int r = r0 + l;
  const bool row_ok = own && r < ph;
  const int tiles = num_tiles(pw);
  const int f0 = blockIdx.y * frames_per_cta;
  const int f1 = min(nframes, f0 + frames_per_cta);
  float2* my_line = sm + min(l, lines - 1) * pitch;

  float2 pconj[kOwn];
  float2 acc[kOwn];
#pragma unroll
  for (int k = 0; k < kOwn; ++k) {
    const int c = t + k * plan.threads;
    acc[k] = make_float2(0.f, 0.f);
    pconj[k] = (row_ok && c < pw) ? cconj(__ldg(&probe[r * pw + c])) : make_float2(0.f, 0.f);
  }
  for (int f = f0; f < f1; ++f) {
    const long long x0 = pos[2 * f], y0 = pos[2 * f + 1];
    const bool ok = window_ok(x0, y0, ph, pw, H, W);
    const int run = nrows * kTile;
    for (int i = tid; i < tiles * run; i += blockDim.x) {
      const int ct = i / run;
      const int rem = i - ct * run;
      const int li = rem / kTile, cc = rem - li * kTile;
      const int c = ct * kTile + cc;
      if (c < pw) sm[li * pitch + c] = scratch[(((size_t)f * tiles + ct) * ph + r0 + li) * kTile + cc];
    }
    __syncthreads();
    line_fft<NR, true>(my_line, plan, t);
    if (row_ok && ok) {
      const float2* orow = sample + (y0 + r) * W + x0;
      float2* grow = grad_sample + (y0 + r) * W + x0;
#pragma unroll
      for (int k = 0; k < kOwn; ++k) {
        const int c = t + k * plan.threads;
        if (c < pw) {
          const float2 G = my_line[c];
          atomicAdd(&grow[c], cmul(G, pconj[k]));
          acc[k] = cadd(acc[k], cmulc(G, orow[c]));
        }
      }
    }
    __syncthreads();
  }
  if (row_ok) {
#pragma unroll
    for (int k = 0; k < kOwn; ++k) {
      const int c = t + k * plan.threads;
      if (c < pw) atomicAdd(&grad_probe[r * pw + c], acc[k]);
    }
  }
}


// ---------------------------------------------------------------------------------------
// Register-FFT kernels for power-of-two line lengths (the hot sizes).  Each thread keeps
// RegShape<N>::N1 values of its line in registers from the global load to the global
// store; one shared-memory transpose per 1-D transform.
// ---------------------------------------------------------------------------------------

template <int N>
struct RowCfg {
  static constexpr int LP = row_line_pitch<N>();
};

// Row pass 1 (register FFT): gather O rows x probe rows, forward row DFT, store tiled.
// Work units are (row group, frame) pairs in row-group-major order over one wave of
// resident CTAs (CTA b takes the contiguous units [u0, u1)).  The probe rows of the
// current row group and the twiddle table sit in shared memory; each unit's object rows
// arrive by 16-byte cp.async that bypasses L1 (evict-last in L2, the object is re-read by
// every frame) into the line buffer, and the next unit's rows are requested as soon as
// this unit's transform has released the buffer, so they land while it stores.
template <int N>
struct FwdCfg {
  static constexpr int BP = RowCfg<N>::LP > N + 2 ? RowCfg<N>::LP : N + 2;
  static_assert(BP % 2 == 0, "16-byte landing lines");
  static int smem(int lines) { return (lines * (BP + N) + N) * (int)sizeof(float2); }
};

template <int N>
__global__ void __launch_bounds__(128, 3) base_rows_forward_reg(
    const float2* __restrict__ sample, int H, int W, const float2* __restrict__ probe, int ph,
    const int64_t* __restrict__ pos, int nframes, int rowgroups, float2* __restrict__ scratch,
    const float2* __restrict__ tw, int lines, unsigned* __restrict__ err) {
  pdl_wait();
  using S = RegShape<N>;
  using Cfg = FwdCfg<N>;
  constexpr int kTiles = N / kTile;
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
  float2* pbuf = sm + lines * Cfg::BP + l * N;
  float2* tws = sm + lines * (Cfg::BP + N);
  load_twiddles_by_thread<N>(tws, tw);
  __syncthreads();
  const uint64_t pol_last = policy_evict_last();
  // object row of unit (row, frame) into buf; returns its shift (or -1 when not copied)
  auto request = [&](int row, int frame) -> int {
    const long long x0 = pos[2 * frame], y0 = pos[2 * frame + 1];
    if (row >= ph || !window_ok(x0, y0, ph, N, H, W)) return -1;
    const float2* orow = sample + (y0 + row) * W + x0;
    const int s = half_shift(orow);
    copy_row_shifted<N>(buf, orow, s, t, pol_last);
    cp_async_commit();
    return s;
  };
  int r = g * lines + l;
  int shift = request(r, f);
  bool new_group = true;
  for (long long u = u0; u < u1; ++u) {
    const bool row_ok = r < ph;
    if (tid == 0 && !window_ok(pos[2 * f], pos[2 * f + 1], ph, N, H, W)) atomicOr(err, 1u);
    if (new_group && row_ok) {
      // probe row of the new row group (each thread copies and later reads its own elements)
#pragma unroll
      for (int m = 0; m < S::N1; ++m) pbuf[t + S::T * m] = __ldg(&probe[(size_t)r * N + t + S::T * m]);
    }
    new_group = false;
    cp_async_wait_all();
    __syncwarp();
    float2 v[S::N1];
    if (shift >= 0) {
#pragma unroll
      for (int j = 0; j < S::N1; ++j) {
        const int c = t + S::T * j;
        v[j] = cmul(buf[c + shift], pbuf[c]);
      }
    } else {
#pragma unroll
      for (int j = 0; j < S::N1; ++j) v[j] = make_float2(0.f, 0.f);
    }
    __syncwarp();
    reg_fft<N, false, false, true>(v, buf, t, tws);
    const bool more = u + 1 < u1;
    int gn = g, fn = f + 1;
    if (fn == nframes) {
      gn = g + 1;
      fn = 0;
    }
    const int rn = gn * lines + l;
    const int shift_next = more ? request(rn, fn) : -1;
    if (row_ok) {
      float2* base = scratch + (size_t)f * kTiles * ph * kTile + (size_t)r * kTile;
#pragma unroll
      for (int m = 0; m < S::N1; ++m) {
        const int kc = t + S::T * m;
        base[(size_t)(kc / kTile) * ph * kTile + (kc % kTile)] = v[m];
      }
    }
    if (gn != g) new_group = true;
    g = gn;
    f = fn;
    r = rn;
    shift = shift_next;
  }
}

// Column pass (register FFT), same three modes as base_cols_rt.  A CTA owns kColsReg
// columns of one frame; threads run column-fastest (thread (t, c) owns column c).  In
// the sweep mode the uint16 counts of the CTA's columns are prefetched into shared
// memory with cp.async before the forward column DFT, so their latency hides behind it.
constexpr int kColsReg = 8;

template <int N>
struct ColCfg {
  static constexpr int LP = col_line_pitch<N>();
  static constexpr int kMeasOffsetBytes = ((kColsReg * LP * (int)sizeof(float2)) + 15) / 16 * 16;
  static constexpr int kSmemBytes = kMeasOffsetBytes + N * kColsReg * (int)sizeof(uint16_t);
};

template <int MODE, int N>
__global__ void __launch_bounds__(256, 2) base_cols_reg(
    float2* __restrict__ scratch, int pw, int frame0, const float2* __restrict__ tw,
    const uint16_t* __restrict__ measured, const float* __restrict__ lut, float grad_scale, double inv_numel,
    double* __restrict__ loss, float2* __restrict__ far_field, float* __restrict__ amplitude,
    const float* __restrict__ grad_output) {
  using S = RegShape<N>;
  constexpr int LP = ColCfg<N>::LP;
  extern __shared__ float2 sm[];
  __shared__ double red[32];
  uint16_t* meas_s = reinterpret_cast<uint16_t*>(reinterpret_cast<char*>(sm) + ColCfg<N>::kMeasOffsetBytes);
  const int tid = threadIdx.x;
  const int c = tid % kColsReg;
  const int t = tid / kColsReg;
  constexpr int kSubs = kTile / kColsReg;
  const int ct = blockIdx.x / kSubs;
  const int c0 = ct * kTile + (blockIdx.x - ct * kSubs) * kColsReg;  // first column of the CTA
  const int f = blockIdx.y;
  const int kc = c0 + c;
  const bool col_ok = kc < pw;
  const int tiles = num_tiles(pw);
  float2* tile = scratch + ((size_t)f * tiles + ct) * N * kTile + (c0 - ct * kTile);
  const size_t g = (size_t)frame0 + f;
  float2* buf = sm + c * LP;
  int ic = kc + pw / 2;
  if (ic >= pw) ic -= pw;
  float2 v[S::N1];

  if (MODE == kColSweep) {
    // counts of rows kr (unshifted) -> meas_s[kr][c]
    int ic0 = c0 + pw / 2;
    if (ic0 >= pw) ic0 -= pw;
    const bool fast = (pw % (2 * kColsReg) == 0) && ((reinterpret_cast<uintptr_t>(measured) & 15) == 0);
    if (fast) {
      for (int kr = tid; kr < N; kr += blockDim.x) {
        const int ir = (kr + N / 2) & (N - 1);
        cp_async16(meas_s + kr * kColsReg, measured + (g * N + ir) * pw + ic0);
      }
      cp_async_commit();
    } else {
      for (int i = tid; i < N * kColsReg; i += blockDim.x) {
        const int kr = i / kColsReg, cc = i - kr * kColsReg;
        const int ir = (kr + N / 2) & (N - 1);
        int icc = c0 + cc + pw / 2;
        if (icc >= pw) icc -= pw;
        meas_s[i] = (c0 + cc < pw) ? measured[(g * N + ir) * pw + icc] : 0;
      }
    }
  }

  if (MODE != kColBackward) {
#pragma unroll
    for (int j = 0; j < S::N1; ++j) {
      v[j] = col_ok ? tile[(t + S::T * j) * kTile + c] : make_float2(0.f, 0.f);
    }
    reg_fft<N, false, true>(v, buf, t, tw);
  }

  if (MODE == kColSweep) {
    cp_async_wait_all();
    __syncthreads();
    float part = 0.f;  // this thread's N1 squared residuals; summed in FP64 across the grid
#pragma unroll
    for (int m = 0; m < S::N1; ++m) {
      const int kr = t + S::T * m;
      const float2 F = v[m];
      float2 out = make_float2(0.f, 0.f);
      if (col_ok) {
        const float y = __ldg(&lut[meas_s[kr * kColsReg + c]]);
        float a, inv;
        abs_and_inv(F, kEps, a, inv);
        const float rr = a - y;
        part = fmaf(rr, rr, part);
        out = cscale(F, grad_scale * rr * inv);
      }
      v[m] = out;
    }
    double acc = static_cast<double>(part);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((tid & 31) == 0) red[tid >> 5] = acc;
    __syncthreads();
    if (tid < 32) {
      const int nw = (blockDim.x + 31) >> 5;
      double w = (tid < nw) ? red[tid] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
      if (tid == 0) atomicAdd(loss, w * inv_numel);
    }
  } else if (MODE == kColForward) {
    if (col_ok) {
#pragma unroll
      for (int m = 0; m < S::N1; ++m) {
        const int kr = t + S::T * m;
        const int ir = (kr + N / 2) & (N - 1);
        const size_t idx = (g * N + ir) * pw + ic;
        if (far_field) far_field[idx] = v[m];
        amplitude[idx] = cabsf(v[m]);
      }
    }
    return;
  } else {  // kColBackward
#pragma unroll
    for (int m = 0; m < S::N1; ++m) {
      const int kr = t + S::T * m;
      const int ir = (kr + N / 2) & (N - 1);
      float2 out = make_float2(0.f, 0.f);
      if (col_ok) {
        const size_t idx = (g * N + ir) * pw + ic;
        const float2 F = far_field[idx];
        out = cscale(F, grad_output[idx] / fmaxf(cabsf(F), kEps));
      }
      v[m] = out;
    }
  }
  reg_fft<N, true, true>(v, buf, t, tw);
  if (col_ok) {
#pragma unroll
    for (int m = 0; m < S::N1; ++m) tile[(t + S::T * m) * kTile + c] = v[m];
  }
}

// Shared memory of the adjoint row pass, per line: the exchange / scratch landing line
// (BP), the object row (OP = N + 2: a 16-byte aligned copy shifted by the row's 8-byte
// misalignment) and the probe row (N); per CTA: the twiddle table (N).
template <int N>
struct AdjCfg {
  static constexpr int BP = RowCfg<N>::LP > N ? RowCfg<N>::LP : N;
  static constexpr int OP = N + 2;
  static_assert(BP % 2 == 0, "16-byte landing lines");
  static int smem(int lines) { return (lines * (BP + OP + N) + N) * (int)sizeof(float2); }
};

// Row pass 2 (register FFT): inverse row DFT, scatter G conj(P) into grad_O, accumulate
// G conj(O) for grad_P in registers.  Work units are (row group, frame) pairs in
// row-group-major order; the grid is one wave of resident CTAs and CTA b takes the
// contiguous units [u0, u1), so every CTA does the same number of frame-rows and covers at
// most a few row groups.  Per unit the scratch rows and the object rows arrive by 16-byte
// cp.async that bypasses L1 (scratch marked evict-first in L2, the object evict-last), so
// L1 is left to the atomics; the probe rows of the current row group and the twiddle
// table sit in shared memory.  The next unit's scratch row lands while this unit scatters.
template <int N>
__global__ void __launch_bounds__(128, 2) base_rows_adjoint_reg(
    const float2* __restrict__ scratch, const float2* __restrict__ sample, int H, int W,
    const float2* __restrict__ probe, int ph, const int64_t* __restrict__ pos, int nframes, int rowgroups,
    float2* __restrict__ grad_sample, float2* __restrict__ grad_probe, const float2* __restrict__ tw, int lines) {
  pdl_wait();
  using S = RegShape<N>;
  using Cfg = AdjCfg<N>;
  constexpr int kTiles = N / kTile;
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
  float2* obuf = sm + lines * Cfg::BP + l * Cfg::OP;
  float2* pbuf = sm + lines * (Cfg::BP + Cfg::OP) + l * N;
  float2* tws = sm + lines * (Cfg::BP + Cfg::OP + N);
  load_twiddles_by_thread<N>(tws, tw);
  __syncthreads();
  const uint64_t pol_first = policy_evict_first();
  const uint64_t pol_last = policy_evict_last();
  float2 acc[S::N1];
#pragma unroll
  for (int m = 0; m < S::N1; ++m) acc[m] = make_float2(0.f, 0.f);
  // the scratch row (row, frame) into buf: N/2 16-byte chunks, chunk q = t + T i
  auto prefetch_row = [&](int row, int frame) {
    const float2* base = scratch + (size_t)frame * kTiles * ph * kTile + (size_t)row * kTile;
#pragma unroll
    for (int i = 0; i < S::N1 / 2; ++i) {
      const int c = 2 * (t + S::T * i);
      cp_async16_hint(buf + c, base + (size_t)(c / kTile) * ph * kTile + (c % kTile), pol_first);
    }
    cp_async_commit();
  };
  int r = g * lines + l;
  bool row_ok = r < ph;
  bool new_group = true;
  if (row_ok) prefetch_row(r, f);
  for (long long u = u0; u < u1; ++u) {
    const long long x0 = pos[2 * f], y0 = pos[2 * f + 1];
    const bool ok = window_ok(x0, y0, ph, N, H, W);
    const float2* orow = sample + (y0 + r) * W + x0;
    const int shift = half_shift(orow);
    if (row_ok && ok) {
      copy_row_shifted<N>(obuf, orow, shift, t, pol_last);
      cp_async_commit();
    }
    if (new_group && row_ok) {
      // probe row of the new row group (each thread copies and later reads its own elements)
#pragma unroll
      for (int m = 0; m < S::N1; ++m) pbuf[t + S::T * m] = __ldg(&probe[(size_t)r * N + t + S::T * m]);
    }
    new_group = false;
    float2 v[S::N1];
    if (row_ok) {
      // the scratch row (committed before the object row); other lanes of the line copied
      // part of it, so the line's lanes meet at a warp barrier before reading
      if (ok) {
        asm volatile("cp.async.wait_group 1;\n" ::: "memory");
      } else {
        cp_async_wait_all();
      }
    }
    __syncwarp();
    if (row_ok) {
#pragma unroll
      for (int j = 0; j < S::N1; ++j) v[j] = buf[t + S::T * j];
    } else {
#pragma unroll
      for (int j = 0; j < S::N1; ++j) v[j] = make_float2(0.f, 0.f);
    }
    __syncwarp();
    reg_fft<N, true, false, true>(v, buf, t, tws);
    const bool more = u + 1 < u1;
    int gn = g, fn = f + 1;
    if (fn == nframes) {
      gn = g + 1;
      fn = 0;
    }
    const int rn = gn * lines + l;
    const bool pf = more && rn < ph;
    if (pf) prefetch_row(rn, fn);
    if (row_ok && ok) {
      float2* grow = grad_sample + (y0 + r) * W + x0;
      if (pf) {
        asm volatile("cp.async.wait_group 1;\n" ::: "memory");
      } else {
        cp_async_wait_all();
      }
      __syncwarp();
#pragma unroll
      for (int m = 0; m < S::N1; ++m) {
        const int c = t + S::T * m;
        const float2 G = v[m];
        atomicAdd(&grow[c], cmulc(G, pbuf[c]));
        acc[m] = cadd(acc[m], cmulc(G, obuf[c + shift]));
      }
    } else {
      __syncwarp();
    }
    if (!more || gn != g) {
      if (row_ok) {
#pragma unroll
        for (int m = 0; m < S::N1; ++m) {
          atomicAdd(&grad_probe[(size_t)r * N + t + S::T * m], acc[m]);
          acc[m] = make_float2(0.f, 0.f);
        }
      }
      new_group = true;
    }
    g = gn;
    f = fn;
    r = rn;
    row_ok = rn < ph;
  }
}

// ---------------------------------------------------------------------------------------
// Small frames (square power-of-two probes up to 128): the whole sweep of a frame in one
// CTA.  A 128 x 128 complex frame is 128 KB, so it stays in shared memory from the gather
// to the gradient scatter: gather O x P, row DFTs, column DFTs with the loss epilogue and the
// inverse column DFTs, inverse row DFTs and the scatter of G conj(P) into grad_O and
// G conj(O) into grad_P (float2 atomics), with no scratch frames in HBM and one launch per
// sweep.  CTAs are persistent over frames (frame f = blockIdx.x + k gridDim.x).  The same
// arithmetic as the three-pass sweep: register DFTs of the rows and columns, the amplitude
// epilogue on fftshifted counts decoded through the table.
// STAGE: the frame's counts land in shared memory by cp.async during the gather and row
// DFTs (row pitch N + 8: the column epilogue's reads of 8 rows x 4 columns per warp hit
// distinct banks) instead of being read from global memory in the column epilogue (2% of
// the 121 x 128^2 sweep); it needs 16-byte aligned counts.
template <int N, bool STAGE>
struct FrameCfg {
  static constexpr int kThreads = 256;
  static constexpr int T = RegShape<N>::T;
  static constexpr int kLines = kThreads / T;          // lines transformed at once
  static constexpr int FP = N + 4;                     // frame row pitch (float2): conflict-free columns
  static constexpr int LP = row_line_pitch<N>();       // exchange buffer per line
  static constexpr int kFrameF2 = N * FP;
  static constexpr int CP = N + 8;                     // staged count row pitch (uint16)
  static constexpr int kSmemBytes =
      (kFrameF2 + kLines * LP) * (int)sizeof(float2) + (STAGE ? N * CP * (int)sizeof(uint16_t) : 0);
};

template <int N, bool STAGE>
__global__ void __launch_bounds__(256, 1) base_sweep_frame(
    const float2* __restrict__ sample, int H, int W, const float2* __restrict__ probe,
    const int64_t* __restrict__ pos, int nframes, const uint16_t* __restrict__ measured,
    const float* __restrict__ lut, float grad_scale, double inv_numel, double* __restrict__ loss,
    float2* __restrict__ grad_sample, float2* __restrict__ grad_probe, const float2* __restrict__ tw,
    unsigned* __restrict__ err) {
  pdl_wait();
  using S = RegShape<N>;
  using Cfg = FrameCfg<N, STAGE>;
  extern __shared__ float2 sm[];
  float2* F = sm;                                       // [N][FP]
  const int tid = threadIdx.x;
  const int l = tid / S::T, t = tid - l * S::T;
  float2* buf = sm + Cfg::kFrameF2 + l * Cfg::LP;
  uint16_t* cnt_s = reinterpret_cast<uint16_t*>(sm + Cfg::kFrameF2 + Cfg::kLines * Cfg::LP);  // [N][CP]
  double part = 0.0;
  for (int f = blockIdx.x; f < nframes; f += gridDim.x) {
    const long long x0 = pos[2 * f], y0 = pos[2 * f + 1];
    if (!window_ok(x0, y0, N, N, H, W)) {
      if (tid == 0) atomicOr(err, 1u);
      continue;  // uniform across the CTA
    }
    if constexpr (STAGE) {
      // 16-byte pieces of the frame's counts (the previous frame's epilogue read cnt_s before
      // the barrier that ends its iteration)
      const uint16_t* src = measured + (size_t)f * N * N;
      for (int i = tid; i < N * N / 8; i += Cfg::kThreads) {
        const int r = i / (N / 8), q = i - r * (N / 8);
        cp_async16(cnt_s + r * Cfg::CP + 8 * q, src + (size_t)r * N + 8 * q);
      }
      cp_async_commit();
    }
    const float2* win = sample + y0 * W + x0;
    // gather O x P
    for (int i = tid; i < N * N; i += Cfg::kThreads) {
      const int r = i / N, c = i - r * N;
      F[r * Cfg::FP + c] = cmul(win[(size_t)r * W + c], __ldg(&probe[i]));
    }
    __syncthreads();
    // forward row DFTs
    for (int r = l; r < N; r += Cfg::kLines) {
      float2 v[S::N1];
#pragma unroll
      for (int j = 0; j < S::N1; ++j) v[j] = F[r * Cfg::FP + t + S::T * j];
      reg_fft<N, false, false>(v, buf, t, tw);
#pragma unroll
      for (int m = 0; m < S::N1; ++m) F[r * Cfg::FP + t + S::T * m] = v[m];
    }
    if constexpr (STAGE) cp_async_wait_all();
    __syncthreads();
    // column DFTs, amplitude-loss epilogue against the fftshifted counts, inverse column DFTs
    const uint16_t* cnt = measured + (size_t)f * N * N;
    for (int c = l; c < N; c += Cfg::kLines) {
      float2 v[S::N1];
#pragma unroll
      for (int j = 0; j < S::N1; ++j) v[j] = F[(t + S::T * j) * Cfg::FP + c];
      reg_fft<N, false, false>(v, buf, t, tw);
      const int ic = (c + N / 2) & (N - 1);
#pragma unroll
      for (int m = 0; m < S::N1; ++m) {
        const int kr = t + S::T * m;
        const int ir = (kr + N / 2) & (N - 1);
        const float y = __ldg(&lut[STAGE ? cnt_s[ir * Cfg::CP + ic] : cnt[ir * N + ic]]);
        float a, inv;
        abs_and_inv(v[m], kEps, a, inv);
        const float rr = a - y;
        part += static_cast<double>(rr * rr);
        v[m] = cscale(v[m], grad_scale * rr * inv);
      }
      reg_fft<N, true, false>(v, buf, t, tw);
#pragma unroll
      for (int j = 0; j < S::N1; ++j) F[(t + S::T * j) * Cfg::FP + c] = v[j];
    }
    __syncthreads();
    // inverse row DFTs and the gradient scatter
    float2* gwin = grad_sample + y0 * W + x0;
    for (int r = l; r < N; r += Cfg::kLines) {
      float2 v[S::N1];
#pragma unroll
      for (int j = 0; j < S::N1; ++j) v[j] = F[r * Cfg::FP + t + S::T * j];
      reg_fft<N, true, false>(v, buf, t, tw);
#pragma unroll
      for (int m = 0; m < S::N1; ++m) {
        const int c = t + S::T * m;
        const float2 G = v[m];
        atomicAdd(&gwin[(size_t)r * W + c], cmulc(G, __ldg(&probe[r * N + c])));
        atomicAdd(&grad_probe[r * N + c], cmulc(G, win[(size_t)r * W + c]));
      }
    }
    __syncthreads();
  }
  block_add_double(part, inv_numel, loss);
}

template <int N>
struct RegLaunch {
  static constexpr int T = RegShape<N>::T;
  // rows per CTA (multiple of 32 / T so the block is whole warps)
  static int lines(int threads, int ph) {
    int l = threads / T;
    const int quantum = T >= 32 ? 1 : 32 / T;
    const int need = ((ph + quantum - 1) / quantum) * quantum;
    return l < need ? l : need;
  }
  static int row_smem(int lines) { return lines * RowCfg<N>::LP * (int)sizeof(float2); }
  static int adj_smem(int lines) { return AdjCfg<N>::smem(lines); }
  static int col_threads() { return kColsReg * T; }
  static int col_smem() { return ColCfg<N>::kSmemBytes; }
};

// Flag (bit 0 of *err) a window of `pos` that leaves the H x W object.  Used by the adjoint
// entry point, whose row passes skip such windows without flagging them.
static __global__ void window_check_kernel(const int64_t* __restrict__ pos, int n, int ph, int pw, int H, int W,
                                           unsigned* __restrict__ err) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < n && !window_ok(pos[2 * b], pos[2 * b + 1], ph, pw, H, W)) atomicOr(err, 1u);
}

struct BaseGeom {
  int H, W, ph, pw, batch;
  LinePlan row, col;
  RowShape rs;
  ColShape cs;
  size_t frame_bytes;
  int chunk;
  unsigned* err;
  float* lut;
  float2* scratch;
};

int check_common(const void* sample, int H, int W, const void* probe, int ph, int pw,
                 const int64_t* pos, int batch, void* ws, size_t ws_bytes, BaseGeom* g) {
  if (!sample || !probe || (!pos && batch > 0) || !ws) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "null pointer argument");
  }
  if (H <= 0 || W <= 0 || ph <= 0 || pw <= 0 || batch < 0) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "non-positive shape");
  }
  if (reinterpret_cast<uintptr_t>(ws) & 255) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "workspace must start on a 256-byte boundary");
  }
  if (ph > H || pw > W) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "probe (%d x %d) larger than sample (%d x %d)", ph, pw, H, W);
  }
  g->H = H; g->W = W; g->ph = ph; g->pw = pw; g->batch = batch;
  if (int st = get_line_plan(pw, &g->row)) return st;
  if (int st = get_line_plan(ph, &g->col)) return st;
  if ((mix_ops(pw) && !g->row.mix_twt) || (mix_ops(ph) && !g->col.mix_twt)) {
    return set_error(PTX_ERR_UNSUPPORTED_SIZE, "no mixed-radix twiddle tables for %d x %d", ph, pw);
  }
  g->rs = row_shape(g->row, ph);
  g->cs = col_shape(g->col);
  g->frame_bytes = (size_t)num_tiles(pw) * kTile * ph * sizeof(float2);
  if (ws_bytes < kHeaderBytes + g->frame_bytes) {
    return set_error(PTX_ERR_WORKSPACE, "workspace of %zu bytes is smaller than one frame (%zu)",
                     ws_bytes, kHeaderBytes + g->frame_bytes);
  }
  size_t fit = (ws_bytes - kHeaderBytes) / g->frame_bytes;
  // frames of one chunk: what the workspace holds, at most the batch, and at most 65535
  // (the column passes put the frame in gridDim.y)
  g->chunk = static_cast<int>(std::min<size_t>({fit, (size_t)std::max(batch, 1), (size_t)65535}));
  g->err = reinterpret_cast<unsigned*>(ws);
  g->lut = reinterpret_cast<float*>(static_cast<char*>(ws) + 256);
  g->scratch = reinterpret_cast<float2*>(static_cast<char*>(ws) + kHeaderBytes);
  int st = PTX_OK;
  dispatch_len(pw, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    if constexpr (N > 0) {
      using L = RegLaunch<N>;
      if (!st) st = ensure_smem((const void*)base_rows_forward_reg<N>, FwdCfg<N>::smem(L::lines(128, ph)));
      if (!st) st = ensure_smem((const void*)base_rows_adjoint_reg<N>, L::adj_smem(L::lines(128, ph)));
    } else if (const MixOps* mo = mix_ops(pw)) {
      if (!st) st = mo->prepare();
    } else {
      if (!st) st = ensure_smem((const void*)base_rows_forward_rt<0>, g->rs.smem);
      if (!st) st = ensure_smem((const void*)base_rows_adjoint_rt<0>, g->rs.smem);
    }
  });
  dispatch_len(ph, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    if constexpr (N > 0) {
      const int sm = RegLaunch<N>::col_smem();
      if (!st) st = ensure_smem((const void*)cols_sweep_pair<N, false, true>, ColPairCfg<N>::kSmemBytes);
      if (!st) st = ensure_smem((const void*)cols_sweep_pair<N, false, true, true, true>, ColPairCfg<N>::kSmemBytes);
      if (!st) st = ensure_smem((const void*)base_cols_reg<kColForward, N>, sm);
      if (!st) st = ensure_smem((const void*)base_cols_reg<kColBackward, N>, sm);
    } else if (const MixOps* mo = mix_ops(ph)) {
      if (!st) st = mo->prepare();
    } else {
      if (!st) st = ensure_smem((const void*)base_cols_rt<kColSweep, 0>, g->cs.smem);
      if (!st) st = ensure_smem((const void*)base_cols_rt<kColForward, 0>, g->cs.smem);
      if (!st) st = ensure_smem((const void*)base_cols_rt<kColBackward, 0>, g->cs.smem);
    }
  });
  if (st) return st;
  return PTX_OK;
}

int frames_per_cta_for(int rowgroups, int nframes, int target_ctas) {
  const long long ctas_one = (long long)rowgroups * nframes;
  int fpc = static_cast<int>(ctas_one / std::max(target_ctas, 1));
  return std::max(1, std::min(fpc, nframes));
}

void launch_rows_forward(const BaseGeom& g, const float2* sample, const float2* probe, const int64_t* pos,
                         int nframes, cudaStream_t s) {
  prof_begin(kBaseRowsForward, s);
  dispatch_len(g.pw, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    if constexpr (N > 0) {
      using L = RegLaunch<N>;
      const int lines = L::lines(128, g.ph);
      const int rowgroups = (g.ph + lines - 1) / lines;
      const int threads = lines * L::T, smem = FwdCfg<N>::smem(lines);
      const int grid = persistent_grid((const void*)base_rows_forward_reg<N>, threads, smem, (long long)rowgroups * nframes);
      launch_pdl(base_rows_forward_reg<N>, grid, threads, smem, s, sample, g.H, g.W, probe, g.ph, pos, nframes, rowgroups,
                                                           g.scratch, g.row.tw, lines, g.err);
    } else if (const MixOps* mo = mix_ops(g.pw)) {
      MixRowsArgs a{sample, g.H, g.W, probe, g.ph, g.pw, pos, nframes, g.scratch, g.row.mix_twt, g.row.mix_twi,
                    g.err, nullptr, nullptr};
      mo->rows_forward(a, s);
    } else {
      const int rowgroups = (g.ph + g.rs.lines - 1) / g.rs.lines;
      dim3 grid(rowgroups, nframes);
      base_rows_forward_rt<0><<<grid, g.rs.threads, g.rs.smem, s>>>(sample, g.H, g.W, probe, g.ph, g.pw, pos,
                                                                    nframes, 1, g.scratch, g.row, g.rs.lines, g.err);
    }
  });
  prof_end(kBaseRowsForward, s);
}

void launch_rows_adjoint(const BaseGeom& g, const float2* sample, const float2* probe, const int64_t* pos,
                         int nframes, float2* grad_sample, float2* grad_probe, cudaStream_t s) {
  prof_begin(kBaseRowsAdjoint, s);
  dispatch_len(g.pw, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    if constexpr (N > 0) {
      using L = RegLaunch<N>;
      const int lines = L::lines(128, g.ph);
      const int rowgroups = (g.ph + lines - 1) / lines;
      const int threads = lines * L::T, smem = L::adj_smem(lines);
      const long long units = (long long)rowgroups * nframes;
      const int grid = persistent_grid((const void*)base_rows_adjoint_reg<N>, threads, smem, units);
      launch_pdl(base_rows_adjoint_reg<N>, grid, threads, smem, s, g.scratch, sample, g.H, g.W, probe, g.ph, pos, nframes,
                                                           rowgroups, grad_sample, grad_probe, g.row.tw, lines);
    } else if (const MixOps* mo = mix_ops(g.pw)) {
      MixRowsArgs a{sample, g.H, g.W, probe, g.ph, g.pw, pos, nframes, g.scratch, g.row.mix_twt, g.row.mix_twi,
                    g.err, grad_sample, grad_probe};
      mo->rows_adjoint(a, s);
    } else {
      const int rowgroups = (g.ph + g.rs.lines - 1) / g.rs.lines;
      const int fpc = frames_per_cta_for(rowgroups, nframes, sm_count() * 8);
      dim3 grid(rowgroups, (nframes + fpc - 1) / fpc);
      base_rows_adjoint_rt<0><<<grid, g.rs.threads, g.rs.smem, s>>>(g.scratch, sample, g.H, g.W, probe, g.ph,
                                                                    g.pw, pos, nframes, fpc, grad_sample,
                                                                    grad_probe, g.row, g.rs.lines);
    }
  });
  prof_end(kBaseRowsAdjoint, s);
}

template <int MODE>
void launch_cols(const BaseGeom& g, int frame0, int nframes, const uint16_t* measured, float scale,
                 float grad_scale, double inv_numel, double* loss, float2* far_field, float* amplitude,
                 const float* grad_output, cudaStream_t s) {
  prof_begin(kBaseCols, s);
  dispatch_len(g.ph, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    if constexpr (N > 0) {
      using L = RegLaunch<N>;
      if constexpr (MODE == kColSweep) {
        // column DFT, amplitude-loss epilogue and inverse column DFT; counts fftshifted
        dim3 grid(num_tiles(g.pw), nframes);
        if (g.pw % kTile == 0) {
          launch_pdl(cols_sweep_pair<N, false, true, true, true>, grid, ColPairCfg<N>::kThreads, ColPairCfg<N>::kSmemBytes, s,
              g.scratch, g.pw, frame0, g.col.tw, measured, g.lut, 1.0f, grad_scale, inv_numel, loss);
        } else {
          launch_pdl(cols_sweep_pair<N, false, true>, grid, ColPairCfg<N>::kThreads, ColPairCfg<N>::kSmemBytes, s,
              g.scratch, g.pw, frame0, g.col.tw, measured, g.lut, 1.0f, grad_scale, inv_numel, loss);
        }
        return;
      }
      dim3 grid(num_tiles(g.pw) * (kTile / kColsReg), nframes);
      base_cols_reg<MODE, N><<<grid, L::col_threads(), L::col_smem(), s>>>(
          g.scratch, g.pw, frame0, g.col.tw, measured, g.lut, grad_scale, inv_numel, loss, far_field, amplitude,
          grad_output);
    } else if (const MixOps* mo = mix_ops(g.ph)) {
      MixColsArgs a{g.scratch, g.ph, g.pw, frame0, nframes, g.col.mix_twt, g.col.mix_twi, measured, g.lut,
                    grad_scale, inv_numel, loss, far_field, amplitude, grad_output};
      mo->cols(MODE == kColSweep ? kMixColSweep : MODE == kColForward ? kMixColForward : kMixColBackward, a, s);
    } else {
      dim3 grid(num_tiles(g.pw) * (kTile / g.cs.cols), nframes);
      base_cols_rt<MODE, 0><<<grid, g.cs.threads, g.cs.smem, s>>>(g.scratch, g.ph, g.pw, frame0, g.col,
                                                                  g.cs.cols, measured, scale, grad_scale,
                                                                  inv_numel, loss, far_field, amplitude,
                                                                  grad_output);
    }
  });
  prof_end(kBaseCols, s);
}

}  // namespace

int base_cols_pass(bool forward, float2* scratch, int ph, int pw, int frame0, int nframes, float2* far_field,
                   float* amplitude, const float* grad_output, cudaStream_t s) {
  BaseGeom g{};
  g.ph = ph;
  g.pw = pw;
  g.scratch = scratch;
  if (int st = get_line_plan(ph, &g.col)) return st;
  if (mix_ops(ph) && !g.col.mix_twt) {
    return set_error(PTX_ERR_UNSUPPORTED_SIZE, "no mixed-radix twiddle tables for length %d", ph);
  }
  g.cs = col_shape(g.col);
  int st = PTX_OK;
  dispatch_len(ph, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    if constexpr (N > 0) {
      const int sm = RegLaunch<N>::col_smem();
      st = ensure_smem(forward ? (const void*)base_cols_reg<kColForward, N> : (const void*)base_cols_reg<kColBackward, N>,
                       sm);
    } else if (const MixOps* mo = mix_ops(ph)) {
      st = mo->prepare();
    } else {
      st = ensure_smem(forward ? (const void*)base_cols_rt<kColForward, 0> : (const void*)base_cols_rt<kColBackward, 0>,
                       g.cs.smem);
    }
  });
  if (st) return st;
  if (forward) {
    launch_cols<kColForward>(g, frame0, nframes, nullptr, 0.f, 0.f, 0.0, nullptr, far_field, amplitude, nullptr, s);
  } else {
    launch_cols<kColBackward>(g, frame0, nframes, nullptr, 0.f, 0.f, 0.0, nullptr, far_field, nullptr, grad_output, s);
  }
  return PTX_OK;
}

}  // namespace ptx

using namespace ptx;

extern "C" {

size_t ptx_base_workspace_bytes(int probe_h, int probe_w, int batch) {
  if (probe_h <= 0 || probe_w <= 0) return 0;
  const size_t frame = (size_t)num_tiles(probe_w) * kTile * probe_h * sizeof(float2);
  size_t frames = std::max<size_t>(1, kTargetScratch / frame);
  frames = std::min<size_t>(frames, (size_t)std::max(batch, 1));
  return kHeaderBytes + frames * frame;
}

int ptx_base_forward(const float* sample, int sample_h, int sample_w, const float* probe, int probe_h,
                     int probe_w, const int64_t* positions_xy, int batch, float* far_field, float* amplitude,
                     void* workspace, size_t workspace_bytes, void* stream) {
  BaseGeom g;
  if (int st = check_common(sample, sample_h, sample_w, probe, probe_h, probe_w, positions_xy, batch, workspace,
                            workspace_bytes, &g)) {
    return st;
  }
  if (!amplitude && batch > 0) return set_error(PTX_ERR_INVALID_ARGUMENT, "amplitude is null");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaMemsetAsync(g.err, 0, sizeof(unsigned), s);
  const float2* S = reinterpret_cast<const float2*>(sample);
  const float2* P = reinterpret_cast<const float2*>(probe);
  for (int b0 = 0; b0 < batch; b0 += g.chunk) {
    const int nf = std::min(g.chunk, batch - b0);
    launch_rows_forward(g, S, P, positions_xy + 2 * (size_t)b0, nf, s);
    launch_cols<kColForward>(g, b0, nf, nullptr, 0.f, 0.f, 0.0, nullptr, reinterpret_cast<float2*>(far_field),
                             amplitude, nullptr, s);
  }
  return cuda_status(cudaGetLastError(), "ptx_base_forward launch");
}

int ptx_base_backward(const float* grad_output, const float* far_field, const float* sample, int sample_h,
                      int sample_w, const float* probe, int probe_h, int probe_w, const int64_t* positions_xy,
                      int batch, float* grad_sample, float* grad_probe, void* workspace, size_t workspace_bytes,
                      void* stream) {
  BaseGeom g;
  if (int st = check_common(sample, sample_h, sample_w, probe, probe_h, probe_w, positions_xy, batch, workspace,
                            workspace_bytes, &g)) {
    return st;
  }
  if (((!grad_output || !far_field) && batch > 0) || !grad_sample || !grad_probe) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "null pointer argument");
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  float2* GS = reinterpret_cast<float2*>(grad_sample);
  float2* GP = reinterpret_cast<float2*>(grad_probe);
  cudaMemsetAsync(GS, 0, sizeof(float2) * (size_t)sample_h * sample_w, s);
  cudaMemsetAsync(GP, 0, sizeof(float2) * (size_t)probe_h * probe_w, s);
  cudaMemsetAsync(g.err, 0, sizeof(unsigned), s);
  if (batch > 0) {
    prof_begin(kMiscKernel, s);
    window_check_kernel<<<(batch + 255) / 256, 256, 0, s>>>(positions_xy, batch, probe_h, probe_w, sample_h, sample_w,
                                                            g.err);
    prof_end(kMiscKernel, s);
  }
  const float2* S = reinterpret_cast<const float2*>(sample);
  const float2* P = reinterpret_cast<const float2*>(probe);
  for (int b0 = 0; b0 < batch; b0 += g.chunk) {
    const int nf = std::min(g.chunk, batch - b0);
    launch_cols<kColBackward>(g, b0, nf, nullptr, 0.f, 0.f, 0.0, nullptr,
                              const_cast<float2*>(reinterpret_cast<const float2*>(far_field)), nullptr, grad_output,
                              s);
    launch_rows_adjoint(g, S, P, positions_xy + 2 * (size_t)b0, nf, GS, GP, s);
  }
  return cuda_status(cudaGetLastError(), "ptx_base_backward launch");
}

int ptx_base_sweep(const float* sample, int sample_h, int sample_w, const float* probe, int probe_h, int probe_w,
                   const int64_t* positions_xy, int batch, const uint16_t* measured, float scale, double* loss,
                   float* grad_sample, float* grad_probe, void* workspace, size_t workspace_bytes, void* stream) {
  BaseGeom g;
  if (int st = check_common(sample, sample_h, sample_w, probe, probe_h, probe_w, positions_xy, batch, workspace,
                            workspace_bytes, &g)) {
    return st;
  }
  if ((!measured && batch > 0) || !loss || !grad_sample || !grad_probe) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "null pointer argument");
  }
  if (!(scale > 0.f)) return set_error(PTX_ERR_INVALID_ARGUMENT, "scale must be positive");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  float2* GS = reinterpret_cast<float2*>(grad_sample);
  float2* GP = reinterpret_cast<float2*>(grad_probe);
  const double numel = (double)batch * probe_h * probe_w;
  const float grad_scale = static_cast<float>(2.0 / std::max(numel, 1.0));
  {
    const size_t ns = (size_t)sample_h * sample_w, np = (size_t)probe_h * probe_w;
    prof_begin(kMiscKernel, s);
    launch_pdl(sweep_prologue_kernel, prologue_blocks(ns, sm_count()), 256, 0, s, GS, ns, GP, np, loss, g.err, g.lut, scale);
    prof_end(kMiscKernel, s);
  }
  const float2* S = reinterpret_cast<const float2*>(sample);
  const float2* P = reinterpret_cast<const float2*>(probe);
  for (int b0 = 0; b0 < batch; b0 += g.chunk) {
    const int nf = std::min(g.chunk, batch - b0);
    const int64_t* pos = positions_xy + 2 * (size_t)b0;
    launch_rows_forward(g, S, P, pos, nf, s);
    launch_cols<kColSweep>(g, b0, nf, measured, scale, grad_scale, 1.0 / std::max(numel, 1.0), loss, nullptr,
                           nullptr, nullptr, s);
    launch_rows_adjoint(g, S, P, pos, nf, GS, GP, s);
  }
  return cuda_status(cudaGetLastError(), "ptx_base_sweep launch");
}

int ptx_workspace_status(const void* workspace, unsigned* status, void* stream) {
  if (!workspace || !status) return set_error(PTX_ERR_INVALID_ARGUMENT, "null pointer argument");
  if (reinterpret_cast<uintptr_t>(workspace) & 255) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "workspace must start on a 256-byte boundary");
  }
  return cuda_status(cudaMemcpyAsync(status, workspace, sizeof(unsigned), cudaMemcpyDefault,
                                     static_cast<cudaStream_t>(stream)),
                     "ptx_workspace_status copy");
}

int ptx_status_code(unsigned status) { return (status & 1u) ? PTX_ERR_OUT_OF_BOUNDS : PTX_OK; }

int ptx_base_sweep_small(const float* sample, int sample_h, int sample_w, const float* probe, int probe_h,
                         int probe_w, const int64_t* positions_xy, int batch, const uint16_t* measured, float scale,
                         double* loss, float* grad_sample, float* grad_probe, void* workspace, size_t workspace_bytes,
                         void* stream) {
  if (!(probe_h == probe_w && (probe_w == 32 || probe_w == 64 || probe_w == 128))) {
    return set_error(PTX_ERR_UNSUPPORTED_SIZE, "ptx_base_sweep_small takes square 32, 64 or 128 probes (got %d x %d)",
                     probe_h, probe_w);
  }
  BaseGeom g;
  if (int st = check_common(sample, sample_h, sample_w, probe, probe_h, probe_w, positions_xy, batch, workspace,
                            workspace_bytes, &g)) {
    return st;
  }
  if ((!measured && batch > 0) || !loss || !grad_sample || !grad_probe) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "null pointer argument");
  }
  if (!(scale > 0.f)) return set_error(PTX_ERR_INVALID_ARGUMENT, "scale must be positive");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  float2* GS = reinterpret_cast<float2*>(grad_sample);
  float2* GP = reinterpret_cast<float2*>(grad_probe);
  const double numel = (double)batch * probe_h * probe_w;
  const float grad_scale = static_cast<float>(2.0 / std::max(numel, 1.0));
  {
    const size_t ns = (size_t)sample_h * sample_w, np = (size_t)probe_h * probe_w;
    prof_begin(kMiscKernel, s);
    launch_pdl(sweep_prologue_kernel, prologue_blocks(ns, sm_count()), 256, 0, s, GS, ns, GP, np, loss, g.err, g.lut, scale);
    prof_end(kMiscKernel, s);
  }
  if (batch == 0) return cuda_status(cudaGetLastError(), "ptx_base_sweep_small launch");
  const float2* S = reinterpret_cast<const float2*>(sample);
  const float2* P = reinterpret_cast<const float2*>(probe);
  int st = PTX_OK;
  dispatch_len(probe_w, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    if constexpr (N == 32 || N == 64 || N == 128) {
      auto run = [&](auto kern, int threads, int smem) {
        st = ensure_smem((const void*)kern, smem);
        if (st) return;
        const int grid = persistent_grid((const void*)kern, threads, smem, batch);
        prof_begin(kBaseRowsForward, s);
        launch_pdl(kern, grid, threads, smem, s, S, sample_h, sample_w, P, positions_xy, batch, measured, g.lut,
                   grad_scale, 1.0 / std::max(numel, 1.0), loss, GS, GP, g.row.tw, g.err);
        prof_end(kBaseRowsForward, s);
      };
      if ((reinterpret_cast<uintptr_t>(measured) & 15) == 0) {
        using Cfg = FrameCfg<N, true>;
        run(base_sweep_frame<N, true>, Cfg::kThreads, Cfg::kSmemBytes);
      } else {
        using Cfg = FrameCfg<N, false>;
        run(base_sweep_frame<N, false>, Cfg::kThreads, Cfg::kSmemBytes);
      }
    }
  });
  if (st) return st;
  return cuda_status(cudaGetLastError(), "ptx_base_sweep_small launch");
}

}  // extern "C"
