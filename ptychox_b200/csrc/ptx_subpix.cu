// Conventional ptychography at sub-pixel scan positions.
//
// The reference crops integer windows only (python/ptychoX/base/ops.py:61-62).  Here a float
// position (x, y) takes the window at the rounded corner (x0, y0) = floor(p + 1/2) and shifts
// it by the fraction (dx, dy) = p - (x0, y0) with a Fourier phase ramp -- the reference's
// shift_phase_ramp (coded/ops.py:157-171) applied to the patch, i.e. a band-limited circular
// shift S = ifft2(fft2(C) exp(2 pi i (dx kx / pw + dy ky / ph))) -- before the probe
// multiply and the conventional far field A = |fftshift(fft2(S P))|.
//
// The ramp is separable, so the shift splits into a column shift and a row shift, and the
// sweep is five passes over tiled scratch frames ([tile][row][16], as the integer sweep):
//   1. columns: gather the window's columns from the object, column DFT, x ramp_y, inverse;
//   2. rows:    row DFT, x ramp_x, inverse (= S, kept for the probe gradient), x P, row DFT;
//   3. columns: the integer sweep's column pass (column DFT, amplitude-loss epilogue against
//               the counts, inverse column DFT);
//   4. rows:    inverse row DFT (= G), grad_P += G conj(S), G conj(P), then the row shift's
//               adjoint (row DFT, x conj(ramp_x), inverse);
//   5. columns: the column shift's adjoint (column DFT, x conj(ramp_y), inverse) and the
//               scatter-add into grad_O at the window.
// The ramps (with the inverse transforms' 1/n folded in) are tabulated per frame in FP64 by a
// prologue kernel and rounded once to FP32.  Frame sides are {2,3,5}-smooth in [16, 1024]:
// powers of two run the register-FFT kernels below, other sides the mixed-radix kernels of
// ptx_mixsubpix.cuh (each pass picks by the side it transforms), through the same layout.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "ptx_internal.h"
#include "ptx_passes.cuh"

namespace ptx {
namespace {

constexpr size_t kSpHeader = 256 + kLutBytes;       // error word + padding, count-decode table
constexpr size_t kSpTargetScratch = 4096ull << 20;  // upper bound on workspace frames
constexpr int kSpCols = 8;                          // columns per column-pass CTA
constexpr int kSpRowThreads = 128;

__device__ __forceinline__ void sp_corner(const double* __restrict__ pos, int f, long long& x0, long long& y0) {
  x0 = static_cast<long long>(floor(pos[2 * f] + 0.5));
  y0 = static_cast<long long>(floor(pos[2 * f + 1] + 0.5));
}

__device__ __forceinline__ bool sp_window_ok(long long x0, long long y0, int ph, int pw, int H, int W) {
  return x0 >= 0 && y0 >= 0 && x0 + pw <= W && y0 + ph <= H;
}

// Per frame f: rx[f][k] = exp(2 pi i dx kf / pw) / pw and ry[f][k] = exp(2 pi i dy kf / ph) / ph,
// kf the signed frequency of bin k (fftfreq * n), in FP64 rounded once to FP32.  Also flags
// (bit 0 of *err) every window that leaves the object.
__global__ void subpix_ramp_kernel(const double* __restrict__ pos, int nframes, int ph, int pw, int H, int W,
                                   float2* __restrict__ rx, float2* __restrict__ ry, unsigned* __restrict__ err) {
  const long long per = (long long)pw + ph;
  const long long total = per * nframes;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int f = static_cast<int>(i / per);
    const int k = static_cast<int>(i - (long long)f * per);
    const bool along_x = k < pw;
    const int n = along_x ? pw : ph;
    const int kk = along_x ? k : k - pw;
    const double p = pos[2 * f + (along_x ? 0 : 1)];
    const double d = p - floor(p + 0.5);
    const int kf = kk <= (n - 1) / 2 ? kk : kk - n;  // numpy fftfreq * n, odd n too
    double s, c;
    sincospi(2.0 * d * kf / n, &s, &c);
    const float2 v = make_float2(static_cast<float>(c / n), static_cast<float>(s / n));
    if (along_x) {
      rx[(size_t)f * pw + kk] = v;
    } else {
      ry[(size_t)f * ph + kk] = v;
    }
    if (k == 0) {
      long long x0, y0;
      sp_corner(pos, f, x0, y0);
      if (!sp_window_ok(x0, y0, ph, pw, H, W)) atomicOr(err, 1u);
    }
  }
}

// Column shift passes (frame side N along the columns).  A CTA owns kSpCols columns of one
// frame, threads column-fastest (thread (t, c) owns column c).  GATHER: the window's columns
// from the object (zero for a window outside it), column DFT, x ramp_y, inverse DFT, stored
// into the tiled frame.  Otherwise: the tiled frame's columns, column DFT, x conj(ramp_y),
// inverse DFT, added into grad_sample at the window (float2 atomics; windows outside the
// object are skipped).
template <int N, bool GATHER>
__global__ void __launch_bounds__(kSpCols * RegShape<N>::T) subpix_cols_kernel(
    const float2* __restrict__ sample, float2* __restrict__ grad_sample, int H, int W, int pw,
    const double* __restrict__ pos, int frame0, float2* __restrict__ scratch, const float2* __restrict__ ry_all,
    const float2* __restrict__ tw) {
  using S = RegShape<N>;
  constexpr int LP = col_line_pitch<N>();
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x;
  const int c = tid % kSpCols;
  const int t = tid / kSpCols;
  constexpr int kSubs = kTile / kSpCols;
  const int ct = blockIdx.x / kSubs;
  const int c0 = ct * kTile + (blockIdx.x - ct * kSubs) * kSpCols;
  const int kc = c0 + c;
  const bool col_ok = kc < pw;
  const int f = blockIdx.y;
  const int g = frame0 + f;
  const int tiles = num_tiles(pw);
  float2* tile = scratch + ((size_t)f * tiles + ct) * N * kTile + (c0 - ct * kTile);
  long long x0, y0;
  sp_corner(pos, g, x0, y0);
  const bool ok = sp_window_ok(x0, y0, N, pw, H, W);
  const float2* ry = ry_all + (size_t)g * N;
  float2* buf = sm + c * LP;
  float2 v[S::N1];
  if (GATHER) {
    const float2* col = sample + y0 * W + x0 + kc;
#pragma unroll
    for (int j = 0; j < S::N1; ++j) v[j] = (ok && col_ok) ? __ldg(&col[(size_t)(t + S::T * j) * W]) : make_float2(0.f, 0.f);
  } else {
#pragma unroll
    for (int j = 0; j < S::N1; ++j) v[j] = col_ok ? tile[(t + S::T * j) * kTile + c] : make_float2(0.f, 0.f);
  }
  reg_fft<N, false, true>(v, buf, t, tw);
#pragma unroll
  for (int m = 0; m < S::N1; ++m) {
    float2 w = __ldg(&ry[t + S::T * m]);
    if (!GATHER) w.y = -w.y;
    v[m] = cmul(v[m], w);
  }
  reg_fft<N, true, true>(v, buf, t, tw);
  if (GATHER) {
    if (col_ok) {
#pragma unroll
      for (int j = 0; j < S::N1; ++j) tile[(t + S::T * j) * kTile + c] = v[j];
    }
  } else if (ok && col_ok) {
    float2* col = grad_sample + y0 * W + x0 + kc;
#pragma unroll
    for (int j = 0; j < S::N1; ++j) atomicAdd(&col[(size_t)(t + S::T * j) * W], v[j]);
  }
}

// Row passes (frame side M along the rows).  A CTA owns `lines` rows (T threads each, one
// line per T lanes of a warp) of the frames [f0, f1); its probe rows, and in the adjoint the
// grad_P partials of its rows, sit in shared memory (each thread touches only its own
// elements, so no barrier guards them).
// FORWARD: row DFT, x ramp_x, inverse DFT (= S, stored into `sbuf` when STORE_S), x P, row
// DFT (stored in place when STORE_OUT).  Adjoint: inverse row DFT (= G),
// grad_P += G conj(S) (one float2 atomic per element per CTA at the end), G conj(P), row DFT,
// x conj(ramp_x), inverse DFT, stored in place.
template <int M, bool FORWARD, bool STORE_S, bool STORE_OUT>
__global__ void __launch_bounds__(kSpRowThreads) subpix_rows_kernel(
    float2* __restrict__ scratch, float2* __restrict__ sbuf, int ph, const float2* __restrict__ probe, int nframes,
    int frame0, int frames_per_cta, const float2* __restrict__ rx_all, float2* __restrict__ grad_probe,
    const float2* __restrict__ tw, int lines) {
  using S = RegShape<M>;
  constexpr int LP = row_line_pitch<M>();
  constexpr int kTiles = M / kTile;
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x;
  const int l = tid / S::T;  // blockDim.x = lines * T (whole warps: T and lines are powers of two)
  const int t = tid - l * S::T;
  const int r = blockIdx.x * lines + l;
  const bool row_ok = r < ph;
  float2* buf = sm + l * LP;
  float2* pbuf = sm + lines * LP + l * M;
  float2* acc = sm + lines * (LP + M) + l * M;  // adjoint only
  const int f0 = blockIdx.y * frames_per_cta;
  const int f1 = min(nframes, f0 + frames_per_cta);
#pragma unroll
  for (int m = 0; m < S::N1; ++m) {
    const int k = t + S::T * m;
    pbuf[k] = row_ok ? __ldg(&probe[(size_t)r * M + k]) : make_float2(0.f, 0.f);
    if (!FORWARD) acc[k] = make_float2(0.f, 0.f);
  }
  for (int f = f0; f < f1; ++f) {
    const float2* rx = rx_all + (size_t)(frame0 + f) * M;
    const size_t row0 = (size_t)f * kTiles * ph * kTile + (size_t)r * kTile;
    float2 v[S::N1];
#pragma unroll
    for (int j = 0; j < S::N1; ++j) {
      const int k = t + S::T * j;
      v[j] = row_ok ? scratch[row0 + (size_t)(k / kTile) * ph * kTile + (k % kTile)] : make_float2(0.f, 0.f);
    }
    if (FORWARD) {
      reg_fft<M, false, false>(v, buf, t, tw);
#pragma unroll
      for (int m = 0; m < S::N1; ++m) v[m] = cmul(v[m], __ldg(&rx[t + S::T * m]));
      reg_fft<M, true, false>(v, buf, t, tw);
      if (STORE_S && row_ok) {
#pragma unroll
        for (int j = 0; j < S::N1; ++j) {
          const int k = t + S::T * j;
          sbuf[row0 + (size_t)(k / kTile) * ph * kTile + (k % kTile)] = v[j];
        }
      }
      if constexpr (STORE_OUT) {
#pragma unroll
        for (int m = 0; m < S::N1; ++m) v[m] = cmul(v[m], pbuf[t + S::T * m]);
        reg_fft<M, false, false>(v, buf, t, tw);
      }
    } else {
      reg_fft<M, true, false>(v, buf, t, tw);
#pragma unroll
      for (int m = 0; m < S::N1; ++m) {
        const int k = t + S::T * m;
        const float2 s = row_ok ? sbuf[row0 + (size_t)(k / kTile) * ph * kTile + (k % kTile)] : make_float2(0.f, 0.f);
        acc[k] = cadd(acc[k], cmulc(v[m], s));
        v[m] = cmulc(v[m], pbuf[k]);
      }
      reg_fft<M, false, false>(v, buf, t, tw);
#pragma unroll
      for (int m = 0; m < S::N1; ++m) v[m] = cmulc(v[m], __ldg(&rx[t + S::T * m]));
      reg_fft<M, true, false>(v, buf, t, tw);
    }
    if (row_ok && (STORE_OUT || !FORWARD)) {
#pragma unroll
      for (int j = 0; j < S::N1; ++j) {
        const int k = t + S::T * j;
        scratch[row0 + (size_t)(k / kTile) * ph * kTile + (k % kTile)] = v[j];
      }
    }
  }
  if (!FORWARD && row_ok) {
#pragma unroll
    for (int m = 0; m < S::N1; ++m) {
      const int k = t + S::T * m;
      atomicAdd(&grad_probe[(size_t)r * M + k], acc[k]);
    }
  }
}

bool sp_side_ok(int n) { return n >= 16 && n <= 1024 && ((n & (n - 1)) == 0 || mix_subpix_ops(n) != nullptr); }

// a tiled frame [tile][row][16]
size_t sp_frame_bytes(int ph, int pw) { return (size_t)num_tiles(pw) * kTile * ph * sizeof(float2); }

size_t sp_ramp_bytes(int ph, int pw, int batch) {
  return align_up((size_t)std::max(batch, 1) * (ph + pw) * sizeof(float2), 256);
}

struct SpGeom {
  int H, W, ph, pw, batch, chunk;
  LinePlan row, col;
  const MixSubpixOps* mcol;  // mixed-radix column passes (ph not a power of two), else null
  const MixSubpixOps* mrow;  // mixed-radix row passes (pw not a power of two), else null
  unsigned* err;
  float* lut;
  float2* rx;
  float2* ry;
  float2* scratch;
  float2* sbuf;
};

int sp_check(const void* sample, int H, int W, const void* probe, int ph, int pw, const double* pos, int batch,
             void* ws, size_t ws_bytes, SpGeom* g) {
  if (!sample || !probe || (!pos && batch > 0) || !ws) return set_error(PTX_ERR_INVALID_ARGUMENT, "null pointer argument");
  if (H <= 0 || W <= 0 || batch < 0) return set_error(PTX_ERR_INVALID_ARGUMENT, "non-positive shape");
  if (!sp_side_ok(ph) || !sp_side_ok(pw)) {
    return set_error(PTX_ERR_UNSUPPORTED_SIZE,
                     "sub-pixel sweeps take probe sides that are 2^a 3^b 5^c in [16, 1024] (got %d x %d)", ph, pw);
  }
  if (ph > H || pw > W) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "probe (%d x %d) larger than sample (%d x %d)", ph, pw, H, W);
  }
  if (reinterpret_cast<uintptr_t>(ws) & 255) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "workspace must start on a 256-byte boundary");
  }
  const size_t frame = sp_frame_bytes(ph, pw);
  const size_t fixed = kSpHeader + sp_ramp_bytes(ph, pw, batch);
  if (ws_bytes < fixed + 2 * frame) {
    return set_error(PTX_ERR_WORKSPACE, "workspace of %zu bytes is smaller than the tables and one frame (%zu)",
                     ws_bytes, fixed + 2 * frame);
  }
  g->H = H; g->W = W; g->ph = ph; g->pw = pw; g->batch = batch;
  // frames per chunk: what the workspace holds, at most the batch and 65535 (a grid dimension)
  g->chunk = static_cast<int>(
      std::min<size_t>({(ws_bytes - fixed) / (2 * frame), (size_t)std::max(batch, 1), (size_t)65535}));
  if (int st = get_line_plan(pw, &g->row)) return st;
  if (int st = get_line_plan(ph, &g->col)) return st;
  g->mcol = (ph & (ph - 1)) ? mix_subpix_ops(ph) : nullptr;
  g->mrow = (pw & (pw - 1)) ? mix_subpix_ops(pw) : nullptr;
  if ((g->mcol && !g->col.mix_twt) || (g->mrow && !g->row.mix_twt)) {
    return set_error(PTX_ERR_UNSUPPORTED_SIZE, "no mixed-radix twiddle tables for %d x %d", ph, pw);
  }
  if (g->mcol) {
    if (int st = g->mcol->prepare()) return st;
  }
  if (g->mrow) {
    if (int st = g->mrow->prepare()) return st;
  }
  if (const MixOps* mo = (ph & (ph - 1)) ? mix_ops(ph) : nullptr) {  // the loss column pass
    if (int st = mo->prepare()) return st;
  }
  char* base = static_cast<char*>(ws);
  g->err = reinterpret_cast<unsigned*>(base);
  g->lut = reinterpret_cast<float*>(base + 256);
  g->rx = reinterpret_cast<float2*>(base + kSpHeader);
  g->ry = g->rx + (size_t)std::max(batch, 1) * pw;
  g->scratch = reinterpret_cast<float2*>(base + fixed);
  g->sbuf = g->scratch + (size_t)g->chunk * (frame / sizeof(float2));  // tiled frames, padded tiles included
  return PTX_OK;
}

void sp_launch_ramps(const SpGeom& g, const double* pos, cudaStream_t s) {
  if (g.batch == 0) return;
  const long long total = (long long)g.batch * (g.ph + g.pw);
  const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, (long long)sm_count() * 8));
  prof_begin(kMiscKernel, s);
  subpix_ramp_kernel<<<blocks, 256, 0, s>>>(pos, g.batch, g.ph, g.pw, g.H, g.W, g.rx, g.ry, g.err);
  prof_end(kMiscKernel, s);
}

MixSubpixArgs sp_mix_args(const SpGeom& g, const double* pos, int frame0, int nf) {
  MixSubpixArgs a{};
  a.H = g.H;
  a.W = g.W;
  a.ph = g.ph;
  a.pw = g.pw;
  a.pos = pos;
  a.frame0 = frame0;
  a.nframes = nf;
  a.scratch = g.scratch;
  a.sbuf = g.sbuf;
  a.rx = g.rx;
  a.ry = g.ry;
  a.twt_col = g.col.mix_twt;
  a.twi_col = g.col.mix_twi;
  a.twt_row = g.row.mix_twt;
  a.twi_row = g.row.mix_twi;
  return a;
}

template <bool GATHER>
int sp_launch_cols(const SpGeom& g, const float2* sample, float2* grad_sample, const double* pos, int frame0, int nf,
                   cudaStream_t s) {
  if (g.mcol) {
    MixSubpixArgs a = sp_mix_args(g, pos, frame0, nf);
    a.sample = sample;
    a.grad_sample = grad_sample;
    prof_begin(kSubpixCols, s);
    g.mcol->cols(GATHER, a, s);
    prof_end(kSubpixCols, s);
    return PTX_OK;
  }
  int st = PTX_OK;
  dispatch_pow2(g.ph, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    if constexpr (N >= 16) {
      constexpr int threads = kSpCols * RegShape<N>::T;
      const int smem = kSpCols * col_line_pitch<N>() * (int)sizeof(float2);
      st = ensure_smem((const void*)subpix_cols_kernel<N, GATHER>, smem);
      if (st) return;
      dim3 grid(num_tiles(g.pw) * (kTile / kSpCols), nf);
      prof_begin(kSubpixCols, s);
      subpix_cols_kernel<N, GATHER><<<grid, threads, smem, s>>>(sample, grad_sample, g.H, g.W, g.pw, pos, frame0,
                                                                g.scratch, g.ry, g.col.tw);
      prof_end(kSubpixCols, s);
    }
  });
  return st;
}

template <bool FORWARD, bool STORE_S, bool STORE_OUT>
int sp_launch_rows(const SpGeom& g, const float2* probe, float2* grad_probe, int frame0, int nf, cudaStream_t s,
                   const double* pos) {
  if (g.mrow) {
    MixSubpixArgs a = sp_mix_args(g, pos, frame0, nf);
    a.probe = probe;
    a.grad_probe = grad_probe;
    const int variant = !FORWARD ? kMixSubpixAdjoint
                        : (STORE_S && STORE_OUT) ? kMixSubpixSweepForward
                        : STORE_S ? kMixSubpixShiftOnly : kMixSubpixForwardOnly;
    prof_begin(kSubpixRows, s);
    g.mrow->rows(variant, a, s);
    prof_end(kSubpixRows, s);
    return PTX_OK;
  }
  int st = PTX_OK;
  dispatch_pow2(g.pw, [&](auto NT) {
    constexpr int M = decltype(NT)::value;
    if constexpr (M >= 16) {
      const int lines = std::min(kSpRowThreads / RegShape<M>::T, g.ph);
      const int rowgroups = (g.ph + lines - 1) / lines;
      const int smem = lines * (row_line_pitch<M>() + (FORWARD ? 1 : 2) * M) * (int)sizeof(float2);
      auto kern = subpix_rows_kernel<M, FORWARD, STORE_S, STORE_OUT>;
      st = ensure_smem((const void*)kern, smem);
      if (st) return;
      // about 8 CTAs per SM in all; each CTA keeps its probe rows (and grad_P partials) over its frames
      const long long target = (long long)sm_count() * 8;
      int fpc = static_cast<int>(std::max<long long>(1, ((long long)rowgroups * nf) / target));
      fpc = std::min(fpc, std::max(nf, 1));
      dim3 grid(rowgroups, (nf + fpc - 1) / fpc);
      prof_begin(kSubpixRows, s);
      kern<<<grid, lines * RegShape<M>::T, smem, s>>>(g.scratch, g.sbuf, g.ph, probe, nf, frame0, fpc, g.rx,
                                                      grad_probe, g.row.tw, lines);
      prof_end(kSubpixRows, s);
    }
  });
  return st;
}

int sp_launch_cols_sweep(const SpGeom& g, int frame0, int nf, const uint16_t* measured, float grad_scale,
                         double inv_numel, double* loss, cudaStream_t s) {
  if (const MixOps* mo = (g.ph & (g.ph - 1)) ? mix_ops(g.ph) : nullptr) {
    MixColsArgs a{g.scratch, g.ph, g.pw, frame0, nf, g.col.mix_twt, g.col.mix_twi, measured, g.lut,
                  grad_scale, inv_numel, loss, nullptr, nullptr, nullptr};
    prof_begin(kBaseCols, s);
    mo->cols(kMixColSweep, a, s);
    prof_end(kBaseCols, s);
    return PTX_OK;
  }
  int st = PTX_OK;
  dispatch_pow2(g.ph, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    if constexpr (N >= 16) {
      // the full-tile variant needs whole 16-column tiles
      auto kern = (g.pw % kTile == 0) ? cols_sweep_pair<N, false, true, true, true> : cols_sweep_pair<N, false, true, true>;
      st = ensure_smem((const void*)kern, ColPairCfg<N>::kSmemBytes);
      if (st) return;
      dim3 grid(num_tiles(g.pw), nf);
      prof_begin(kBaseCols, s);
      kern<<<grid, ColPairCfg<N>::kThreads, ColPairCfg<N>::kSmemBytes, s>>>(g.scratch, g.pw, frame0, g.col.tw,
                                                                            measured, g.lut, 1.0f, grad_scale,
                                                                            inv_numel, loss);
      prof_end(kBaseCols, s);
    }
  });
  return st;
}

}  // namespace
}  // namespace ptx

using namespace ptx;

extern "C" {

size_t ptx_base_subpix_workspace_bytes(int probe_h, int probe_w, int batch) {
  if (!sp_side_ok(probe_h) || !sp_side_ok(probe_w) || batch < 0) return 0;
  const size_t frame = sp_frame_bytes(probe_h, probe_w);
  size_t frames = std::max<size_t>(1, kSpTargetScratch / (2 * frame));
  frames = std::min<size_t>(frames, (size_t)std::max(batch, 1));
  return kSpHeader + sp_ramp_bytes(probe_h, probe_w, batch) + frames * 2 * frame;
}

int ptx_base_subpix_sweep(const float* sample, int sample_h, int sample_w, const float* probe, int probe_h,
                          int probe_w, const double* positions_xy, int batch, const uint16_t* measured, float scale,
                          double* loss, float* grad_sample, float* grad_probe, void* workspace,
                          size_t workspace_bytes, void* stream) {
  SpGeom g;
  if (int st = sp_check(sample, sample_h, sample_w, probe, probe_h, probe_w, positions_xy, batch, workspace,
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
  const float2* S = reinterpret_cast<const float2*>(sample);
  const float2* P = reinterpret_cast<const float2*>(probe);
  const double numel = (double)batch * probe_h * probe_w;
  const float grad_scale = static_cast<float>(2.0 / std::max(numel, 1.0));
  {
    const size_t ns = (size_t)sample_h * sample_w, np = (size_t)probe_h * probe_w;
    prof_begin(kMiscKernel, s);
    sweep_prologue_kernel<<<prologue_blocks(ns, sm_count()), 256, 0, s>>>(GS, ns, GP, np, loss, g.err, g.lut, scale);
    prof_end(kMiscKernel, s);
  }
  sp_launch_ramps(g, positions_xy, s);
  for (int b0 = 0; b0 < batch; b0 += g.chunk) {
    const int nf = std::min(g.chunk, batch - b0);
    int st = sp_launch_cols<true>(g, S, nullptr, positions_xy, b0, nf, s);
    if (!st) st = sp_launch_rows<true, true, true>(g, P, nullptr, b0, nf, s, positions_xy);
    if (!st) st = sp_launch_cols_sweep(g, b0, nf, measured, grad_scale, 1.0 / std::max(numel, 1.0), loss, s);
    if (!st) st = sp_launch_rows<false, false, false>(g, P, GP, b0, nf, s, positions_xy);
    if (!st) st = sp_launch_cols<false>(g, nullptr, GS, positions_xy, b0, nf, s);
    if (st) return st;
  }
  return cuda_status(cudaGetLastError(), "ptx_base_subpix_sweep launch");
}

int ptx_base_subpix_forward(const float* sample, int sample_h, int sample_w, const float* probe, int probe_h,
                            int probe_w, const double* positions_xy, int batch, float* far_field, float* amplitude,
                            void* workspace, size_t workspace_bytes, void* stream) {
  SpGeom g;
  if (int st = sp_check(sample, sample_h, sample_w, probe, probe_h, probe_w, positions_xy, batch, workspace,
                        workspace_bytes, &g)) {
    return st;
  }
  if (!amplitude && batch > 0) return set_error(PTX_ERR_INVALID_ARGUMENT, "amplitude is null");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaMemsetAsync(g.err, 0, sizeof(unsigned), s);
  sp_launch_ramps(g, positions_xy, s);
  const float2* S = reinterpret_cast<const float2*>(sample);
  const float2* P = reinterpret_cast<const float2*>(probe);
  for (int b0 = 0; b0 < batch; b0 += g.chunk) {
    const int nf = std::min(g.chunk, batch - b0);
    int st = sp_launch_cols<true>(g, S, nullptr, positions_xy, b0, nf, s);
    if (!st) st = sp_launch_rows<true, false, true>(g, P, nullptr, b0, nf, s, positions_xy);
    if (!st) {
      st = base_cols_pass(true, g.scratch, probe_h, probe_w, b0, nf, reinterpret_cast<float2*>(far_field), amplitude,
                          nullptr, s);
    }
    if (st) return st;
  }
  return cuda_status(cudaGetLastError(), "ptx_base_subpix_forward launch");
}

int ptx_base_subpix_backward(const float* grad_output, const float* far_field, const float* sample, int sample_h,
                             int sample_w, const float* probe, int probe_h, int probe_w, const double* positions_xy,
                             int batch, float* grad_sample, float* grad_probe, void* workspace,
                             size_t workspace_bytes, void* stream) {
  SpGeom g;
  if (int st = sp_check(sample, sample_h, sample_w, probe, probe_h, probe_w, positions_xy, batch, workspace,
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
  sp_launch_ramps(g, positions_xy, s);
  const float2* S = reinterpret_cast<const float2*>(sample);
  const float2* P = reinterpret_cast<const float2*>(probe);
  for (int b0 = 0; b0 < batch; b0 += g.chunk) {
    const int nf = std::min(g.chunk, batch - b0);
    // the shifted patches S (for the probe gradient), then g F/|F| through the inverse column DFT
    int st = sp_launch_cols<true>(g, S, nullptr, positions_xy, b0, nf, s);
    if (!st) st = sp_launch_rows<true, true, false>(g, P, nullptr, b0, nf, s, positions_xy);
    if (!st) {
      st = base_cols_pass(false, g.scratch, probe_h, probe_w, b0, nf,
                          const_cast<float2*>(reinterpret_cast<const float2*>(far_field)), nullptr, grad_output, s);
    }
    if (!st) st = sp_launch_rows<false, false, false>(g, P, GP, b0, nf, s, positions_xy);
    if (!st) st = sp_launch_cols<false>(g, nullptr, GS, positions_xy, b0, nf, s);
    if (st) return st;
  }
  return cuda_status(cudaGetLastError(), "ptx_base_subpix_backward launch");
}

}  // extern "C"
