// Fourier ptychography (FPM): forward, adjoint and the fused forward+loss+adjoint sweep.
//
// Math (python/ptychoX/fpm/ops.py:180-183 forward, :209-221 adjoint, :113-124 windows):
//   S = fft2(O);  sub_b[r,c] = S[(ly+r+H/2) % H, (lx+c+W/2) % W]
//   image_b = ifft2(fftshift(sub_b * pupil)),  A_b = |image_b|
//   Gl_b = ifftshift(fft2(g_b * image/max(|image|, eps)) / (h w))
//   grad_pupil = sum_b Gl_b conj(sub_b);  grad_S[window_b] += Gl_b conj(pupil)
//   grad_O = ifft2(grad_S) * H W
//
// Per frame (one LED) the same three-pass structure as the conventional sweep:
//   row pass   gather the window of S (with wrap), x pupil, fftshift placement, inverse
//              row DFT                                                         -> scratch
//   col pass   inverse column DFT, image = X/(h w), |image|, residual vs sqrt(scale I),
//              FP64 loss, g image/|image|, forward column DFT                  -> scratch
//   row pass   forward row DFT, /(h w), ifftshift placement, grad_S += Gl conj(pupil)
//              (float2 atomics, with wrap), grad_pupil += Gl conj(S) in registers
// S = fft2(O) before the frames and grad_O = n ifft2(grad_S) after them use the generic
// 2-D passes.  When all four sides are powers of two (4..1024) the kernels below run (every
// modulo a mask); any other {2,3,5}-smooth sides take the mixed-radix kernels of
// ptx_mixfpm.cuh through the same workspace layout.
#include <cuda_runtime.h>

#include <algorithm>

#include "ptx_internal.h"
#include "ptx_passes.cuh"

namespace ptx {
namespace {

constexpr size_t kHdr = 256 + kLutBytes;  // padding, count-decode table
enum FpmMode { kFpmSweep = 0, kFpmForward = 1, kFpmBackward = 2 };

__device__ __forceinline__ int wrap2(long long v, int n) { return static_cast<int>(v & (long long)(n - 1)); }

// Shared memory of the FPM row passes, per line: the exchange / landing line (BP) and
// two rows of N values (the gathered spectrum window row and the pupil row); per CTA the
// twiddle table laid out by thread.
template <int NW>
struct FpmRowCfg {
  static constexpr int BP = RowPass<NW>::LP > NW ? RowPass<NW>::LP : NW;
  static int smem(int lines) { return (lines * (BP + 2 * NW) + NW) * (int)sizeof(float2); }
};

// Forward row pass: gather the sub-aperture window of the spectrum (wrapping), multiply by
// the pupil, inverse row DFT, store tiled.  Work units are (row group, frame) pairs in
// row-group-major order over one wave of resident CTAs (CTA b takes the contiguous units
// [u0, u1)); the pupil rows of the current row group and the twiddle table sit in shared
// memory, and the next unit's window row is requested by cp.async (evict-last in L2: the
// spectrum is re-read by every LED) as soon as this unit's transform has released the
// line buffer, so it lands while this unit stores.
template <int NW>
__global__ void __launch_bounds__(128, 3) fpm_rows_forward(
    const float2* __restrict__ spec, int oh, int ow, const float2* __restrict__ pupil, int lh,
    const int64_t* __restrict__ led, int nframes, int rowgroups, float2* __restrict__ scratch,
    const float2* __restrict__ tw, int lines) {
  pdl_wait();
  using S = RegShape<NW>;
  using Cfg = FpmRowCfg<NW>;
  constexpr int kTiles = (NW + kTile - 1) / kTile;
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
  float2* pbuf = sm + lines * Cfg::BP + l * NW;
  float2* tws = sm + lines * (Cfg::BP + 2 * NW);
  load_twiddles_by_thread<NW>(tws, tw);
  __syncthreads();
  const uint64_t pol_last = policy_evict_last();
  // window row of G row i (= fftshift(sub * pupil)) of `frame` into buf[t + T j]
  auto request = [&](int i, int frame) -> bool {
    if (i >= lh) return false;
    const long long lx = led[2 * frame], ly = led[2 * frame + 1];
    const int r = (i + lh / 2) & (lh - 1);
    const float2* srow = spec + (size_t)wrap2(ly + r + oh / 2, oh) * ow;
#pragma unroll
    for (int j = 0; j < S::N1; ++j) {
      const int c = (t + S::T * j + NW / 2) & (NW - 1);
      cp_async8_hint(buf + t + S::T * j, srow + wrap2(lx + c + ow / 2, ow), pol_last);
    }
    cp_async_commit();
    return true;
  };
  int i = g * lines + l;
  bool have = request(i, f);
  bool new_group = true;
  for (long long u = u0; u < u1; ++u) {
    const bool row_ok = i < lh;
    if (new_group && row_ok) {
      const int r = (i + lh / 2) & (lh - 1);
#pragma unroll
      for (int j = 0; j < S::N1; ++j) {
        const int c = (t + S::T * j + NW / 2) & (NW - 1);
        pbuf[t + S::T * j] = __ldg(&pupil[(size_t)r * NW + c]);
      }
    }
    new_group = false;
    cp_async_wait_all();  // own copies only: thread t copied exactly the elements it reads
    float2 v[S::N1];
#pragma unroll
    for (int j = 0; j < S::N1; ++j) {
      v[j] = have ? cmul(buf[t + S::T * j], pbuf[t + S::T * j]) : make_float2(0.f, 0.f);
    }
    __syncwarp();
    reg_fft<NW, true, false, true>(v, buf, t, tws);
    const bool more = u + 1 < u1;
    int gn = g, fn = f + 1;
    if (fn == nframes) {
      gn = g + 1;
      fn = 0;
    }
    const int in = gn * lines + l;
    const bool have_next = more ? request(in, fn) : false;
    if (row_ok) {
      float2* base = scratch + (size_t)f * kTiles * lh * kTile + (size_t)i * kTile;
#pragma unroll
      for (int m = 0; m < S::N1; ++m) {
        const int kc = t + S::T * m;
        base[(size_t)(kc / kTile) * lh * kTile + (kc % kTile)] = v[m];
      }
    }
    if (gn != g) new_group = true;
    g = gn;
    f = fn;
    i = in;
    have = have_next;
  }
}

template <int MODE, int NH>
__global__ void __launch_bounds__(256, 2) fpm_cols(
    float2* __restrict__ scratch, int lw, int frame0, const float2* __restrict__ tw,
    const uint16_t* __restrict__ measured, const float* __restrict__ lut, float norm, float grad_scale,
    double inv_numel,
    double* __restrict__ loss, float2* __restrict__ image_out, float* __restrict__ amplitude,
    const float* __restrict__ grad_output) {
  using S = RegShape<NH>;
  using CP = ColPass<NH>;
  extern __shared__ float2 sm[];
  uint16_t* meas_s = reinterpret_cast<uint16_t*>(reinterpret_cast<char*>(sm) + CP::kMeasOffsetBytes);
  const int tid = threadIdx.x;
  const int c = tid % kColsPerCta;
  const int t = tid / kColsPerCta;
  constexpr int kSubs = kTile / kColsPerCta;
  const int ct = blockIdx.x / kSubs;
  const int c0 = ct * kTile + (blockIdx.x - ct * kSubs) * kColsPerCta;
  const int f = blockIdx.y;
  const int kc = c0 + c;
  const bool col_ok = kc < lw;
  const int tiles = num_tiles(lw);
  float2* tile = scratch + ((size_t)f * tiles + ct) * NH * kTile + (c0 - ct * kTile);
  const size_t g = (size_t)frame0 + f;
  float2* buf = sm + c * CP::LP;
  float2 v[S::N1];

  if (MODE == kFpmSweep) {
    const bool fast = (lw % (2 * kColsPerCta) == 0) && ((reinterpret_cast<uintptr_t>(measured) & 15) == 0);
    if (fast) {
      for (int kr = tid; kr < NH; kr += blockDim.x) cp_async16(meas_s + kr * kColsPerCta, measured + (g * NH + kr) * lw + c0);
      cp_async_commit();
    } else {
      for (int q = tid; q < NH * kColsPerCta; q += blockDim.x) {
        const int kr = q / kColsPerCta, cc = q - kr * kColsPerCta;
        meas_s[q] = (c0 + cc < lw) ? measured[(g * NH + kr) * lw + c0 + cc] : 0;
      }
    }
  }
  if (MODE != kFpmBackward) {
#pragma unroll
    for (int j = 0; j < S::N1; ++j) v[j] = col_ok ? tile[(t + S::T * j) * kTile + c] : make_float2(0.f, 0.f);
    reg_fft<NH, true, true>(v, buf, t, tw);
  }
  if (MODE == kFpmSweep) {
    cp_async_wait_all();
    __syncthreads();
    float part = 0.f;  // this thread's squared residuals; summed in FP64 across the grid
#pragma unroll
    for (int m = 0; m < S::N1; ++m) {
      const int kr = t + S::T * m;
      const float2 im = cscale(v[m], norm);
      float2 out = make_float2(0.f, 0.f);
      if (col_ok) {
        const float y = __ldg(&lut[meas_s[kr * kColsPerCta + c]]);
        float a, inv;
        abs_and_inv(im, kEpsF32, a, inv);
        const float rr = a - y;
        part = fmaf(rr, rr, part);
        out = cscale(im, grad_scale * rr * inv);
      }
      v[m] = out;
    }
    block_add_double(static_cast<double>(part), inv_numel, loss);
  } else if (MODE == kFpmForward) {
    if (col_ok) {
#pragma unroll
      for (int m = 0; m < S::N1; ++m) {
        const size_t idx = (g * NH + t + S::T * m) * lw + kc;
        const float2 im = cscale(v[m], norm);
        if (image_out) image_out[idx] = im;
        amplitude[idx] = cabsf(im);
      }
    }
    return;
  } else {
#pragma unroll
    for (int m = 0; m < S::N1; ++m) {
      float2 out = make_float2(0.f, 0.f);
      if (col_ok) {
        const size_t idx = (g * NH + t + S::T * m) * lw + kc;
        const float2 im = image_out[idx];
        out = cscale(im, grad_output[idx] / fmaxf(cabsf(im), kEpsF32));
      }
      v[m] = out;
    }
  }
  reg_fft<NH, false, true>(v, buf, t, tw);
  if (col_ok) {
#pragma unroll
    for (int m = 0; m < S::N1; ++m) tile[(t + S::T * m) * kTile + c] = v[m];
  }
}

template <int NW>
__global__ void __launch_bounds__(128, 3) fpm_rows_adjoint(
    const float2* __restrict__ scratch, const float2* __restrict__ spec, int oh, int ow,
    const float2* __restrict__ pupil, int lh, const int64_t* __restrict__ led, int nframes, int rowgroups,
    float norm, float2* __restrict__ grad_spec, float2* __restrict__ grad_pupil, const float2* __restrict__ tw,
    int lines) {
  pdl_wait();
  using S = RegShape<NW>;
  constexpr int kTiles = (NW + kTile - 1) / kTile;
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
  using Cfg = FpmRowCfg<NW>;
  float2* buf = sm + l * Cfg::BP;
  float2* sbuf = sm + lines * Cfg::BP + l * NW;  // prefetched window row of S
  float2* pbuf = sm + lines * (Cfg::BP + NW) + l * NW;  // pupil row of the current row group
  float2* tws = sm + lines * (Cfg::BP + 2 * NW);
  load_twiddles_by_thread<NW>(tws, tw);
  __syncthreads();
  const uint64_t pol_last = policy_evict_last();
  bool new_group = true;
  float2 acc[S::N1];
#pragma unroll
  for (int m = 0; m < S::N1; ++m) acc[m] = make_float2(0.f, 0.f);
  for (long long u = u0; u < u1; ++u) {
    const int i = g * lines + l;
    const bool row_ok = i < lh;
    const int r = (i + lh / 2) & (lh - 1);
    const long long lx = led[2 * f], ly = led[2 * f + 1];
    const size_t srow = (size_t)wrap2(ly + r + oh / 2, oh) * ow;
    if (row_ok) {
#pragma unroll
      for (int m = 0; m < S::N1; ++m) {
        const int jj = t + S::T * m;
        const int c = (jj + NW / 2) & (NW - 1);
        cp_async8_hint(sbuf + jj, spec + srow + wrap2(lx + c + ow / 2, ow), pol_last);
      }
      cp_async_commit();
      if (new_group) {
#pragma unroll
        for (int m = 0; m < S::N1; ++m) {
          const int c = (t + S::T * m + NW / 2) & (NW - 1);
          pbuf[t + S::T * m] = __ldg(&pupil[(size_t)r * NW + c]);
        }
      }
    }
    new_group = false;
    float2 v[S::N1];
    if (row_ok) {
      const float2* base = scratch + (size_t)f * kTiles * lh * kTile + (size_t)i * kTile;
#pragma unroll
      for (int j = 0; j < S::N1; ++j) {
        const int cc = t + S::T * j;
        v[j] = base[(size_t)(cc / kTile) * lh * kTile + (cc % kTile)];
      }
    } else {
#pragma unroll
      for (int j = 0; j < S::N1; ++j) v[j] = make_float2(0.f, 0.f);
    }
    reg_fft<NW, false, false, true>(v, buf, t, tws);
    if (row_ok) {
      cp_async_wait_all();
#pragma unroll
      for (int m = 0; m < S::N1; ++m) {
        const int jj = t + S::T * m;
        const int c = (jj + NW / 2) & (NW - 1);
        const float2 gl = cscale(v[m], norm);
        atomicAdd(&grad_spec[srow + wrap2(lx + c + ow / 2, ow)], cmulc(gl, pbuf[jj]));
        acc[m] = cadd(acc[m], cmulc(gl, sbuf[jj]));
      }
    }
    int gn = g, fn = f + 1;
    if (fn == nframes) {
      gn = g + 1;
      fn = 0;
    }
    if (u + 1 == u1 || gn != g) {
      new_group = true;
      // leaving this row group: fold its pupil-gradient partial sums into grad_pupil
      if (row_ok) {
#pragma unroll
        for (int m = 0; m < S::N1; ++m) {
          const int c = (t + S::T * m + NW / 2) & (NW - 1);
          atomicAdd(&grad_pupil[(size_t)r * NW + c], acc[m]);
          acc[m] = make_float2(0.f, 0.f);
        }
      }
    }
    g = gn;
    f = fn;
  }
}

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------

struct FpmGeom {
  int oh, ow, lh, lw, batch;
  LinePlan p_ow, p_oh, p_lw, p_lh;
  bool generic;  // a side is not a power of two: the mixed-radix kernels
  const MixFpmOps *m_ow, *m_oh, *m_lw, *m_lh;
  size_t spec_bytes, tmp_bytes, frame_bytes;
  int chunk;
  float2* spec;   // workspace spectrum (sweep)
  float2* gspec;  // gradient w.r.t. the spectrum
  float2* tmp;    // tiled temporary of the 2-D passes
  float2* frames;
  float* lut;     // count-decode table (sweep)
};

size_t fpm_fixed_bytes(int oh, int ow) {
  const size_t spec = (size_t)oh * ow * sizeof(float2);
  const size_t tmp = (size_t)num_tiles(ow) * kTile * oh * sizeof(float2);
  return kHdr + 2 * spec + tmp;
}

int fpm_check(const void* object, int oh, int ow, const void* pupil, int lh, int lw, const int64_t* led, int batch,
              void* ws, size_t ws_bytes, FpmGeom* g) {
  if (!object || !pupil || (!led && batch > 0) || !ws) return set_error(PTX_ERR_INVALID_ARGUMENT, "null pointer argument");
  if (batch < 0) return set_error(PTX_ERR_INVALID_ARGUMENT, "negative batch");
  if (reinterpret_cast<uintptr_t>(ws) & 255) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "workspace must start on a 256-byte boundary");
  }
  g->generic = !(is_pow2_len(oh) && is_pow2_len(ow) && is_pow2_len(lh) && is_pow2_len(lw));
  for (int n : {oh, ow, lh, lw}) {
    if (!(g->generic ? mix_fpm_ops(n) != nullptr : is_pow2_len(n))) {
      return set_error(PTX_ERR_UNSUPPORTED_SIZE, "FPM sides must be 2^a 3^b 5^c in [4, 1024] (got %d)", n);
    }
  }
  if (lh > oh || lw > ow) return set_error(PTX_ERR_INVALID_ARGUMENT, "pupil larger than the object spectrum");
  g->oh = oh; g->ow = ow; g->lh = lh; g->lw = lw; g->batch = batch;
  if (int st = get_line_plan(ow, &g->p_ow)) return st;
  if (int st = get_line_plan(oh, &g->p_oh)) return st;
  if (int st = get_line_plan(lw, &g->p_lw)) return st;
  if (int st = get_line_plan(lh, &g->p_lh)) return st;
  g->spec_bytes = (size_t)oh * ow * sizeof(float2);
  g->tmp_bytes = (size_t)num_tiles(ow) * kTile * oh * sizeof(float2);
  g->frame_bytes = (size_t)num_tiles(lw) * kTile * lh * sizeof(float2);
  const size_t fixed = fpm_fixed_bytes(oh, ow);
  if (ws_bytes < fixed + g->frame_bytes) {
    return set_error(PTX_ERR_WORKSPACE, "workspace of %zu bytes is smaller than the %zu bytes needed", ws_bytes,
                     fixed + g->frame_bytes);
  }
  // frames per chunk: what the workspace holds, at most the batch and 65535 (the column
  // passes put the frame in gridDim.y)
  g->chunk = static_cast<int>(
      std::min<size_t>({(ws_bytes - fixed) / g->frame_bytes, (size_t)std::max(batch, 1), (size_t)65535}));
  g->lut = reinterpret_cast<float*>(static_cast<char*>(ws) + 256);
  char* p = static_cast<char*>(ws) + kHdr;
  g->spec = reinterpret_cast<float2*>(p);
  g->gspec = reinterpret_cast<float2*>(p + g->spec_bytes);
  g->tmp = reinterpret_cast<float2*>(p + 2 * g->spec_bytes);
  g->frames = reinterpret_cast<float2*>(p + 2 * g->spec_bytes + g->tmp_bytes);
  int st = PTX_OK;
  if (g->generic) {
    g->m_ow = mix_fpm_ops(ow);
    g->m_oh = mix_fpm_ops(oh);
    g->m_lw = mix_fpm_ops(lw);
    g->m_lh = mix_fpm_ops(lh);
    for (const LinePlan* p : {&g->p_ow, &g->p_oh, &g->p_lw, &g->p_lh}) {
      if (!p->mix_twt) return set_error(PTX_ERR_UNSUPPORTED_SIZE, "no mixed-radix twiddle tables for length %d", p->n);
    }
    for (const MixFpmOps* o : {g->m_ow, g->m_oh, g->m_lw, g->m_lh}) {
      if (!st) st = o->prepare();
    }
    return st;
  }
  g->m_ow = g->m_oh = g->m_lw = g->m_lh = nullptr;
  dispatch_pow2(ow, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    if (!st) st = ensure_smem((const void*)fft2_rows_kernel<N, false>, RowPass<N>::smem(RowPass<N>::lines(256, oh)));
    if (!st) st = ensure_smem((const void*)fft2_rows_kernel<N, true>, RowPass<N>::smem(RowPass<N>::lines(256, oh)));
  });
  dispatch_pow2(oh, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    const int sm = kColsPerCta * ColPass<N>::LP * (int)sizeof(float2);
    if (!st) st = ensure_smem((const void*)fft2_cols_kernel<N, false>, sm);
    if (!st) st = ensure_smem((const void*)fft2_cols_kernel<N, true>, sm);
  });
  dispatch_pow2(lw, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    if (!st) st = ensure_smem((const void*)fpm_rows_forward<N>, FpmRowCfg<N>::smem(RowPass<N>::lines(128, lh)));
    if (!st) st = ensure_smem((const void*)fpm_rows_adjoint<N>, FpmRowCfg<N>::smem(RowPass<N>::lines(128, lh)));
  });
  dispatch_pow2(lh, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    if (!st) st = ensure_smem((const void*)cols_sweep_pair<N, true, false>, ColPairCfg<N>::kSmemBytes);
    if (!st) st = ensure_smem((const void*)cols_sweep_pair<N, true, false, false, true>, ColPairCfg<N>::kSmemBytes);
    if (!st) st = ensure_smem((const void*)fpm_cols<kFpmForward, N>, ColPass<N>::kSmemBytes);
    if (!st) st = ensure_smem((const void*)fpm_cols<kFpmBackward, N>, ColPass<N>::kSmemBytes);
  });
  return st;
}

// out = DFT2 (INV=false) or unnormalised inverse DFT2 (INV=true) of the H x W image in, via tmp.
template <bool INV>
void launch_fft2(const FpmGeom& g, const float2* in, int H, int W, float2* out, float scale, float2* tmp,
                 const LinePlan& prow, const LinePlan& pcol, cudaStream_t s) {
  if (g.generic) {
    prof_begin(kFft2Rows, s);
    g.m_ow->fft2_rows(INV, in, H, tmp, prow.mix_twt, s);
    prof_end(kFft2Rows, s);
    prof_begin(kFft2Cols, s);
    g.m_oh->fft2_cols(INV, tmp, W, out, scale, pcol.mix_twt, s);
    prof_end(kFft2Cols, s);
    return;
  }
  prof_begin(kFft2Rows, s);
  dispatch_pow2(W, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    // 128-thread CTAs: the 1024 rows of a 1024^2 spectrum make 256 CTAs, every SM busy in
    // the single wave (10.8 against 11.4 us per pass with 256-thread CTAs on 128 SMs)
    const int lines = RowPass<N>::lines(128, H);
    launch_pdl(fft2_rows_kernel<N, INV>, (H + lines - 1) / lines, lines * RowPass<N>::T, RowPass<N>::smem(lines), s,
        in, H, tmp, prow.tw, lines);
  });
  prof_end(kFft2Rows, s);
  prof_begin(kFft2Cols, s);
  dispatch_pow2(H, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    const int sm = kColsPerCta * ColPass<N>::LP * (int)sizeof(float2);
    launch_pdl(fft2_cols_kernel<N, INV>, num_tiles(W) * (kTile / kColsPerCta), ColPass<N>::kThreads, sm, s,
        tmp, W, out, scale, pcol.tw);
  });
  prof_end(kFft2Cols, s);
}

void launch_rows_forward(const FpmGeom& g, const float2* spec, const float2* pupil, const int64_t* led, int nf,
                         cudaStream_t s) {
  prof_begin(kFpmRowsForward, s);
  if (g.generic) {
    MixFpmRowsArgs a{spec, g.oh, g.ow, pupil, g.lh, led, nf, g.frames, g.p_lw.mix_twt, g.p_lw.mix_twi, 0.f,
                     nullptr, nullptr};
    g.m_lw->rows_forward(a, s);
    prof_end(kFpmRowsForward, s);
    return;
  }
  dispatch_pow2(g.lw, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    const int lines = RowPass<N>::lines(128, g.lh);
    const int rowgroups = (g.lh + lines - 1) / lines;
    const int threads = lines * RowPass<N>::T, smem = FpmRowCfg<N>::smem(lines);
    const int grid = persistent_grid((const void*)fpm_rows_forward<N>, threads, smem, (long long)rowgroups * nf);
    launch_pdl(fpm_rows_forward<N>, grid, threads, smem, s, spec, g.oh, g.ow, pupil, g.lh, led, nf, rowgroups, g.frames,
                                                    g.p_lw.tw, lines);
  });
  prof_end(kFpmRowsForward, s);
}

template <int MODE>
void launch_cols(const FpmGeom& g, int frame0, int nf, const uint16_t* measured, float grad_scale,
                 double inv_numel, double* loss, float2* image, float* amplitude, const float* grad_output,
                 cudaStream_t s) {
  const float norm = 1.0f / static_cast<float>((double)g.lh * g.lw);
  prof_begin(kFpmCols, s);
  if (g.generic) {
    MixFpmColsArgs a{g.frames, g.lw, frame0, nf, g.p_lh.mix_twt, g.p_lh.mix_twi, measured, g.lut, norm, grad_scale,
                     inv_numel, loss, image, amplitude, grad_output};
    g.m_lh->cols(MODE == kFpmSweep ? kMixColSweep : MODE == kFpmForward ? kMixColForward : kMixColBackward, a, s);
    prof_end(kFpmCols, s);
    return;
  }
  dispatch_pow2(g.lh, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    if constexpr (MODE == kFpmSweep) {
      // inverse column DFT, 1/(h w), amplitude-loss epilogue, forward column DFT
      dim3 grid(num_tiles(g.lw), nf);
      if (g.lw % kTile == 0) {
        launch_pdl(cols_sweep_pair<N, true, false, false, true>, grid, ColPairCfg<N>::kThreads, ColPairCfg<N>::kSmemBytes, s,
            g.frames, g.lw, frame0, g.p_lh.tw, measured, g.lut, norm, grad_scale, inv_numel, loss);
      } else {
        launch_pdl(cols_sweep_pair<N, true, false>, grid, ColPairCfg<N>::kThreads, ColPairCfg<N>::kSmemBytes, s,
            g.frames, g.lw, frame0, g.p_lh.tw, measured, g.lut, norm, grad_scale, inv_numel, loss);
      }
      return;
    }
    dim3 grid(num_tiles(g.lw) * (kTile / kColsPerCta), nf);
    fpm_cols<MODE, N><<<grid, ColPass<N>::kThreads, ColPass<N>::kSmemBytes, s>>>(
        g.frames, g.lw, frame0, g.p_lh.tw, measured, g.lut, norm, grad_scale, inv_numel, loss, image, amplitude,
        grad_output);
  });
  prof_end(kFpmCols, s);
}

void launch_rows_adjoint(const FpmGeom& g, const float2* spec, const float2* pupil, const int64_t* led, int nf,
                         float2* grad_spec, float2* grad_pupil, cudaStream_t s) {
  const float norm = 1.0f / static_cast<float>((double)g.lh * g.lw);
  prof_begin(kFpmRowsAdjoint, s);
  if (g.generic) {
    MixFpmRowsArgs a{spec, g.oh, g.ow, pupil, g.lh, led, nf, g.frames, g.p_lw.mix_twt, g.p_lw.mix_twi, norm,
                     grad_spec, grad_pupil};
    g.m_lw->rows_adjoint(a, s);
    prof_end(kFpmRowsAdjoint, s);
    return;
  }
  dispatch_pow2(g.lw, [&](auto NT) {
    constexpr int N = decltype(NT)::value;
    const int lines = RowPass<N>::lines(128, g.lh);
    const int rowgroups = (g.lh + lines - 1) / lines;
    const int threads = lines * RowPass<N>::T, smem = FpmRowCfg<N>::smem(lines);
    const int grid = persistent_grid((const void*)fpm_rows_adjoint<N>, threads, smem, (long long)rowgroups * nf);
    launch_pdl(fpm_rows_adjoint<N>, grid, threads, smem, s, g.frames, spec, g.oh, g.ow, pupil, g.lh, led, nf, rowgroups,
                                                    norm, grad_spec, grad_pupil, g.p_lw.tw, lines);
  });
  prof_end(kFpmRowsAdjoint, s);
}

}  // namespace
}  // namespace ptx

using namespace ptx;

extern "C" {

size_t ptx_fpm_workspace_bytes(int object_h, int object_w, int low_h, int low_w, int batch) {
  if (object_h <= 0 || object_w <= 0 || low_h <= 0 || low_w <= 0) return 0;
  const size_t frame = (size_t)num_tiles(low_w) * kTile * low_h * sizeof(float2);
  const size_t frames = std::max<size_t>(1, std::min<size_t>((size_t)std::max(batch, 1), (4096ull << 20) / frame));
  return fpm_fixed_bytes(object_h, object_w) + frames * frame;
}

int ptx_fpm_forward(const float* object, int object_h, int object_w, const float* pupil, int low_h, int low_w,
                    const int64_t* led_indices_xy, int batch, float* spectrum, float* image, float* amplitude,
                    void* workspace, size_t workspace_bytes, void* stream) {
  FpmGeom g;
  if (int st = fpm_check(object, object_h, object_w, pupil, low_h, low_w, led_indices_xy, batch, workspace,
                         workspace_bytes, &g)) {
    return st;
  }
  if (!spectrum || (!amplitude && batch > 0)) return set_error(PTX_ERR_INVALID_ARGUMENT, "null output");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  float2* spec = reinterpret_cast<float2*>(spectrum);
  launch_fft2<false>(g, reinterpret_cast<const float2*>(object), object_h, object_w, spec, 1.0f, g.tmp, g.p_ow, g.p_oh,
                     s);
  const float2* P = reinterpret_cast<const float2*>(pupil);
  for (int b0 = 0; b0 < batch; b0 += g.chunk) {
    const int nf = std::min(g.chunk, batch - b0);
    launch_rows_forward(g, spec, P, led_indices_xy + 2 * (size_t)b0, nf, s);
    launch_cols<kFpmForward>(g, b0, nf, nullptr, 0.f, 0.0, nullptr, reinterpret_cast<float2*>(image),
                             amplitude, nullptr, s);
  }
  return cuda_status(cudaGetLastError(), "ptx_fpm_forward launch");
}

int ptx_fpm_backward(const float* grad_output, const float* image, const float* spectrum, int object_h,
                     int object_w, const float* pupil, int low_h, int low_w, const int64_t* led_indices_xy, int batch,
                     float* grad_object, float* grad_pupil, void* workspace, size_t workspace_bytes, void* stream) {
  FpmGeom g;
  if (int st = fpm_check(spectrum, object_h, object_w, pupil, low_h, low_w, led_indices_xy, batch, workspace,
                         workspace_bytes, &g)) {
    return st;
  }
  if (((!grad_output || !image) && batch > 0) || !grad_object || !grad_pupil) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "null pointer argument");
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaMemsetAsync(g.gspec, 0, g.spec_bytes, s);
  cudaMemsetAsync(grad_pupil, 0, sizeof(float2) * (size_t)low_h * low_w, s);
  const float2* spec = reinterpret_cast<const float2*>(spectrum);
  const float2* P = reinterpret_cast<const float2*>(pupil);
  float2* GP = reinterpret_cast<float2*>(grad_pupil);
  for (int b0 = 0; b0 < batch; b0 += g.chunk) {
    const int nf = std::min(g.chunk, batch - b0);
    launch_cols<kFpmBackward>(g, b0, nf, nullptr, 0.f, 0.0, nullptr,
                              const_cast<float2*>(reinterpret_cast<const float2*>(image)), nullptr, grad_output, s);
    launch_rows_adjoint(g, spec, P, led_indices_xy + 2 * (size_t)b0, nf, g.gspec, GP, s);
  }
  launch_fft2<true>(g, g.gspec, object_h, object_w, reinterpret_cast<float2*>(grad_object), 1.0f, g.tmp, g.p_ow, g.p_oh,
                    s);
  return cuda_status(cudaGetLastError(), "ptx_fpm_backward launch");
}

int ptx_fpm_sweep(const float* object, int object_h, int object_w, const float* pupil, int low_h, int low_w,
                  const int64_t* led_indices_xy, int batch, const uint16_t* measured, float scale, double* loss,
                  float* grad_object, float* grad_pupil, void* workspace, size_t workspace_bytes, void* stream) {
  FpmGeom g;
  if (int st = fpm_check(object, object_h, object_w, pupil, low_h, low_w, led_indices_xy, batch, workspace,
                         workspace_bytes, &g)) {
    return st;
  }
  if ((!measured && batch > 0) || !loss || !grad_object || !grad_pupil) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "null pointer argument");
  }
  if (!(scale > 0.f)) return set_error(PTX_ERR_INVALID_ARGUMENT, "scale must be positive");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const double numel = (double)batch * low_h * low_w;
  const float grad_scale = static_cast<float>(2.0 / std::max(numel, 1.0));
  {
    const size_t ns = g.spec_bytes / sizeof(float2), np = (size_t)low_h * low_w;
    prof_begin(kMiscKernel, s);
    launch_pdl(sweep_prologue_kernel, prologue_blocks(ns, sm_count()), 256, 0, s,
        g.gspec, ns, reinterpret_cast<float2*>(grad_pupil), np, loss, nullptr, g.lut, scale);
    prof_end(kMiscKernel, s);
  }
  launch_fft2<false>(g, reinterpret_cast<const float2*>(object), object_h, object_w, g.spec, 1.0f, g.tmp, g.p_ow, g.p_oh,
                     s);
  const float2* P = reinterpret_cast<const float2*>(pupil);
  float2* GP = reinterpret_cast<float2*>(grad_pupil);
  for (int b0 = 0; b0 < batch; b0 += g.chunk) {
    const int nf = std::min(g.chunk, batch - b0);
    const int64_t* led = led_indices_xy + 2 * (size_t)b0;
    launch_rows_forward(g, g.spec, P, led, nf, s);
    launch_cols<kFpmSweep>(g, b0, nf, measured, grad_scale, 1.0 / std::max(numel, 1.0), loss, nullptr, nullptr,
                           nullptr, s);
    launch_rows_adjoint(g, g.spec, P, led, nf, g.gspec, GP, s);
  }
  launch_fft2<true>(g, g.gspec, object_h, object_w, reinterpret_cast<float2*>(grad_object), 1.0f, g.tmp, g.p_ow, g.p_oh,
                    s);
  return cuda_status(cudaGetLastError(), "ptx_fpm_sweep launch");
}

}  // extern "C"
