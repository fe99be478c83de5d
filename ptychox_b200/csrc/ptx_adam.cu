// Fused Adam step on complex64 parameters, with the reference drivers' constraints.
//
// The reference optimises object, probe / pupil / coded surface with torch.optim.Adam
// (python/train_ptychography.py:500-507, train_fpm.py, train_coded.py), which treats a
// complex parameter as its (re, im) pairs (torch/optim/adam.py, view_as_real):
//   m = lerp(m, g, 1 - b1);  v = b2 v + (1 - b2) g^2
//   p -= (lr / (1 - b1^t)) * m / (sqrt(v) / sqrt(1 - b2^t) + eps)
// followed, where the drivers do so, by a projection: |z| <= 1 keeping the phase (the
// MATLAB reconstruction scripts' amplitude clamp, matlab/Benchmarks/.../test_recon.m:172-181)
// or z -> max(Re z, 0) (the real non-negative coded surface, train_coded.py:242-244).
//
// One pass reads p, g, m, v and writes p, m, v (HBM-bound, 56 bytes per element).  The
// step count lives on the device so a captured CUDA graph can replay the step: a
// one-thread kernel advances it and computes the two bias-correction scalars in FP64.
#include <cuda_runtime.h>

#include <cmath>

#include "ptx_internal.h"

namespace ptx {
namespace {

struct AdamState {
  int step;
  float step_size;   // lr / (1 - b1^t)
  float bc2_sqrt;    // sqrt(1 - b2^t)
  float pad;
};

__global__ void adam_advance(AdamState* st, float lr, float beta1, float beta2) {
  const int t = st->step + 1;
  st->step = t;
  const double bc1 = 1.0 - pow((double)beta1, (double)t);
  const double bc2 = 1.0 - pow((double)beta2, (double)t);
  st->step_size = static_cast<float>((double)lr / bc1);
  st->bc2_sqrt = static_cast<float>(sqrt(bc2));
}

__device__ __forceinline__ float adam_update(float p, float g, float& m, float& v, float one_m_b1, float beta2,
                                             float one_m_b2, float eps, float step_size, float bc2_sqrt) {
  m = fmaf(one_m_b1, g - m, m);
  v = fmaf(one_m_b2, g * g, beta2 * v);
  const float denom = sqrtf(v) / bc2_sqrt + eps;
  return p - step_size * (m / denom);
}

__global__ void adam_complex(float4* __restrict__ param, const float4* __restrict__ grad, float4* __restrict__ m,
                             float4* __restrict__ v, size_t n_pairs, const AdamState* __restrict__ st, float beta1,
                             float beta2, float eps, int constraint) {
  const float step_size = st->step_size, bc2_sqrt = st->bc2_sqrt;
  const float one_m_b1 = 1.0f - beta1, one_m_b2 = 1.0f - beta2;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n_pairs; i += (size_t)gridDim.x * blockDim.x) {
    float4 p = param[i], g = grad[i], mm = m[i], vv = v[i];
    p.x = adam_update(p.x, g.x, mm.x, vv.x, one_m_b1, beta2, one_m_b2, eps, step_size, bc2_sqrt);
    p.y = adam_update(p.y, g.y, mm.y, vv.y, one_m_b1, beta2, one_m_b2, eps, step_size, bc2_sqrt);
    p.z = adam_update(p.z, g.z, mm.z, vv.z, one_m_b1, beta2, one_m_b2, eps, step_size, bc2_sqrt);
    p.w = adam_update(p.w, g.w, mm.w, vv.w, one_m_b1, beta2, one_m_b2, eps, step_size, bc2_sqrt);
    if (constraint == PTX_CONSTRAIN_UNIT_AMPLITUDE) {
      const float a0 = sqrtf(p.x * p.x + p.y * p.y), a1 = sqrtf(p.z * p.z + p.w * p.w);
      if (a0 > 1.f) { p.x /= a0; p.y /= a0; }
      if (a1 > 1.f) { p.z /= a1; p.w /= a1; }
    } else if (constraint == PTX_CONSTRAIN_REAL_NONNEGATIVE) {
      p.x = fmaxf(p.x, 0.f); p.y = 0.f;
      p.z = fmaxf(p.z, 0.f); p.w = 0.f;
    }
    param[i] = p;
    m[i] = mm;
    v[i] = vv;
  }
}

// odd trailing element (n_complex odd)
__global__ void adam_tail(float2* __restrict__ param, const float2* __restrict__ grad, float2* __restrict__ m,
                          float2* __restrict__ v, const AdamState* __restrict__ st, float beta1, float beta2,
                          float eps, int constraint) {
  float2 p = *param, g = *grad, mm = *m, vv = *v;
  p.x = adam_update(p.x, g.x, mm.x, vv.x, 1.f - beta1, beta2, 1.f - beta2, eps, st->step_size, st->bc2_sqrt);
  p.y = adam_update(p.y, g.y, mm.y, vv.y, 1.f - beta1, beta2, 1.f - beta2, eps, st->step_size, st->bc2_sqrt);
  if (constraint == PTX_CONSTRAIN_UNIT_AMPLITUDE) {
    const float a = sqrtf(p.x * p.x + p.y * p.y);
    if (a > 1.f) { p.x /= a; p.y /= a; }
  } else if (constraint == PTX_CONSTRAIN_REAL_NONNEGATIVE) {
    p.x = fmaxf(p.x, 0.f); p.y = 0.f;
  }
  *param = p; *m = mm; *v = vv;
}

}  // namespace
}  // namespace ptx

using namespace ptx;

extern "C" int ptx_adam_step(float* param, const float* grad, float* exp_avg, float* exp_avg_sq, size_t n_complex,
                             void* state, float lr, float beta1, float beta2, float eps, int constraint, void* stream) {
  if (!param || !grad || !exp_avg || !exp_avg_sq || !state) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "null pointer argument");
  }
  if (constraint < PTX_CONSTRAIN_NONE || constraint > PTX_CONSTRAIN_REAL_NONNEGATIVE) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "unknown constraint %d", constraint);
  }
  for (const void* p : {(const void*)param, (const void*)grad, (const void*)exp_avg, (const void*)exp_avg_sq}) {
    if (reinterpret_cast<uintptr_t>(p) & 15) return set_error(PTX_ERR_INVALID_ARGUMENT, "arrays must be 16-byte aligned");
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  AdamState* st = static_cast<AdamState*>(state);
  prof_begin(kMiscKernel, s);
  adam_advance<<<1, 1, 0, s>>>(st, lr, beta1, beta2);
  const size_t pairs = n_complex / 2;
  if (pairs) {
    const int threads = 256;
    const size_t want = (pairs + threads - 1) / threads;
    const int blocks = static_cast<int>(std::min<size_t>(want, (size_t)sm_count() * 16));
    adam_complex<<<blocks, threads, 0, s>>>(reinterpret_cast<float4*>(param), reinterpret_cast<const float4*>(grad),
                                            reinterpret_cast<float4*>(exp_avg), reinterpret_cast<float4*>(exp_avg_sq),
                                            pairs, st, beta1, beta2, eps, constraint);
  }
  if (n_complex & 1) {
    const size_t last = n_complex - 1;
    adam_tail<<<1, 1, 0, s>>>(reinterpret_cast<float2*>(param) + last, reinterpret_cast<const float2*>(grad) + last,
                              reinterpret_cast<float2*>(exp_avg) + last, reinterpret_cast<float2*>(exp_avg_sq) + last,
                              st, beta1, beta2, eps, constraint);
  }
  prof_end(kMiscKernel, s);
  return cuda_status(cudaGetLastError(), "ptx_adam_step launch");
}
