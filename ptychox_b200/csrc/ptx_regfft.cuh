// Register-resident two-step FFT for compile-time power-of-two lengths 4..1024.
//
// A line of length N = N1 * T is held by T threads, thread t owning the N1 values
// x[t + T j] (j < N1) -- consecutive threads own consecutive elements, so a line is
// loaded from and stored to global memory with coalesced accesses straight from
// registers.  The transform is the two-factor Cooley-Tukey decomposition
//   X[k1 + N1 k2] = sum_t W_T^{t k2} [ W_N^{t k1} sum_j x[t + T j] W_N1^{j k1} ]:
//   1. each thread: DFT-N1 over its own values (registers), twiddle by W_N^{t k1};
//   2. one transpose through a padded shared-memory buffer;
//   3. each thread: N1/T DFT-T over rows k1 = q T + t.
// The output lands in the input layout (thread t owns X[t + T m], m < N1), so a
// pointwise epilogue and a second transform along the same axis need no reshuffle.
// In-register DFTs are Cooley-Tukey compositions of radix-2/4/8 kernels with constant
// twiddles; inter-step twiddles come from the FP64-derived table of the line plan.
#pragma once

#include "ptx_fft.cuh"

namespace ptx {

__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n / 2); }

template <int N>
struct RegShape {
  static constexpr int LOG = ilog2c(N);
  static constexpr int N1 = 1 << ((LOG + 1) / 2);  // values per thread
  static constexpr int T = N / N1;                 // threads per line
  static constexpr int C = N1 / T;                 // step-3 DFTs per thread (1 or 2)
  static constexpr int RP = T + 1;                 // exchange row pitch (odd)
  static constexpr int BUF = N1 * RP;              // exchange buffer per line (float2)
  static constexpr int RPV = T + 2;                // even pitch of the row-pass exchange
  static constexpr int BUFV = N1 * RPV;            // its buffer per line (float2)
  static_assert((1 << LOG) == N && N >= 4 && N <= 1024, "power of two in [4, 1024]");
};

// cos(2 pi m / 32) and sin(2 pi m / 32), m in [0, 32): after unrolling, m is a compile-time
// constant and the switch folds to an immediate.
__host__ __device__ __forceinline__ float cos32(int m) {
  switch (m & 31) {
    case 0: return 1.0f;
    case 1: return 0.9807852804032304f;
    case 2: return 0.9238795325112867f;
    case 3: return 0.8314696123025452f;
    case 4: return 0.7071067811865476f;
    case 5: return 0.5555702330196023f;
    case 6: return 0.38268343236508984f;
    case 7: return 0.19509032201612833f;
    case 8: return 0.0f;
    case 9: return -0.1950903220161282f;
    case 10: return -0.3826834323650897f;
    case 11: return -0.555570233019602f;
    case 12: return -0.7071067811865475f;
    case 13: return -0.8314696123025453f;
    case 14: return -0.9238795325112867f;
    case 15: return -0.9807852804032304f;
    case 16: return -1.0f;
    case 17: return -0.9807852804032304f;
    case 18: return -0.9238795325112868f;
    case 19: return -0.8314696123025455f;
    case 20: return -0.7071067811865477f;
    case 21: return -0.5555702330196022f;
    case 22: return -0.38268343236509034f;
    case 23: return -0.19509032201612866f;
    case 24: return 0.0f;
    case 25: return 0.1950903220161283f;
    case 26: return 0.38268343236509f;
    case 27: return 0.5555702330196018f;
    case 28: return 0.7071067811865474f;
    case 29: return 0.8314696123025452f;
    case 30: return 0.9238795325112865f;
    case 31: return 0.9807852804032303f;
    default: return 0.f;
  }
}
__host__ __device__ __forceinline__ float sin32(int m) {
  switch (m & 31) {
    case 0: return 0.0f;
    case 1: return 0.19509032201612825f;
    case 2: return 0.3826834323650898f;
    case 3: return 0.5555702330196022f;
    case 4: return 0.7071067811865475f;
    case 5: return 0.8314696123025452f;
    case 6: return 0.9238795325112867f;
    case 7: return 0.9807852804032304f;
    case 8: return 1.0f;
    case 9: return 0.9807852804032304f;
    case 10: return 0.9238795325112867f;
    case 11: return 0.8314696123025455f;
    case 12: return 0.7071067811865476f;
    case 13: return 0.5555702330196022f;
    case 14: return 0.3826834323650899f;
    case 15: return 0.1950903220161286f;
    case 16: return 0.0f;
    case 17: return -0.19509032201612836f;
    case 18: return -0.38268343236508967f;
    case 19: return -0.555570233019602f;
    case 20: return -0.7071067811865475f;
    case 21: return -0.8314696123025452f;
    case 22: return -0.9238795325112865f;
    case 23: return -0.9807852804032303f;
    case 24: return -1.0f;
    case 25: return -0.9807852804032304f;
    case 26: return -0.9238795325112866f;
    case 27: return -0.8314696123025455f;
    case 28: return -0.7071067811865477f;
    case 29: return -0.5555702330196022f;
    case 30: return -0.3826834323650904f;
    case 31: return -0.19509032201612872f;
    default: return 0.f;
  }
}

// z * exp(-+ 2 pi i m / N) for N dividing 32 and compile-time m; trivial angles avoid
// multiplications (which would not fold without fast-math).
template <int N, bool INV>
__device__ __forceinline__ float2 wroot(float2 z, int m) {
  const int e = ((m % N) + N) % N * (32 / N);  // angle in 32nds of a turn
  if (e == 0) return z;
  if (e == 16) return make_float2(-z.x, -z.y);
  if (e == 8) return mul_i<INV>(z);
  if (e == 24) return mul_i<!INV>(z);
  const float c = cos32(e);
  const float s = INV ? sin32(e) : -sin32(e);
  return make_float2(fmaf(z.x, c, -z.y * s), fmaf(z.x, s, z.y * c));
}

// In-register DFT of length A*B by one Cooley-Tukey step: n = n1 + A n2, k = B k1 + k2.
template <int A, int B, bool INV>
__device__ __forceinline__ void dft_ct(float2* v) {
  constexpr int N = A * B;
  float2 y[N];
#pragma unroll
  for (int n1 = 0; n1 < A; ++n1) {
    float2 col[B];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) col[n2] = v[n1 + A * n2];
    Dft<B, INV>::run(col);
#pragma unroll
    for (int k2 = 0; k2 < B; ++k2) y[n1 * B + k2] = wroot<N, INV>(col[k2], n1 * k2);
  }
#pragma unroll
  for (int k2 = 0; k2 < B; ++k2) {
    float2 row[A];
#pragma unroll
    for (int n1 = 0; n1 < A; ++n1) row[n1] = y[n1 * B + k2];
    Dft<A, INV>::run(row);
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) v[B * k1 + k2] = row[k1];
  }
}

template <int N, bool INV>
struct RegDft {
  __device__ __forceinline__ static void run(float2* v) { Dft<N, INV>::run(v); }
};
template <bool INV>
struct RegDft<16, INV> {
  __device__ __forceinline__ static void run(float2* v) { dft_ct<4, 4, INV>(v); }
};
template <bool INV>
struct RegDft<32, INV> {
  __device__ __forceinline__ static void run(float2* v) { dft_ct<4, 8, INV>(v); }
};

// Line-buffer pitch (float2) for kernels whose threads run t-fastest (row passes): lines
// sharing a half-warp land on disjoint bank sets.
// Sized for the larger (even-pitch) exchange of the row passes.
template <int N>
__host__ __device__ constexpr int row_line_pitch() {
  using S = RegShape<N>;
  return S::T >= 16 ? S::BUFV : S::BUFV + ((S::T - S::BUFV % 16) + 16) % 16;
}
// Line-buffer pitch for kernels whose threads run column-fastest (column passes): a
// half-warp holds 8 columns x 2 line threads, and with a pitch = 2 (mod 16) (in float2)
// next to the odd row pitch their 16 accesses hit 16 distinct bank pairs.
template <int N>
__host__ __device__ constexpr int col_line_pitch() {
  return RegShape<N>::BUF + ((2 - RegShape<N>::BUF % 16) + 16) % 16;
}

// Fill the shared-memory table of reg_fft<..., TW_SHARED = true> from the global table
// exp(-2 pi i m / N): entry k1 * T + t holds m = t * k1 (always < N).  All threads of the
// block call it; the caller synchronises before use.
template <int N>
__device__ __forceinline__ void load_twiddles_by_thread(float2* dst, const float2* __restrict__ tw) {
  using S = RegShape<N>;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const int k1 = i / S::T, t = i - k1 * S::T;
    dst[i] = __ldg(&tw[t * k1]);
  }
}

template <bool BLOCK>
__device__ __forceinline__ void line_sync() {
  if (BLOCK) {
    __syncthreads();
  } else {
    __syncwarp();
  }
}

// Transform the line owned by threads t = 0..T-1 in place (see the file comment for the
// layout).  `buf` is this line's exchange buffer (RegShape<N>::BUF float2).  BLOCK
// selects a block-wide barrier (lines spread over several warps) instead of a warp one;
// every thread of the block (or warp) must call it.  TW_SHARED: `tw` points to a
// shared-memory table laid out by thread, tw[k1 * T + t] = exp(-2 pi i t k1 / N) (see
// load_twiddles_by_thread), so the T lanes of a line read consecutive words.
//
// The row-pass form (TW_SHARED, line buffers of row_line_pitch, 16-byte aligned) lays the
// exchange out with the even pitch RPV, so step 3 reads its contiguous row two elements per
// 16-byte load (half the shared-memory load instructions); with T lanes per line the loads
// of a warp still take the minimum number of shared-memory wavefronts.
template <int N, bool INV, bool BLOCK, bool TW_SHARED = false>
__device__ __forceinline__ void reg_fft(float2 (&v)[RegShape<N>::N1], float2* buf, int t,
                                        const float2* __restrict__ tw) {
  using S = RegShape<N>;
  constexpr int RP = TW_SHARED ? S::RPV : S::RP;
  RegDft<S::N1, INV>::run(v);
#pragma unroll
  for (int k1 = 1; k1 < S::N1; ++k1) {
    float2 w = TW_SHARED ? tw[k1 * S::T + t] : __ldg(&tw[t * k1]);
    if (INV) w.y = -w.y;
    v[k1] = cmul(v[k1], w);
  }
#pragma unroll
  for (int k1 = 0; k1 < S::N1; ++k1) buf[k1 * RP + t] = v[k1];
  line_sync<BLOCK>();
#pragma unroll
  for (int q = 0; q < S::C; ++q) {
    float2 u[S::T];
    if constexpr (TW_SHARED) {
      const float4* row = reinterpret_cast<const float4*>(buf + (q * S::T + t) * RP);
#pragma unroll
      for (int j = 0; j < S::T / 2; ++j) {
        const float4 x = row[j];
        u[2 * j] = make_float2(x.x, x.y);
        u[2 * j + 1] = make_float2(x.z, x.w);
      }
    } else {
#pragma unroll
      for (int j2 = 0; j2 < S::T; ++j2) u[j2] = buf[(q * S::T + t) * RP + j2];
    }
    RegDft<S::T, INV>::run(u);
#pragma unroll
    for (int k2 = 0; k2 < S::T; ++k2) v[q + S::C * k2] = u[k2];
  }
  line_sync<BLOCK>();
}

}  // namespace ptx
