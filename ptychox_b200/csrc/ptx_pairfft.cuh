// Two-line register FFT on packed FP32x2 arithmetic (sm_100).
//
// Blackwell executes FP32 add / multiply / fma on register pairs (`add.f32x2` and
// friends, exposed as __fadd2_rn / __fmul2_rn / __ffma2_rn): one instruction does the same
// IEEE operation on two lanes.  A complex FFT written on (re, im) float2 values cannot use
// them directly, because a complex product mixes the lanes.  Here one thread transforms TWO
// lines at once with their values in structure-of-arrays pairs: CPair{re, im} holds
// re = (line A real, line B real) and im = (line A imag, line B imag).  Every operation of
// the transform is the same for both lines (same indices, same twiddles), so each scalar
// operation of the one-line FFT becomes one packed operation on the pair: half the issue
// slots for the same arithmetic, with results bit-identical to the scalar one-line code
// that uses the same rounding steps.
//
// Layout and algorithm are those of reg_fft (ptx_regfft.cuh): N = N1 * T, thread t of the
// T threads of a line pair owns elements t + T j (j < N1) of both lines; a DFT-N1 in
// registers, twiddles from a table, one exchange through shared memory (one float4
// (reA, reB, imA, imB) per element pair), then C = N1 / T DFT-T per thread.  The result
// lands in the input layout.  Subtractions are written as fma(b, -1, a), which rounds once
// exactly like a - b.
//
// All helpers are __host__ __device__ so the transform can be checked on the CPU.
#pragma once

#include <cuda_runtime.h>

#include "ptx_regfft.cuh"

namespace ptx {

struct CPair {
  float2 re;  // (line A, line B) real parts
  float2 im;  // (line A, line B) imaginary parts
};

__host__ __device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

__host__ __device__ __forceinline__ float2 add2(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  return __fadd2_rn(a, b);
#else
  return make_float2(a.x + b.x, a.y + b.y);
#endif
}
__host__ __device__ __forceinline__ float2 mul2(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  return __fmul2_rn(a, b);
#else
  return make_float2(a.x * b.x, a.y * b.y);
#endif
}
__host__ __device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  return __ffma2_rn(a, b, c);
#else
  return make_float2(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y));
#endif
}
// a - b (one rounding, as the scalar subtraction)
__host__ __device__ __forceinline__ float2 sub2(float2 a, float2 b) { return fma2(b, f2(-1.0f), a); }
__host__ __device__ __forceinline__ float2 neg2(float2 a) { return mul2(a, f2(-1.0f)); }

__host__ __device__ __forceinline__ CPair padd(CPair a, CPair b) { return {add2(a.re, b.re), add2(a.im, b.im)}; }
__host__ __device__ __forceinline__ CPair psub(CPair a, CPair b) { return {sub2(a.re, b.re), sub2(a.im, b.im)}; }
// a + m b and a - m b with m = -i (forward) or +i (inverse): lane swaps fold into the add
template <bool INV>
__host__ __device__ __forceinline__ CPair padd_mi(CPair a, CPair b) {
  // forward: -i b = (b.im, -b.re);  inverse: +i b = (-b.im, b.re)
  return INV ? CPair{sub2(a.re, b.im), add2(a.im, b.re)} : CPair{add2(a.re, b.im), sub2(a.im, b.re)};
}
template <bool INV>
__host__ __device__ __forceinline__ CPair psub_mi(CPair a, CPair b) {
  return INV ? CPair{add2(a.re, b.im), sub2(a.im, b.re)} : CPair{sub2(a.re, b.im), add2(a.im, b.re)};
}
template <bool INV>
__host__ __device__ __forceinline__ CPair pmul_i(CPair z) {
  return INV ? CPair{neg2(z.im), z.re} : CPair{z.im, neg2(z.re)};
}
// z * (c + i s), the same factor on both lanes
__host__ __device__ __forceinline__ CPair pmul(CPair z, float c, float s) {
  return {fma2(z.im, f2(-s), mul2(z.re, f2(c))), fma2(z.im, f2(c), mul2(z.re, f2(s)))};
}

// z * exp(-+ 2 pi i m / N) for N dividing 32 and compile-time m (trivial angles exact)
template <int N, bool INV>
__host__ __device__ __forceinline__ CPair proot(CPair z, int m) {
  const int e = ((m % N) + N) % N * (32 / N);
  if (e == 0) return z;
  if (e == 16) return {neg2(z.re), neg2(z.im)};
  if (e == 8) return pmul_i<INV>(z);
  if (e == 24) return pmul_i<!INV>(z);
  const float c = cos32(e);
  const float s = INV ? sin32(e) : -sin32(e);
  return pmul(z, c, s);
}

template <int R, bool INV>
struct PDft;

template <bool INV>
struct PDft<2, INV> {
  __host__ __device__ __forceinline__ static void run(CPair* v) {
    const CPair a = v[0], b = v[1];
    v[0] = padd(a, b);
    v[1] = psub(a, b);
  }
};

template <bool INV>
struct PDft<4, INV> {
  __host__ __device__ __forceinline__ static void run(CPair* v) {
    const CPair t0 = padd(v[0], v[2]);
    const CPair t1 = psub(v[0], v[2]);
    const CPair t2 = padd(v[1], v[3]);
    const CPair d = psub(v[1], v[3]);
    v[0] = padd(t0, t2);
    v[2] = psub(t0, t2);
    v[1] = padd_mi<INV>(t1, d);
    v[3] = psub_mi<INV>(t1, d);
  }
};

template <bool INV>
struct PDft<8, INV> {
  __host__ __device__ __forceinline__ static void run(CPair* v) {
    constexpr float h = 0.70710678118654752f;
    CPair e[4] = {v[0], v[2], v[4], v[6]};
    CPair o[4] = {v[1], v[3], v[5], v[7]};
    PDft<4, INV>::run(e);
    PDft<4, INV>::run(o);
    // o1 = o[1] exp(-+ i pi/4), o3 = o[3] exp(-+ 3 i pi/4); o[2] enters through padd_mi
    const CPair o1 = INV ? CPair{mul2(f2(h), sub2(o[1].re, o[1].im)), mul2(f2(h), add2(o[1].re, o[1].im))}
                         : CPair{mul2(f2(h), add2(o[1].re, o[1].im)), mul2(f2(h), sub2(o[1].im, o[1].re))};
    const CPair o3 = INV ? CPair{mul2(f2(-h), add2(o[3].re, o[3].im)), mul2(f2(h), sub2(o[3].re, o[3].im))}
                         : CPair{mul2(f2(h), sub2(o[3].im, o[3].re)), mul2(f2(-h), add2(o[3].re, o[3].im))};
    v[0] = padd(e[0], o[0]);
    v[4] = psub(e[0], o[0]);
    v[1] = padd(e[1], o1);
    v[5] = psub(e[1], o1);
    v[2] = padd_mi<INV>(e[2], o[2]);
    v[6] = psub_mi<INV>(e[2], o[2]);
    v[3] = padd(e[3], o3);
    v[7] = psub(e[3], o3);
  }
};

// One Cooley-Tukey step for a length A*B in registers: n = n1 + A n2, k = B k1 + k2.
template <int A, int B, bool INV>
__host__ __device__ __forceinline__ void pdft_ct(CPair* v) {
  constexpr int N = A * B;
  CPair y[N];
#pragma unroll
  for (int n1 = 0; n1 < A; ++n1) {
    CPair col[B];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) col[n2] = v[n1 + A * n2];
    PDft<B, INV>::run(col);
#pragma unroll
    for (int k2 = 0; k2 < B; ++k2) y[n1 * B + k2] = proot<N, INV>(col[k2], n1 * k2);
  }
#pragma unroll
  for (int k2 = 0; k2 < B; ++k2) {
    CPair row[A];
#pragma unroll
    for (int n1 = 0; n1 < A; ++n1) row[n1] = y[n1 * B + k2];
    PDft<A, INV>::run(row);
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) v[B * k1 + k2] = row[k1];
  }
}

template <int N, bool INV>
struct PRegDft {
  __host__ __device__ __forceinline__ static void run(CPair* v) { PDft<N, INV>::run(v); }
};
template <bool INV>
struct PRegDft<16, INV> {
  __host__ __device__ __forceinline__ static void run(CPair* v) { pdft_ct<4, 4, INV>(v); }
};
template <bool INV>
struct PRegDft<32, INV> {
  __host__ __device__ __forceinline__ static void run(CPair* v) { pdft_ct<4, 8, INV>(v); }
};

// Exchange-buffer float4 layout of one element pair
__host__ __device__ __forceinline__ float4 pack4(CPair z) { return make_float4(z.re.x, z.re.y, z.im.x, z.im.y); }
__host__ __device__ __forceinline__ CPair unpack4(float4 q) { return {make_float2(q.x, q.y), make_float2(q.z, q.w)}; }

// Step 1 of the two-line transform: DFT-N1 in registers and the inter-step twiddles
// tw4[t * k1] = (w.x, w.x, w.y, w.y) of exp(-2 pi i t k1 / N) (conjugated for INV).
template <int N, bool INV>
__host__ __device__ __forceinline__ void pair_fft_step1(CPair (&v)[RegShape<N>::N1], int t, const float4* tw4) {
  using S = RegShape<N>;
  PRegDft<S::N1, INV>::run(v);
#pragma unroll
  for (int k1 = 1; k1 < S::N1; ++k1) {
    const float4 w = tw4[t * k1];
    const float2 wx = make_float2(w.x, w.y);
    const float2 wy = INV ? neg2(make_float2(w.z, w.w)) : make_float2(w.z, w.w);
    const CPair z = v[k1];
    v[k1] = {fma2(z.im, neg2(wy), mul2(z.re, wx)), fma2(z.im, wx, mul2(z.re, wy))};
  }
}
// Step 2 of the two-line transform for exchange buffer row r: C DFT-T on the transposed data.
template <int N, bool INV>
__host__ __device__ __forceinline__ void pair_fft_step2_load(CPair (&v)[RegShape<N>::N1], const float4* buf, int t) {
  using S = RegShape<N>;
#pragma unroll
  for (int q = 0; q < S::C; ++q) {
    CPair u[S::T];
#pragma unroll
    for (int j2 = 0; j2 < S::T; ++j2) u[j2] = unpack4(buf[(q * S::T + t) * S::RP + j2]);
    PRegDft<S::T, INV>::run(u);
#pragma unroll
    for (int k2 = 0; k2 < S::T; ++k2) v[q + S::C * k2] = u[k2];
  }
}

// Transform the line pair owned by threads t = 0..T-1 in place.  `buf` is the pair's
// exchange buffer (RegShape<N>::BUF float4); BLOCK selects a block-wide barrier instead of
// a warp one (every thread of the block or warp must call it); `tw4` is the broadcast
// twiddle table (shared memory).
template <int N, bool INV, bool BLOCK>
__device__ __forceinline__ void pair_fft(CPair (&v)[RegShape<N>::N1], float4* buf, int t, const float4* tw4) {
  using S = RegShape<N>;
  pair_fft_step1<N, INV>(v, t, tw4);
#pragma unroll
  for (int k1 = 0; k1 < S::N1; ++k1) buf[k1 * S::RP + t] = pack4(v[k1]);
  line_sync<BLOCK>();
  pair_fft_step2_load<N, INV>(v, buf, t);
  line_sync<BLOCK>();
}

}  // namespace ptx
