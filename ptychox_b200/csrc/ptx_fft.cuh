// Shared-memory Stockham FFT engine for sm_100a.
//
// A "line" is one 1-D transform of length n held contiguously in shared memory.
// ceil(n/16) threads cooperate on a line, each holding at most 16..20 complex values
// in registers per stage.  Lines are transformed in place: each stage loads its
// butterfly inputs into registers, applies the inter-stage twiddles, runs a radix-R
// DFT in registers, synchronises, and writes the outputs back in Stockham autosort
// order, so the result is in natural order with no bit reversal.  Radices 2, 3, 4, 5,
// 8 and 16 are supported; the plan (radix sequence) is chosen on the host.
// The register engines (ptx_regfft.cuh / ptx_pairfft.cuh for powers of two from 16,
// ptx_mixfft.cuh for the other smooth lengths from 6) take every longer line, so in the
// sweeps this engine serves only lengths 2 .. 8 (ptx_fft_engine in include/ptychox.h).
//
// Twiddles come from a per-size table exp(-2 pi i m / n), m < n, computed on the host in
// FP64 (std::cos / std::sin) and rounded once to FP32.  Both directions are
// unnormalised, matching torch.fft.fft2 / n*ifft2 (the conventions the operators of
// python/ptychoX use: base/ops.py:65,95).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ptx {

constexpr int kMaxStages = 12;
constexpr int kValuesPerThread = 16;

struct LinePlan {
  int n;                      // line length
  int threads;                // threads per line = ceil(n / 16)
  int nstages;                // number of radix stages
  unsigned long long radices; // radix of stage s in bits [5s, 5s+5)
  const float2* tw;           // device table exp(-2 pi i m / n), m in [0, n)
  // the mixed-radix engine's split n = A * B (mix::Shape): the two layouts of
  // exp(-2 pi i t u / n), t < B, u < A, mix_twt[u * B + t] = mix_twi[t * A + u]
  const float2* mix_twt;
  const float2* mix_twi;
};

__host__ __device__ __forceinline__ int plan_radix(const LinePlan& p, int s) {
  return static_cast<int>((p.radices >> (5 * s)) & 31ull);
}

// --------------------------------------------------------------------------------------
// complex helpers
// --------------------------------------------------------------------------------------
// complex add / subtract as one packed FP32x2 instruction on sm_100 (a - b as fma(b, -1, a),
// which rounds once exactly like the subtraction)
__device__ __forceinline__ float2 cadd(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  return __fadd2_rn(a, b);
#else
  return make_float2(a.x + b.x, a.y + b.y);
#endif
}
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  return __ffma2_rn(b, make_float2(-1.f, -1.f), a);
#else
  return make_float2(a.x - b.x, a.y - b.y);
#endif
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float cabs2(float2 a) { return fmaf(a.x, a.x, a.y * a.y); }
__device__ __forceinline__ float cabsf(float2 a) { return sqrtf(cabs2(a)); }

// Ampere-style asynchronous global->shared copies (cp.async): the data lands in shared
// memory without passing through registers; each thread waits only for its own copies.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

// First statement of every kernel launched by launch_pdl: wait until the preceding grid on
// the stream has completed and its memory is visible (returns at once for a plain launch).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// L2 eviction policies for the cache-hinted copies below: streamed data (scratch frames)
// evict-first, data re-read across frames (object, spectrum) evict-last.
__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;\n" : "=l"(p));
  return p;
}
// 16-byte global -> shared copy that bypasses L1, with an L2 eviction policy
__device__ __forceinline__ void cp_async16_hint(void* smem, const void* gmem, uint64_t pol) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void cp_async8_hint(void* smem, const void* gmem, uint64_t pol) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "l"(pol)
               : "memory");
}

// 16-byte global load that does not allocate in L1, with an L2 eviction policy (streamed
// scratch elements that this thread reads once)
__device__ __forceinline__ float4 ld_stream4(const float2* p, uint64_t pol) {
  float4 v;
  asm("ld.global.L1::no_allocate.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;\n"
      : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
      : "l"(p), "l"(pol));
  return v;
}

// multiply by -i (forward transform) or +i (inverse transform)
template <bool INV>
__device__ __forceinline__ float2 mul_i(float2 z) {
  return INV ? make_float2(-z.y, z.x) : make_float2(z.y, -z.x);
}
// multiply by exp(-+ 2 pi i m / 16) for the radix-16 internal twiddles
template <bool INV>
__device__ __forceinline__ float2 w16(float2 z, int m) {
  // cos / sin of multiples of pi/8
  constexpr float c1 = 0.92387953251128674f;   // cos(pi/8)
  constexpr float s1 = 0.38268343236508978f;   // sin(pi/8)
  constexpr float h = 0.70710678118654752f;    // cos(pi/4)
  float c, s;  // exp(-i theta) = (c, -s) forward
  switch (m) {
    case 0: return z;
    case 1: c = c1; s = s1; break;
    case 2: c = h; s = h; break;
    case 3: c = s1; s = c1; break;
    case 4: return mul_i<INV>(z);
    case 6: c = -h; s = h; break;
    case 9: c = -c1; s = -s1; break;
    default: c = 1.f; s = 0.f; break;
  }
  const float2 w = INV ? make_float2(c, s) : make_float2(c, -s);
  return cmul(z, w);
}

// --------------------------------------------------------------------------------------
// in-register DFTs (natural order in, natural order out)
// --------------------------------------------------------------------------------------
template <int R, bool INV>
struct Dft;

template <bool INV>
struct Dft<2, INV> {
  __device__ __forceinline__ static void run(float2* v) {
    const float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <bool INV>
struct Dft<4, INV> {
  __device__ __forceinline__ static void run(float2* v) {
    const float2 t0 = cadd(v[0], v[2]);
    const float2 t1 = csub(v[0], v[2]);
    const float2 t2 = cadd(v[1], v[3]);
    const float2 t3 = mul_i<INV>(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[1] = cadd(t1, t3);
    v[2] = csub(t0, t2);
    v[3] = csub(t1, t3);
  }
};

template <bool INV>
struct Dft<8, INV> {
  __device__ __forceinline__ static void run(float2* v) {
    constexpr float h = 0.70710678118654752f;
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    Dft<4, INV>::run(e);
    Dft<4, INV>::run(o);
    // o[k] *= exp(-+ 2 pi i k / 8)
    const float2 o1 = INV ? make_float2(h * (o[1].x - o[1].y), h * (o[1].x + o[1].y))
                          : make_float2(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));
    const float2 o2 = mul_i<INV>(o[2]);
    const float2 o3 = INV ? make_float2(-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y))
                          : make_float2(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], o1);
    v[5] = csub(e[1], o1);
    v[2] = cadd(e[2], o2);
    v[6] = csub(e[2], o2);
    v[3] = cadd(e[3], o3);
    v[7] = csub(e[3], o3);
  }
};

template <bool INV>
struct Dft<16, INV> {
  // 4 x 4 decomposition: n = 4 n1 + n2, k = k1 + 4 k2.
  __device__ __forceinline__ static void run(float2* v) {
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
      float2 col[4] = {v[n2], v[4 + n2], v[8 + n2], v[12 + n2]};
      Dft<4, INV>::run(col);
#pragma unroll
      for (int k1 = 0; k1 < 4; ++k1) v[4 * k1 + n2] = w16<INV>(col[k1], n2 * k1);
    }
    float2 out[16];
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
      float2 row[4] = {v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]};
      Dft<4, INV>::run(row);
#pragma unroll
      for (int k2 = 0; k2 < 4; ++k2) out[k1 + 4 * k2] = row[k2];
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = out[i];
  }
};

template <bool INV>
struct Dft<3, INV> {
  __device__ __forceinline__ static void run(float2* v) {
    constexpr float r3 = 0.86602540378443865f;  // sqrt(3) / 2
    const float2 t = cadd(v[1], v[2]);
    const float2 d = mul_i<INV>(csub(v[1], v[2]));
    const float2 m = make_float2(fmaf(-0.5f, t.x, v[0].x), fmaf(-0.5f, t.y, v[0].y));
    v[0] = cadd(v[0], t);
    v[1] = make_float2(fmaf(r3, d.x, m.x), fmaf(r3, d.y, m.y));
    v[2] = make_float2(fmaf(-r3, d.x, m.x), fmaf(-r3, d.y, m.y));
  }
};

template <bool INV>
struct Dft<5, INV> {
  __device__ __forceinline__ static void run(float2* v) {
    constexpr float c1 = 0.30901699437494742f;   // cos(2 pi / 5)
    constexpr float c2 = -0.80901699437494742f;  // cos(4 pi / 5)
    constexpr float s1 = 0.95105651629515357f;   // sin(2 pi / 5)
    constexpr float s2 = 0.58778525229247313f;   // sin(4 pi / 5)
    const float2 sa = cadd(v[1], v[4]);
    const float2 da = csub(v[1], v[4]);
    const float2 sb = cadd(v[2], v[3]);
    const float2 db = csub(v[2], v[3]);
    const float2 a1 = make_float2(v[0].x + c1 * sa.x + c2 * sb.x, v[0].y + c1 * sa.y + c2 * sb.y);
    const float2 a2 = make_float2(v[0].x + c2 * sa.x + c1 * sb.x, v[0].y + c2 * sa.y + c1 * sb.y);
    const float2 b1 = mul_i<INV>(make_float2(s1 * da.x + s2 * db.x, s1 * da.y + s2 * db.y));
    const float2 b2 = mul_i<INV>(make_float2(s2 * da.x - s1 * db.x, s2 * da.y - s1 * db.y));
    v[0] = make_float2(v[0].x + sa.x + sb.x, v[0].y + sa.y + sb.y);
    v[1] = cadd(a1, b1);
    v[4] = csub(a1, b1);
    v[2] = cadd(a2, b2);
    v[3] = csub(a2, b2);
  }
};

// --------------------------------------------------------------------------------------
// one Stockham stage on a line in shared memory.  Every thread of the block must call
// it (it synchronises the block); threads with t >= threads of the plan only take part
// in the barriers.
// --------------------------------------------------------------------------------------
template <int R, bool INV>
__device__ __forceinline__ void fft_stage(float2* line, int n, int ns, int t, int nthreads,
                                          const float2* __restrict__ tw) {
  constexpr int MAXB = (kValuesPerThread + R - 1) / R;
  const int nb = n / R;
  const int tstride = n / (ns * R);  // table step for r * k = 1
  float2 v[MAXB][R];
  int dst[MAXB];
#pragma unroll
  for (int b = 0; b < MAXB; ++b) {
    const int j = t + b * nthreads;
    dst[b] = -1;
    if (t < nthreads && j < nb) {
      const int k = j % ns;
#pragma unroll
      for (int r = 0; r < R; ++r) v[b][r] = line[j + r * nb];
      if (ns > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          float2 w = __ldg(&tw[r * k * tstride]);
          if (INV) w.y = -w.y;
          v[b][r] = cmul(v[b][r], w);
        }
      }
      Dft<R, INV>::run(v[b]);
      dst[b] = (j - k) * R + k;
    }
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < MAXB; ++b) {
    if (dst[b] >= 0) {
#pragma unroll
      for (int r = 0; r < R; ++r) line[dst[b] + r * ns] = v[b][r];
    }
  }
  __syncthreads();
}

// Runtime-plan path: one non-inlined function per radix keeps each stage's register
// allocation separate (a single inlined switch over six radices spills).
template <int R, bool INV>
__device__ __noinline__ void fft_stage_rt(float2* line, int n, int ns, int t, int nthreads,
                                          const float2* __restrict__ tw) {
  fft_stage<R, INV>(line, n, ns, t, nthreads, tw);
}

template <bool INV>
__device__ __forceinline__ void line_fft_rt(float2* line, const LinePlan& p, int t) {
  int ns = 1;
  for (int s = 0; s < p.nstages; ++s) {
    const int R = plan_radix(p, s);
    switch (R) {
      case 16: fft_stage_rt<16, INV>(line, p.n, ns, t, p.threads, p.tw); break;
      case 8: fft_stage_rt<8, INV>(line, p.n, ns, t, p.threads, p.tw); break;
      case 4: fft_stage_rt<4, INV>(line, p.n, ns, t, p.threads, p.tw); break;
      case 2: fft_stage_rt<2, INV>(line, p.n, ns, t, p.threads, p.tw); break;
      case 3: fft_stage_rt<3, INV>(line, p.n, ns, t, p.threads, p.tw); break;
      case 5: fft_stage_rt<5, INV>(line, p.n, ns, t, p.threads, p.tw); break;
      default: break;
    }
    ns *= R;
  }
}

// Compile-time plan (same radix rule as the host planner): the power-of-two part in
// ceil(a/4) balanced stages, then the factors 3 and 5.
__host__ __device__ constexpr int ct_pow2_bits(int n) {
  int a = 0;
  while (n % 2 == 0) { n /= 2; ++a; }
  return a;
}
__host__ __device__ constexpr int ct_count(int n, int f) {
  int c = 0;
  while (n % f == 0) { n /= f; ++c; }
  return c;
}
__host__ __device__ constexpr int ct_nstages(int n) {
  return (ct_pow2_bits(n) + 3) / 4 + ct_count(n, 3) + ct_count(n, 5);
}
__host__ __device__ constexpr int ct_radix(int n, int s) {
  const int a = ct_pow2_bits(n);
  const int p2 = (a + 3) / 4;
  if (s < p2) {
    int left = a;
    for (int i = 0; i < p2; ++i) {
      const int bits = (left + (p2 - i) - 1) / (p2 - i);
      if (i == s) return 1 << bits;
      left -= bits;
    }
  }
  return (s - p2 < ct_count(n, 3)) ? 3 : 5;
}

template <int N, bool INV, int S = 0, int NS = 1>
__device__ __forceinline__ void line_fft_ct(float2* line, const float2* __restrict__ tw, int t) {
  if constexpr (S < ct_nstages(N)) {
    constexpr int R = ct_radix(N, S);
    fft_stage<R, INV>(line, N, NS, t, (N + kValuesPerThread - 1) / kValuesPerThread, tw);
    line_fft_ct<N, INV, S + 1, NS * R>(line, tw, t);
  }
}

// Transform one line in place.  N > 0 selects the compile-time plan for length N (which
// must equal p.n); N == 0 runs the runtime plan.  `t` is the thread's index within its
// line (t >= p.threads for threads that own no line).  Block-synchronising: every thread
// of the block must call it.
template <int N, bool INV>
__device__ __forceinline__ void line_fft(float2* line, const LinePlan& p, int t) {
  if constexpr (N > 0) {
    line_fft_ct<N, INV>(line, p.tw, t);
  } else {
    line_fft_rt<INV>(line, p, t);
  }
}

// shared-memory pitch of a line: odd in float2 units so column-tile transposes are
// bank-conflict free
__host__ __device__ __forceinline__ int line_pitch(int n) { return n | 1; }

// column tile width of the tiled scratch layout [frame][tile][row][kTile]
constexpr int kTile = 16;
__host__ __device__ __forceinline__ int num_tiles(int width) { return (width + kTile - 1) / kTile; }

}  // namespace ptx
