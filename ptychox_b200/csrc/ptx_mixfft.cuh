// Register-resident two-step FFT for {2,3,5}-smooth lengths that are not powers of two.
//
// A line of length N = A * B (A <= B) is held by B threads and transformed with one exchange
// through shared memory:
//   space layout:     thread t < B owns x[t + B j], j < A;
//   frequency layout: thread u < A owns X[u + A k], k < B.
// Forward (space -> frequency), from n = t + B j, k' = u + A k:
//   X[u + A k] = sum_t W_B^{t k} [ W_N^{t u} sum_j x[t + B j] W_A^{j u} ]
//   1. thread t: DFT-A over its j (registers), twiddle by W_N^{t u}, write row u, column t;
//   2. (after a barrier) thread u: reads row u (B values), DFT-B over t (registers).
// Inverse (frequency -> space), the same steps reversed with conjugate roots:
//   x[t + B j] = sum_u W_A^{-j u} [ W_N^{-t u} sum_k X[u + A k] W_B^{-t k} ]
// so a forward transform, a pointwise step in the frequency layout and an inverse transform
// return the data to the layout it came in.  Neither transform is normalised.
//
// The in-register DFTs of A and B points are Cooley-Tukey compositions of radix 2, 3, 4 and
// 5 kernels; their twiddles are constants, cos and sin of 2 pi m / n evaluated at compile time
// from their Taylor series after an exact reduction of the angle to [-pi/4, pi/4].  The
// inter-step twiddles W_N^{t u} come from tables computed in FP64 on the host.  The steps are
// per-thread __host__ __device__ functions (the caller places the barriers between them), so
// the CPU can run them thread by thread.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

namespace ptx {
namespace mix {

#define PTX_MIX_HD __host__ __device__ __forceinline__

// ---- compile-time roots of unity -----------------------------------------------------

constexpr double kHalfPi = 1.57079632679489661923132169163975144;

constexpr double taylor_sin(double x) {  // |x| <= pi/4: 13 terms reach double precision
  double x2 = x * x, term = x, sum = x;
  for (int k = 1; k < 13; ++k) {
    term *= -x2 / ((2.0 * k) * (2.0 * k + 1.0));
    sum += term;
  }
  return sum;
}

constexpr double taylor_cos(double x) {
  double x2 = x * x, term = 1.0, sum = 1.0;
  for (int k = 1; k < 13; ++k) {
    term *= -x2 / ((2.0 * k - 1.0) * (2.0 * k));
    sum += term;
  }
  return sum;
}

// cos and sin of 2 pi m / n: with q the nearest multiple of a quarter turn, 2 pi m / n =
// q pi / 2 + x, x = (pi / 2) (4 m - q n) / n exactly in integers, |x| <= pi / 4.
constexpr double cos_turn(long m, long n) {
  const long mm = ((m % n) + n) % n;
  const long q = (8 * mm + n) / (2 * n);  // round(4 mm / n)
  const double x = kHalfPi * static_cast<double>(4 * mm - q * n) / static_cast<double>(n);
  switch (q & 3) {
    case 0: return taylor_cos(x);
    case 1: return -taylor_sin(x);
    case 2: return -taylor_cos(x);
    default: return taylor_sin(x);
  }
}
constexpr double sin_turn(long m, long n) {
  const long mm = ((m % n) + n) % n;
  const long q = (8 * mm + n) / (2 * n);
  const double x = kHalfPi * static_cast<double>(4 * mm - q * n) / static_cast<double>(n);
  switch (q & 3) {
    case 0: return taylor_sin(x);
    case 1: return taylor_cos(x);
    case 2: return -taylor_sin(x);
    default: return -taylor_cos(x);
  }
}

template <int N, int M>
struct Root {
  static constexpr int m = ((M % N) + N) % N;
  static constexpr float c = static_cast<float>(cos_turn(m, N));
  static constexpr float s = static_cast<float>(sin_turn(m, N));
};

// ---- complex helpers (host and device) ------------------------------------------------

// Complex add / subtract and real-scalar FMA as single packed FP32x2 instructions on sm_100
// (a - b as fma(b, -1, a), which rounds once exactly like the subtraction); plain FP32 on
// the host.
PTX_MIX_HD float2 add(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  return __fadd2_rn(a, b);
#else
  return make_float2(a.x + b.x, a.y + b.y);
#endif
}
PTX_MIX_HD float2 sub(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  return __ffma2_rn(b, make_float2(-1.f, -1.f), a);
#else
  return make_float2(a.x - b.x, a.y - b.y);
#endif
}
// s * b + a for real s
PTX_MIX_HD float2 axpy(float s, float2 b, float2 a) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  return __ffma2_rn(make_float2(s, s), b, a);
#else
  return make_float2(fmaf(s, b.x, a.x), fmaf(s, b.y, a.y));
#endif
}
// s * b for real s
PTX_MIX_HD float2 scale(float s, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  return __fmul2_rn(make_float2(s, s), b);
#else
  return make_float2(s * b.x, s * b.y);
#endif
}
PTX_MIX_HD float2 mul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
PTX_MIX_HD float2 mulc(float2 a, float2 b) {  // a * conj(b)
  return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
// z * (-i) forward, z * (+i) inverse
template <bool INV>
PTX_MIX_HD float2 rot(float2 z) {
  return INV ? make_float2(-z.y, z.x) : make_float2(z.y, -z.x);
}

// z * exp(-+ 2 pi i M / N) with M, N compile-time; exact quarter turns avoid multiplies.
template <int N, int M, bool INV>
PTX_MIX_HD float2 twiddle(float2 z) {
  constexpr int m = ((M % N) + N) % N;
  if constexpr (m == 0) {
    return z;
  } else if constexpr (4 * m == N) {
    return rot<INV>(z);
  } else if constexpr (2 * m == N) {
    return make_float2(-z.x, -z.y);
  } else if constexpr (4 * m == 3 * N) {
    return rot<!INV>(z);
  } else {
    constexpr float c = Root<N, m>::c;
    constexpr float s = INV ? Root<N, m>::s : -Root<N, m>::s;
    return make_float2(fmaf(z.x, c, -z.y * s), fmaf(z.x, s, z.y * c));
  }
}

template <int I, int E, class F>
PTX_MIX_HD void static_for(F&& f) {
  if constexpr (I < E) {
    f(std::integral_constant<int, I>{});
    static_for<I + 1, E>(f);
  }
}

// ---- in-register DFTs: natural order in and out ----------------------------------------

template <int N, bool INV>
struct Dft;

template <bool INV>
struct Dft<1, INV> {
  PTX_MIX_HD static void run(float2*) {}
};

template <bool INV>
struct Dft<2, INV> {
  PTX_MIX_HD static void run(float2* v) {
    const float2 a = v[0], b = v[1];
    v[0] = add(a, b);
    v[1] = sub(a, b);
  }
};

template <bool INV>
struct Dft<3, INV> {
  PTX_MIX_HD static void run(float2* v) {
    constexpr float r3 = 0.86602540378443865f;  // sin(2 pi / 3)
    const float2 t = add(v[1], v[2]);
    const float2 d = rot<INV>(sub(v[1], v[2]));
    const float2 m = axpy(-0.5f, t, v[0]);
    v[0] = add(v[0], t);
    v[1] = axpy(r3, d, m);
    v[2] = axpy(-r3, d, m);
  }
};

template <bool INV>
struct Dft<4, INV> {
  PTX_MIX_HD static void run(float2* v) {
    const float2 t0 = add(v[0], v[2]);
    const float2 t1 = sub(v[0], v[2]);
    const float2 t2 = add(v[1], v[3]);
    const float2 t3 = rot<INV>(sub(v[1], v[3]));
    v[0] = add(t0, t2);
    v[1] = add(t1, t3);
    v[2] = sub(t0, t2);
    v[3] = sub(t1, t3);
  }
};

template <bool INV>
struct Dft<5, INV> {
  PTX_MIX_HD static void run(float2* v) {
    constexpr float c1 = 0.30901699437494742f;   // cos(2 pi / 5)
    constexpr float c2 = -0.80901699437494742f;  // cos(4 pi / 5)
    constexpr float s1 = 0.95105651629515357f;   // sin(2 pi / 5)
    constexpr float s2 = 0.58778525229247313f;   // sin(4 pi / 5)
    const float2 sa = add(v[1], v[4]);
    const float2 da = sub(v[1], v[4]);
    const float2 sb = add(v[2], v[3]);
    const float2 db = sub(v[2], v[3]);
    const float2 a1 = axpy(c2, sb, axpy(c1, sa, v[0]));
    const float2 a2 = axpy(c1, sb, axpy(c2, sa, v[0]));
    const float2 b1 = rot<INV>(axpy(s2, db, scale(s1, da)));
    const float2 b2 = rot<INV>(axpy(-s1, db, scale(s2, da)));
    v[0] = add(v[0], add(sa, sb));
    v[1] = add(a1, b1);
    v[4] = sub(a1, b1);
    v[2] = add(a2, b2);
    v[3] = sub(a2, b2);
  }
};

// first factor of a composite length: 4, then 2, 3, 5
constexpr int first_factor(int n) {
  return (n % 4 == 0 && n > 4) ? 4 : (n % 2 == 0) ? 2 : (n % 3 == 0) ? 3 : 5;
}

// Composite length N = F * R by one Cooley-Tukey step, n = n1 + F n2, k = R k1 + k2:
//   X[R k1 + k2] = sum_n1 W_F^{n1 k1} W_N^{n1 k2} sum_n2 x[n1 + F n2] W_R^{n2 k2}.
template <int N, bool INV>
struct Dft {
  static_assert(N > 5, "composite lengths only");
  static constexpr int F = first_factor(N);
  static constexpr int R = N / F;
  PTX_MIX_HD static void run(float2* v) {
    float2 y[N];
    static_for<0, F>([&](auto n1c) {
      constexpr int n1 = decltype(n1c)::value;
      float2 col[R];
#pragma unroll
      for (int n2 = 0; n2 < R; ++n2) col[n2] = v[n1 + F * n2];
      Dft<R, INV>::run(col);
      static_for<0, R>([&](auto k2c) {
        constexpr int k2 = decltype(k2c)::value;
        y[n1 * R + k2] = twiddle<N, n1 * k2, INV>(col[k2]);
      });
    });
#pragma unroll
    for (int k2 = 0; k2 < R; ++k2) {
      float2 row[F];
#pragma unroll
      for (int n1 = 0; n1 < F; ++n1) row[n1] = y[n1 * R + k2];
      Dft<F, INV>::run(row);
#pragma unroll
      for (int k1 = 0; k1 < F; ++k1) v[R * k1 + k2] = row[k1];
    }
  }
};

// ---- the two-step line transform -------------------------------------------------------

constexpr bool smooth(int n) {
  if (n <= 0) return false;
  while (n % 2 == 0) n /= 2;
  while (n % 3 == 0) n /= 3;
  while (n % 5 == 0) n /= 5;
  return n == 1;
}

// The split N = A * B with both factors smooth and A <= B, B as small as possible (B is the
// number of threads per line); 0 when N is not smooth.
constexpr int split_b(int n) {
  for (int b = 1; b <= n; ++b) {
    if (n % b == 0 && b >= n / b && smooth(b) && smooth(n / b)) return b;
  }
  return 0;
}

template <int N>
struct Shape {
  static constexpr int B = split_b(N);           // space layout: threads t < B, A values each
  static constexpr int A = N / B;                // frequency layout: threads u < A, B values each
  static constexpr int P = (B % 2) ? B : B + 1;  // odd row pitch of a line's exchange buffer
  static_assert(B > 0 && A * B == N, "N must be {2,3,5}-smooth");
};

// The exchange buffer holds one line as an A x B array, element (u, t) at buf[u * RS + t * CS]:
// RS = P, CS = 1 for lines stored one after another; RS = B * C, CS = C for C lines interleaved
// element by element (the column kernels, whose neighbouring threads own neighbouring lines).
// Twiddle tables, both of N entries: twt[u * B + t] = twi[t * A + u] = exp(-2 pi i t u / N)
// (one per layout, so each step reads consecutive entries from consecutive threads).

// The steps below take the sign of the transform as PLUS: exp(-2 pi i ...) for PLUS = false
// (the forward DFT), exp(+2 pi i ...) for PLUS = true (the unnormalised inverse).  "fwd" steps
// map the space layout to the frequency layout, "inv" steps map back; both exist in both
// signs (a forward transform after an inverse one, as the FPM column pass needs, is an "inv"
// pair with PLUS = false).

// Space -> frequency, step 1, thread t < B: DFT-A of x[t + B j] (in y, j < A), twiddle,
// store row u.
template <int N, int RS, int CS, bool PLUS = false>
PTX_MIX_HD void fwd_step1(float2 (&y)[Shape<N>::A], float2* buf, int t, const float2* twt) {
  using S = Shape<N>;
  Dft<S::A, PLUS>::run(y);
  buf[t * CS] = y[0];
#pragma unroll
  for (int u = 1; u < S::A; ++u) {
    const float2 w = twt[u * S::B + t];
    buf[u * RS + t * CS] = PLUS ? mulc(y[u], w) : mul(y[u], w);
  }
}

// Space -> frequency, step 2, thread u < A: DFT-B over row u -> z[k] = X[u + A k].
template <int N, int RS, int CS, bool PLUS = false>
PTX_MIX_HD void fwd_step2(float2 (&z)[Shape<N>::B], const float2* buf, int u) {
  using S = Shape<N>;
#pragma unroll
  for (int k = 0; k < S::B; ++k) z[k] = buf[u * RS + k * CS];
  Dft<S::B, PLUS>::run(z);
}

// Frequency -> space, step 1, thread u < A: DFT-B of X[u + A k] (in z), twiddle, store row u.
template <int N, int RS, int CS, bool PLUS = true>
PTX_MIX_HD void inv_step1(float2 (&z)[Shape<N>::B], float2* buf, int u, const float2* twi) {
  using S = Shape<N>;
  Dft<S::B, PLUS>::run(z);
  buf[u * RS] = z[0];
#pragma unroll
  for (int t = 1; t < S::B; ++t) {
    const float2 w = twi[t * S::A + u];
    buf[u * RS + t * CS] = PLUS ? mulc(z[t], w) : mul(z[t], w);
  }
}

// Frequency -> space, step 2, thread t < B: DFT-A over column t -> y[j] = x[t + B j].
template <int N, int RS, int CS, bool PLUS = true>
PTX_MIX_HD void inv_step2(float2 (&y)[Shape<N>::A], const float2* buf, int t) {
  using S = Shape<N>;
#pragma unroll
  for (int u = 0; u < S::A; ++u) y[u] = buf[u * RS + t * CS];
  Dft<S::A, PLUS>::run(y);
}

}  // namespace mix
}  // namespace ptx
