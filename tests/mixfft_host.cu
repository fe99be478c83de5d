// Host run of the mixed-radix two-step FFT steps (ptx_mixfft.cuh) against an FP64 DFT.
//
// For each length N the B "threads" of step 1 and the A "threads" of step 2 run one after
// the other, in both buffer layouts (lines one after another; C = 8 lines interleaved) and
// both signs of each direction.  Prints one line per length: N, A, B, the space -> frequency
// and frequency -> space errors (relative RMS, worst of the layouts and signs), and the
// in-register DFT error of the factors A and B.
#include <cmath>
#include <complex>
#include <cstdio>
#include <random>
#include <vector>

#include "ptx_mixfft.cuh"

using cd = std::complex<double>;
using namespace ptx::mix;

static std::vector<cd> dft(const std::vector<cd>& x, int sign) {
  const int n = static_cast<int>(x.size());
  std::vector<cd> out(n);
  for (int k = 0; k < n; ++k) {
    cd acc = 0;
    for (int j = 0; j < n; ++j) {
      const long m = (static_cast<long>(j) * k) % n;
      const double a = sign * 2.0 * M_PI * static_cast<double>(m) / n;
      acc += x[j] * cd(std::cos(a), std::sin(a));
    }
    out[k] = acc;
  }
  return out;
}

static double rel(const std::vector<cd>& a, const std::vector<cd>& b) {
  double num = 0, den = 0;
  for (size_t i = 0; i < a.size(); ++i) {
    num += std::norm(a[i] - b[i]);
    den += std::norm(b[i]);
  }
  return std::sqrt(num / den);
}

template <int M>
static double dft_err(std::mt19937& rng) {
  std::normal_distribution<float> nd;
  std::vector<cd> x(M);
  float2 v[M];
  for (int i = 0; i < M; ++i) {
    v[i] = make_float2(nd(rng), nd(rng));
    x[i] = cd(v[i].x, v[i].y);
  }
  Dft<M, false>::run(v);
  std::vector<cd> got(M);
  for (int i = 0; i < M; ++i) got[i] = cd(v[i].x, v[i].y);
  return rel(got, dft(x, -1));
}

template <int N, int RS, int CS>
static void run_layout(std::mt19937& rng, int c, double* efwd, double* einv) {
  using S = Shape<N>;
  std::normal_distribution<float> nd;
  std::vector<float2> twt(N), twi(N);
  for (int t = 0; t < S::B; ++t) {
    for (int u = 0; u < S::A; ++u) {
      const double a = -2.0 * M_PI * static_cast<double>(t * u) / N;
      const float2 w = make_float2(static_cast<float>(std::cos(a)), static_cast<float>(std::sin(a)));
      twt[u * S::B + t] = w;
      twi[t * S::A + u] = w;
    }
  }
  std::vector<float2> buf(static_cast<size_t>(S::A) * RS + static_cast<size_t>(S::B) * CS + 64);
  float2* line = buf.data() + c;
  std::vector<cd> x(N);
  std::vector<float2> xf(N);
  for (int i = 0; i < N; ++i) {
    xf[i] = make_float2(nd(rng), nd(rng));
    x[i] = cd(xf[i].x, xf[i].y);
  }
  // forward
  for (int t = 0; t < S::B; ++t) {
    float2 y[S::A];
    for (int j = 0; j < S::A; ++j) y[j] = xf[t + S::B * j];
    fwd_step1<N, RS, CS>(y, line, t, twt.data());
  }
  std::vector<cd> got(N);
  for (int u = 0; u < S::A; ++u) {
    float2 z[S::B];
    fwd_step2<N, RS, CS>(z, line, u);
    for (int k = 0; k < S::B; ++k) got[u + S::A * k] = cd(z[k].x, z[k].y);
  }
  const std::vector<cd> ref = dft(x, -1);
  *efwd = rel(got, ref);
  // inverse of the reference spectrum, rounded to FP32
  for (int u = 0; u < S::A; ++u) {
    float2 z[S::B];
    for (int k = 0; k < S::B; ++k) {
      const cd v = ref[u + S::A * k];
      z[k] = make_float2(static_cast<float>(v.real()), static_cast<float>(v.imag()));
    }
    inv_step1<N, RS, CS>(z, line, u, twi.data());
  }
  std::vector<cd> back(N), want(N);
  for (int t = 0; t < S::B; ++t) {
    float2 y[S::A];
    inv_step2<N, RS, CS>(y, line, t);
    for (int j = 0; j < S::A; ++j) back[t + S::B * j] = cd(y[j].x, y[j].y);
  }
  for (int i = 0; i < N; ++i) want[i] = x[i] * static_cast<double>(N);
  *einv = rel(back, want);
  // the opposite signs: space -> frequency with exp(+i), frequency -> space with exp(-i)
  for (int t = 0; t < S::B; ++t) {
    float2 y[S::A];
    for (int j = 0; j < S::A; ++j) y[j] = xf[t + S::B * j];
    fwd_step1<N, RS, CS, true>(y, line, t, twt.data());
  }
  for (int u = 0; u < S::A; ++u) {
    float2 z[S::B];
    fwd_step2<N, RS, CS, true>(z, line, u);
    for (int k = 0; k < S::B; ++k) got[u + S::A * k] = cd(z[k].x, z[k].y);
  }
  *efwd = std::max(*efwd, rel(got, dft(x, +1)));
  for (int u = 0; u < S::A; ++u) {
    float2 z[S::B];
    for (int k = 0; k < S::B; ++k) z[k] = xf[u + S::A * k];
    inv_step1<N, RS, CS, false>(z, line, u, twi.data());
  }
  const std::vector<cd> fw = dft(x, -1);
  for (int t = 0; t < S::B; ++t) {
    float2 y[S::A];
    inv_step2<N, RS, CS, false>(y, line, t);
    for (int j = 0; j < S::A; ++j) back[t + S::B * j] = cd(y[j].x, y[j].y);
  }
  *einv = std::max(*einv, rel(back, fw));
}

template <int N>
static void run_one(std::mt19937& rng) {
  using S = Shape<N>;
  constexpr int C = 8;
  double f1, i1, f2, i2;
  run_layout<N, S::P, 1>(rng, 0, &f1, &i1);
  run_layout<N, S::B * C, C>(rng, 5, &f2, &i2);
  const double ea = dft_err<S::A>(rng), eb = dft_err<S::B>(rng);
  std::printf("%d %d %d %.3e %.3e %.3e %.3e\n", N, S::A, S::B, std::max(f1, f2), std::max(i1, i2), ea, eb);
}

template <int... Ns>
static void run_all(std::mt19937& rng) {
  (run_one<Ns>(rng), ...);
}

int main() {
  std::mt19937 rng(7);
  run_all<4, 5, 6, 8, 9, 10, 12, 15, 16, 18, 20, 24, 25, 27, 30, 32, 36, 40, 45, 48, 50, 54, 60, 64, 72, 75, 80, 81, 90, 96,
          100, 108, 120, 125, 128, 135, 144, 150, 160, 162, 180, 192, 200, 216, 225, 240, 243, 250, 256, 270, 288, 300, 320,
          324, 360, 375, 384, 400, 405, 432, 450, 480, 486, 500, 512, 540, 576, 600, 625, 640, 648, 675, 720, 729,
          750, 768, 800, 810, 864, 900, 960, 972, 1000, 1024>(rng);
  return 0;
}
