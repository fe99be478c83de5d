// Host check of the two-line packed FFT (ptx_pairfft.cuh): for every supported size and
// both directions, two seeded random lines go through the per-thread steps exactly as the
// kernels run them (step 1 per thread, the shared-memory exchange, step 2) and are compared
// with an FP64 DFT.  Prints one line per size: N, forward and inverse relative L2 error.
#include <cstdio>
#include <cmath>
#include <vector>
#include <random>
#include "ptx_pairfft.cuh"
using namespace ptx;
template <int N, bool INV>
double run_one(unsigned seed) {
  using S = RegShape<N>;
  std::mt19937 g(seed);
  std::uniform_real_distribution<float> U(-1, 1);
  std::vector<float2> A(N), B(N);
  for (int i = 0; i < N; ++i) { A[i] = make_float2(U(g), U(g)); B[i] = make_float2(U(g), U(g)); }
  std::vector<float4> tw4(N);
  for (int m = 0; m < N; ++m) {
    double a = -2.0 * M_PI * m / N;
    float c = (float)std::cos(a), s = (float)std::sin(a);
    tw4[m] = make_float4(c, c, s, s);
  }
  std::vector<float4> buf(S::BUF);
  std::vector<std::vector<CPair>> V(S::T, std::vector<CPair>(S::N1));
  for (int t = 0; t < S::T; ++t) {
    CPair v[S::N1];
    for (int j = 0; j < S::N1; ++j) { int c = t + S::T * j; v[j] = {make_float2(A[c].x, B[c].x), make_float2(A[c].y, B[c].y)}; }
    pair_fft_step1<N, INV>(v, t, tw4.data());
    for (int k1 = 0; k1 < S::N1; ++k1) buf[k1 * S::RP + t] = pack4(v[k1]);
  }
  double err = 0, ref = 0;
  for (int t = 0; t < S::T; ++t) {
    CPair v[S::N1];
    pair_fft_step2_load<N, INV>(v, buf.data(), t);
    for (int j = 0; j < S::N1; ++j) {
      int k = t + S::T * j;
      for (int line = 0; line < 2; ++line) {
        const std::vector<float2>& X = line ? B : A;
        double sr = 0, si = 0;
        for (int n = 0; n < N; ++n) {
          double a = (INV ? 2.0 : -2.0) * M_PI * (double)((long long)n * k % N) / N;
          sr += X[n].x * std::cos(a) - X[n].y * std::sin(a);
          si += X[n].x * std::sin(a) + X[n].y * std::cos(a);
        }
        double gr = line ? v[j].re.y : v[j].re.x, gi = line ? v[j].im.y : v[j].im.x;
        err += (gr - sr) * (gr - sr) + (gi - si) * (gi - si);
        ref += sr * sr + si * si;
      }
    }
  }
  return std::sqrt(err / ref);
}
template <int N> void both() {
  printf("%d %.6e %.6e\n", N, run_one<N, false>(N), run_one<N, true>(N + 1));
}
int main() { both<4>(); both<8>(); both<16>(); both<32>(); both<64>(); both<128>(); both<256>(); both<512>(); both<1024>(); }
