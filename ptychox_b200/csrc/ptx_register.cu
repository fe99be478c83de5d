// Sub-pixel registration: the matrix-multiply DFT refinement of dftregistration.
//
// Reference: matlab/Examples/Near-field Ptychography/+misc/dftregistration.m:102-121 (the
// usfac > 2 branch) with its helper dftups (:150-185): around an initial estimate
// (R_row, R_col) / usfac of the shift, the cross-power spectrum Q = buf2ft .* conj(buf1ft)
// (rows x cols) is inverse-transformed onto an n_out x n_out patch of the grid upsampled by
// usfac (n_out = ceil(1.5 usfac)), the patch's origin at dftshift = fix(n_out / 2):
//
//   out[r][c] = sum_m sum_n kr[r][m] Q[m][n] kc[n][c]
//   kc[n][c]  = exp(-2 pi i fc(n) (c - coff) / (cols usfac)),  coff = dftshift - R_col
//   kr[r][m]  = exp(-2 pi i (r - roff) fr(m) / (rows usfac)),  roff = dftshift - R_row
//
// fr, fc the centred frequencies (k for k < ceil(L/2), else k - L).  CC = conj(out); its
// peak |CC| (the first maximum in column-major order, as MATLAB's find(..., 1, 'first'))
// gives the refined shift.
//
// Both products have the form Out[i][j] = sum_k A[i][k] exp(-2 pi i f(k) (j - off) / (L usfac)),
// so one kernel does both, writing its result transposed:
//   stage 1: A = Q [rows][cols] (k = n)    -> T [n_out][rows]  (T[c][m])
//   stage 2: A = T [n_out][rows] (k = m)   -> out [n_out][n_out] (out[r][c])
// The twiddles are generated in the tiles from the exact integer phase
// f(k) (j - off) mod (L usfac), so no angle grows beyond one turn before the sine.
// Twiddles, sums and the intermediate T are FP64: at usfac = 600 neighbouring grid points
// of a smooth correlation peak differ in |CC| by parts in 1e5 and less, below what FP32
// sums over thousands of terms resolve (the input spectrum stays FP32).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "ptx_internal.h"

namespace ptx {
namespace {

constexpr int kRegTile = 64;   // output tile (i and j)
constexpr int kRegK = 16;      // k per shared-memory stage
constexpr int kRegThreads = 256;

__device__ __forceinline__ int centred_freq(int k, int len) { return k < (len + 1) / 2 ? k : k - len; }

// Out^T[b][j][i] = sum_k A[b][i][k] W(k, j) for i < ni, j < nj, k < len;
// W(k, j) = exp(-2 pi i f(k) (j - off_b) / (len usfac)), off_b = dftshift - center[b].
template <typename TIn>
__global__ void __launch_bounds__(kRegThreads) reg_twiddle_gemm_kernel(
    const TIn* __restrict__ a, int ni, int len, int nj, int usfac, int dftshift,
    const int* __restrict__ center, double2* __restrict__ out) {
  __shared__ double2 as[kRegTile][kRegK + 1];
  __shared__ double2 ws[kRegK][kRegTile + 1];
  const int b = blockIdx.z;
  const int i0 = blockIdx.y * kRegTile, j0 = blockIdx.x * kRegTile;
  const int tid = threadIdx.x;
  const int ti = tid / 16, tj = tid % 16;  // thread owns i = i0 + ti + 16 u, j = j0 + tj + 16 v
  const long long period = (long long)len * usfac;
  const int off = dftshift - center[b];
  const TIn* ab = a + (size_t)b * ni * len;
  double2 acc[4][4];
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) acc[u][v] = make_double2(0.0, 0.0);
  for (int k0 = 0; k0 < len; k0 += kRegK) {
    for (int e = tid; e < kRegTile * kRegK; e += kRegThreads) {
      const int ii = e / kRegK, kk = e % kRegK;
      const int i = i0 + ii, k = k0 + kk;
      double2 v = make_double2(0.0, 0.0);
      if (i < ni && k < len) {
        const TIn x = ab[(size_t)i * len + k];
        v = make_double2(x.x, x.y);
      }
      as[ii][kk] = v;
    }
    for (int e = tid; e < kRegK * kRegTile; e += kRegThreads) {
      const int kk = e / kRegTile, jj = e % kRegTile;
      const int k = k0 + kk, j = j0 + jj;
      double2 w = make_double2(0.0, 0.0);
      if (k < len && j < nj) {
        long long p = (long long)centred_freq(k, len) * (long long)(j - off) % period;
        if (p < 0) p += period;
        double sn, cs;
        sincospi(2.0 * static_cast<double>(p) / static_cast<double>(period), &sn, &cs);
        w = make_double2(cs, -sn);
      }
      ws[kk][jj] = w;
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < kRegK; ++kk) {
      double2 av[4], wv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) av[u] = as[ti + 16 * u][kk];
#pragma unroll
      for (int v = 0; v < 4; ++v) wv[v] = ws[kk][tj + 16 * v];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          acc[u][v].x = fma(av[u].x, wv[v].x, fma(-av[u].y, wv[v].y, acc[u][v].x));
          acc[u][v].y = fma(av[u].x, wv[v].y, fma(av[u].y, wv[v].x, acc[u][v].y));
        }
    }
    __syncthreads();
  }
  double2* ob = out + (size_t)b * nj * ni;
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int i = i0 + ti + 16 * u, j = j0 + tj + 16 * v;
      if (i < ni && j < nj) ob[(size_t)j * ni + i] = acc[u][v];
    }
}

// Peak of |out[b]| (n x n, row-major out[r][c]) in column-major order, first maximum on ties;
// writes (r, c) and conj(out[r][c]) (= CC at the peak).
__global__ void __launch_bounds__(1024) reg_peak_kernel(const double2* __restrict__ out, int n,
                                                         int* __restrict__ peak_rc, double2* __restrict__ peak_cc) {
  __shared__ double sv[32];
  __shared__ long long si[32];
  const int b = blockIdx.x;
  const double2* ob = out + (size_t)b * n * n;
  const long long total = (long long)n * n;
  double best = -1.0;
  long long bi = 0;
  for (long long l = threadIdx.x; l < total; l += blockDim.x) {
    const int r = static_cast<int>(l % n), c = static_cast<int>(l / n);
    const double2 z = ob[(size_t)r * n + c];
    const double m = z.x * z.x + z.y * z.y;
    if (m > best) {  // l increases per thread, so the first maximum of the thread is kept
      best = m;
      bi = l;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, best, o);
    const long long oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (ov > best || (ov == best && oi < bi)) {
      best = ov;
      bi = oi;
    }
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    sv[w] = best;
    si[w] = bi;
  }
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    best = lane < nw ? sv[lane] : -2.0;
    bi = lane < nw ? si[lane] : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, best, o);
      const long long oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ov > best || (ov == best && oi < bi)) {
        best = ov;
        bi = oi;
      }
    }
    if (lane == 0) {
      const int r = static_cast<int>(bi % n), c = static_cast<int>(bi / n);
      const double2 z = ob[(size_t)r * n + c];
      peak_rc[2 * b] = r;
      peak_rc[2 * b + 1] = c;
      peak_cc[b] = make_double2(z.x, -z.y);
    }
  }
}

int reg_out_size(int usfac) { return (3 * usfac + 1) / 2; }  // ceil(1.5 usfac)

}  // namespace
}  // namespace ptx

using namespace ptx;

extern "C" {

size_t ptx_reg_workspace_bytes(int batch, int rows, int cols, int usfac) {
  if (batch <= 0 || rows <= 0 || cols <= 0 || usfac <= 2) return 0;
  const size_t n = static_cast<size_t>(reg_out_size(usfac));
  return sizeof(double2) * (size_t)batch * n * ((size_t)rows + n);
}

int ptx_reg_upsampled_peak(const float* cross_power, int batch, int rows, int cols, int usfac,
                           const int* row_center, const int* col_center, int* peak_rc, double* peak_cc,
                           void* workspace, size_t workspace_bytes, void* stream) {
  if (batch < 0 || rows <= 0 || cols <= 0) return set_error(PTX_ERR_INVALID_ARGUMENT, "non-positive shape");
  if (usfac <= 2 || usfac > 100000) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "usfac must lie in [3, 100000] for the upsampled refinement");
  }
  if (batch == 0) return PTX_OK;
  if (!cross_power || !row_center || !col_center || !peak_rc || !peak_cc || !workspace) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "null pointer argument");
  }
  if ((long long)rows * usfac > (1ll << 30) || (long long)cols * usfac > (1ll << 30)) {
    return set_error(PTX_ERR_UNSUPPORTED_SIZE, "rows or cols times usfac exceeds 2^30");
  }
  const size_t need = ptx_reg_workspace_bytes(batch, rows, cols, usfac);
  if (workspace_bytes < need) {
    return set_error(PTX_ERR_WORKSPACE, "workspace of %zu bytes is smaller than %zu", workspace_bytes, need);
  }
  if (batch > 65535) return set_error(PTX_ERR_UNSUPPORTED_SIZE, "at most 65535 images per call");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int n = reg_out_size(usfac);
  const int dftshift = n / 2;
  double2* t = static_cast<double2*>(workspace);       // [batch][n][rows]
  double2* o = t + (size_t)batch * n * rows;           // [batch][n][n]
  const float2* q = reinterpret_cast<const float2*>(cross_power);
  const int tiles_n = (n + kRegTile - 1) / kRegTile;
  prof_begin(kMiscKernel, s);
  reg_twiddle_gemm_kernel<float2><<<dim3(tiles_n, (rows + kRegTile - 1) / kRegTile, batch), kRegThreads, 0, s>>>(
      q, rows, cols, n, usfac, dftshift, col_center, t);
  prof_end(kMiscKernel, s);
  prof_begin(kMiscKernel, s);
  reg_twiddle_gemm_kernel<double2><<<dim3(tiles_n, tiles_n, batch), kRegThreads, 0, s>>>(t, n, rows, n, usfac,
                                                                                        dftshift, row_center, o);
  prof_end(kMiscKernel, s);
  prof_begin(kMiscKernel, s);
  reg_peak_kernel<<<batch, 1024, 0, s>>>(o, n, peak_rc, reinterpret_cast<double2*>(peak_cc));
  prof_end(kMiscKernel, s);
  return cuda_status(cudaGetLastError(), "ptx_reg_upsampled_peak launch");
}

}  // extern "C"
