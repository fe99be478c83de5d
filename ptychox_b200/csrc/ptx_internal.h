// Host-side internals shared by the translation units of libptychox.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <string>
#include <type_traits>

#include "../../include/ptychox.h"
#include "ptx_fft.cuh"

namespace ptx {

// Record an error message for ptx_last_error() and return `code`.
int set_error(int code, const char* fmt, ...);
// Map a CUDA error to PTX_ERR_CUDA with a message; returns PTX_OK for cudaSuccess.
int cuda_status(cudaError_t e, const char* what);

// Build (or fetch from the per-device cache) the line plan for length n on the current
// device.  Returns PTX_OK or PTX_ERR_UNSUPPORTED_SIZE / PTX_ERR_CUDA.
int get_line_plan(int n, LinePlan* out);
bool size_supported(int n);

// Raise a kernel's dynamic shared memory cap to `bytes` when they come near the 48 KB default
// (which static shared memory also counts against).  Remembered per (device, kernel), so
// repeated calls cost no driver call; ptx_clear_cache forgets it.
int ensure_smem(const void* kernel, int bytes);
void clear_smem_cache();

// Programmatic dependent launch: the sweep kernels are launched with programmatic stream
// serialisation, so a grid is scheduled while the previous grid on the stream drains; each
// such kernel starts with pdl_wait() (griddepcontrol.wait: it returns once the preceding
// grid has completed and its writes are visible), so the order of memory effects is that of
// plain stream order.  Off when the environment sets PTYCHOX_PDL=0 (read once).
bool pdl_enabled();

template <typename... KArgs, typename... Args>
void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args&&... args) {
  if (!pdl_enabled()) {
    kernel<<<grid, block, smem, s>>>(static_cast<KArgs>(args)...);
    return;
  }
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Launch shapes shared by the pass kernels.
struct RowShape {
  int lines;    // lines (rows) per CTA
  int threads;  // threads per CTA
  int smem;     // dynamic shared memory bytes
};
RowShape row_shape(const LinePlan& p, int rows_available);
struct ColShape {
  int cols;     // columns per CTA (a divisor of kTile)
  int threads;
  int smem;
};
ColShape col_shape(const LinePlan& p);


int sm_count();

// Column pass of the conventional operator over `nframes` tiled scratch frames ([tile][row][16],
// ph x pw) whose counts / far fields start at frame `frame0`: forward (column DFT; the fftshifted
// far field, when non-null, and the amplitude) or backward (g F / max(|F|, eps) from the saved
// far field, inverse column DFT into the frames).
int base_cols_pass(bool forward, float2* scratch, int ph, int pw, int frame0, int nframes, float2* far_field,
                   float* amplitude, const float* grad_output, cudaStream_t s);

// Forget the cached device addresses of the allocation-free sweep's scratch array (looked
// up again by its next call on each device).
void clear_noalloc_cache();

// CTAs of `kernel` (launched with `threads` threads and `smem` dynamic shared bytes) that
// the current device holds at once: SMs x resident CTAs per SM, at least 1.  Cached per
// (device, kernel, threads, smem).
int resident_ctas(const void* kernel, int threads, int smem);

// Grid of a persistent pass over `units` work units: one wave of resident CTAs, or, when
// ptx_set_units_per_cta(k > 0) is in force, enough CTAs that none takes more than k units.
int persistent_grid(const void* kernel, int threads, int smem, long long units);
// The bound in force for launches of the calling thread: its own bound when one is set
// (set_thread_units_per_cta), else the process-wide one of ptx_set_units_per_cta (0: one
// wave, no bound).
int units_per_cta();
// Set the calling thread's bound (units >= 0) or drop it (units < 0); returns the previous
// value (-1 when none was set).
int set_thread_units_per_cta(int units);

// Kernel kinds for the launch counter and the optional per-kernel event profiler.
enum KernelId {
  kBaseRowsForward = 0,
  kBaseCols,
  kBaseRowsAdjoint,
  kFpmRowsForward,
  kFpmCols,
  kFpmRowsAdjoint,
  kFft2Rows,
  kFft2Cols,
  kCodedRows,
  kCodedCols,
  kMiscKernel,
  kSubpixCols,
  kSubpixRows,
  kNumKernelIds
};
// Call around every kernel launch: counts launches and, when profiling is on, records
// a CUDA event pair on the launch stream.
void prof_begin(int id, cudaStream_t s);
void prof_end(int id, cudaStream_t s);

// Power-of-two line lengths 4..1024 (the register-FFT kernels); returns false (and calls
// nothing) for any other length.
template <typename F>
bool dispatch_pow2(int n, F&& f) {
  switch (n) {
    case 4: f(std::integral_constant<int, 4>{}); return true;
    case 8: f(std::integral_constant<int, 8>{}); return true;
    case 16: f(std::integral_constant<int, 16>{}); return true;
    case 32: f(std::integral_constant<int, 32>{}); return true;
    case 64: f(std::integral_constant<int, 64>{}); return true;
    case 128: f(std::integral_constant<int, 128>{}); return true;
    case 256: f(std::integral_constant<int, 256>{}); return true;
    case 512: f(std::integral_constant<int, 512>{}); return true;
    case 1024: f(std::integral_constant<int, 1024>{}); return true;
    default: return false;
  }
}
inline bool is_pow2_len(int n) { return n >= 4 && n <= 1024 && (n & (n - 1)) == 0; }

// Power-of-two line lengths with compile-time register FFT kernels in the conventional
// passes; every other length gets template argument 0 (the mixed-radix kernels where
// mix_ops(n) is non-null, else the runtime-plan kernels).
template <typename F>
void dispatch_len(int n, F&& f) {
  switch (n) {
    case 16: f(std::integral_constant<int, 16>{}); return;
    case 32: f(std::integral_constant<int, 32>{}); return;
    case 64: f(std::integral_constant<int, 64>{}); return;
    case 128: f(std::integral_constant<int, 128>{}); return;
    case 256: f(std::integral_constant<int, 256>{}); return;
    case 512: f(std::integral_constant<int, 512>{}); return;
    case 1024: f(std::integral_constant<int, 1024>{}); return;
    default: f(std::integral_constant<int, 0>{}); return;
  }
}

// ---- conventional passes on the mixed-radix register FFT (ptx_mix.cuh) ---------------
// Compiled for a list of {2,3,5}-smooth lengths that are not powers of two; mix_ops(n)
// is null for every other length (those run the runtime-plan kernels).
struct MixRowsArgs {
  const float2* sample;  // object, H x W
  int H, W;
  const float2* probe;   // ph x pw
  int ph, pw;
  const int64_t* pos;    // (x, y) of each frame's window
  int nframes;
  float2* scratch;       // tiled frames [frame][tile][row][16]
  const float2* twt;     // row-length twiddles (LinePlan::mix_twt / mix_twi)
  const float2* twi;
  unsigned* err;         // window error word (forward pass)
  float2* grad_sample;   // adjoint pass outputs (float2 atomics)
  float2* grad_probe;
};
struct MixColsArgs {
  float2* scratch;
  int ph, pw, frame0, nframes;
  const float2* twt;     // column-length twiddles
  const float2* twi;
  const uint16_t* measured;  // sweep: fftshifted counts
  const float* lut;          // sweep: count -> observed amplitude
  float grad_scale;
  double inv_numel;
  double* loss;
  float2* far_field;         // forward: optional output; backward: input
  float* amplitude;          // forward output
  const float* grad_output;  // backward input
};
enum MixColMode { kMixColSweep = 0, kMixColForward = 1, kMixColBackward = 2 };
struct MixOps {
  int (*prepare)();  // raise the dynamic shared memory limits of the kernels
  void (*rows_forward)(const MixRowsArgs&, cudaStream_t);
  void (*rows_adjoint)(const MixRowsArgs&, cudaStream_t);
  void (*cols)(int mode, const MixColsArgs&, cudaStream_t);
};
const MixOps* mix_ops(int n);

// ---- Fourier ptychography on the mixed-radix engine (ptx_mixfpm.cuh) -------------------
// Used when any of the four FPM sides is not a power of two; compiled for every
// {2,3,5}-smooth length 4..1024 (mix_fpm_ops(n) is null for every other length).
struct MixFpmRowsArgs {
  const float2* spec;   // object spectrum, oh x ow
  int oh, ow;
  const float2* pupil;  // lh x lw
  int lh;
  const int64_t* led;   // (x, y) window corner of each frame in the shifted spectrum
  int nframes;
  float2* scratch;      // tiled frames [frame][tile][row][16], lh x lw
  const float2* twt;    // row-length (lw) twiddles
  const float2* twi;
  float norm;           // 1 / (lh lw) (adjoint)
  float2* grad_spec;    // adjoint outputs (float2 atomics)
  float2* grad_pupil;
};
struct MixFpmColsArgs {
  float2* scratch;
  int lw, frame0, nframes;
  const float2* twt;  // column-length (lh) twiddles
  const float2* twi;
  const uint16_t* measured;  // sweep: counts (not shifted)
  const float* lut;
  float norm;                // 1 / (lh lw)
  float grad_scale;
  double inv_numel;
  double* loss;
  float2* image;             // forward: optional output; backward: input
  float* amplitude;          // forward output
  const float* grad_output;  // backward input
};
struct MixFpmOps {
  int (*prepare)();
  // one image: rows (natural [H][n] -> tiled [tiles(n)][H][16]) and columns (tiled
  // [tiles(W)][n][16] -> natural [n][W] times `scale`); plus: exp(+i) (unnormalised inverse)
  void (*fft2_rows)(bool plus, const float2* in, int H, float2* tiled, const float2* twt, cudaStream_t);
  void (*fft2_cols)(bool plus, const float2* tiled, int W, float2* out, float scale, const float2* twt,
                    cudaStream_t);
  void (*rows_forward)(const MixFpmRowsArgs&, cudaStream_t);
  void (*rows_adjoint)(const MixFpmRowsArgs&, cudaStream_t);
  void (*cols)(int mode, const MixFpmColsArgs&, cudaStream_t);
};
const MixFpmOps* mix_fpm_ops(int n);

// ---- coded / near-field on the mixed-radix engine (ptx_mixcoded.cuh) --------------------
// Field sides that are {2,3,5}-smooth but not powers of two, 16..1000 (mix_coded_ops(n) is
// null for every other side).
struct MixCodedArgs {
  float2* scratch;          // tiled frames [frame][tile][row][16], n x n
  const float2* ospec;      // O^ = fft2(O)
  const float2* t1;         // first transfer function (null: near-field)
  const float2* t2;
  const float* shifts;      // (dx, dy) per frame of this chunk
  float inv_n;              // 1 / n^2
  float2* grad_ospec;
  const float2* twt;        // line twiddles of n (LinePlan::mix_twt / mix_twi)
  const float2* twi;
  double* grad_shifts;      // pass 7, optional
  const float2* mask;       // coded surface M
  float2* xstore;           // x = ifft2(O^ T1 R) per frame of this chunk
  float2* grad_mask;
  int ds, frame0, nframes;
  const uint16_t* measured;  // pass 4 (sweep)
  float scale, grad_scale;
  double inv_numel;
  double* loss;
  float2* sensor;            // pass 4: forward output / backward input
  float* amplitude;
  const float* grad_output;
};
struct MixCodedOps {
  int (*prepare)(int ds);  // also rejects a downsample whose row group does not fit a CTA
  void (*cols)(int stage, bool conj, const MixCodedArgs&, cudaStream_t);  // passes 1, 3 / 5, 7
  void (*rows_mask)(const MixCodedArgs&, cudaStream_t);                   // pass 2
  void (*rows_pool)(int mode, const MixCodedArgs&, cudaStream_t);         // pass 4 (MixColMode)
  void (*rows_grad_mask)(const MixCodedArgs&, cudaStream_t);              // pass 6
};
const MixCodedOps* mix_coded_ops(int n);

// ---- sub-pixel conventional passes on the mixed-radix engine (ptx_mixsubpix.cuh) ---------
// Probe sides that are {2,3,5}-smooth but not powers of two, 16..1000 (mix_subpix_ops(n) is
// null for every other side); the column passes run on the column side ph, the row passes on
// the row side pw.
struct MixSubpixArgs {
  const float2* sample;  // object, H x W (gather)
  float2* grad_sample;   // scatter target
  int H, W, ph, pw;
  const double* pos;     // float (x, y) of every frame of the batch
  int frame0, nframes;   // this chunk
  float2* scratch;       // tiled frames [frame][tile][row][16] of the chunk
  float2* sbuf;          // the shifted patches S, same layout
  const float2* rx;      // row ramps [batch][pw], column ramps [batch][ph] (1/n folded in)
  const float2* ry;
  const float2* probe;
  float2* grad_probe;
  const float2* twt_col;  // mixed-radix twiddles of ph and pw
  const float2* twi_col;
  const float2* twt_row;
  const float2* twi_row;
};
enum MixSubpixRows {
  kMixSubpixSweepForward = 0,  // shift (S stored), x P, row DFT (stored)
  kMixSubpixShiftOnly = 1,     // shift (S stored)
  kMixSubpixForwardOnly = 2,   // shift, x P, row DFT (stored)
  kMixSubpixAdjoint = 3        // inverse row DFT, grad_P, x conj(P), row DFT, opposite shift
};
struct MixSubpixOps {
  int (*prepare)();
  void (*cols)(bool gather, const MixSubpixArgs&, cudaStream_t);  // column side ph
  void (*rows)(int variant, const MixSubpixArgs&, cudaStream_t);  // row side pw
};
const MixSubpixOps* mix_subpix_ops(int n);

}  // namespace ptx
