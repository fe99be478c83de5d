/*
 * libptychox — C ABI of the B200-native (sm_100a) ptychography operators.
 *
 * Conventions shared by every entry point:
 *   - complex arrays are interleaved complex64 (float re, float im), row-major,
 *     contiguous, in device memory; they are passed as float* / const float*;
 *   - positions / LED indices are device int64 pairs (x, y), zero-based;
 *   - `stream` is a cudaStream_t (NULL = legacy default stream); every launch is
 *     stream-ordered and nothing synchronises the host;
 *   - outputs are caller-allocated; temporary frames live in a caller-provided
 *     workspace whose minimum size the *_workspace_bytes functions return (a larger
 *     workspace processes more frames per launch); the workspace must start on a
 *     256-byte boundary (cudaMalloc and PyTorch allocations do);
 *   - the return value is a status code (PTX_OK = 0); ptx_last_error() gives the
 *     calling thread's last message.
 *
 * Gradients follow PyTorch's convention for complex inputs of a real loss
 * (dL/dRe + i dL/dIm), as the reference's hand-written backward functions do.
 *
 * Reference interfaces replaced (THUHoloLab/PtychoX, python/ptychoX/csrc):
 *   pybind11 `_C.forward` / `_C.backward` / `_C.clear_plan_cache` of
 *   base_extension.cpp:21-66, fpm_extension.cpp:21-66, coded_extension.cpp:26-94.
 */
#ifndef PTYCHOX_H_
#define PTYCHOX_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------- */
#define PTX_OK 0
#define PTX_ERR_INVALID_ARGUMENT 1  /* bad pointer, shape or scalar          -> ValueError   */
#define PTX_ERR_UNSUPPORTED_SIZE 2  /* frame side not {2,3,5}-smooth / too big -> ValueError   */
#define PTX_ERR_WORKSPACE 3         /* workspace smaller than one frame      -> RuntimeError */
#define PTX_ERR_CUDA 4              /* CUDA launch / runtime error           -> RuntimeError */
#define PTX_ERR_OUT_OF_BOUNDS 5     /* a scan window leaves the object       -> ValueError   */
#define PTX_ERR_TIMEOUT 6           /* a bounded device wait gave up         -> RuntimeError */

/* ---- library ------------------------------------------------------------------- */

/* Library version as 10000*major + 100*minor + patch. */
int ptx_version(void);

/* Message of the calling thread's last failed call ("" if none). */
const char* ptx_last_error(void);

/* Drop cached FFT plans (twiddle tables are rebuilt on next use) and the cached device
 * address of ptx_base_sweep_noalloc's scratch array (looked up again by its next call).
 * Replaces `_C.clear_plan_cache` (base_extension.cpp:65, fpm_extension.cpp:65,
 * coded_extension.cpp:93) and ptychoX.clear_cuda_plan_cache (ptychoX/__init__.py:10-13). */
int ptx_clear_cache(void);

/* Number of kernels this library has launched in the process (all devices). */
long long ptx_launch_count(void);

/* Work granularity of the persistent row passes (process-wide, default 0).  0: each such
 * pass runs one wave of resident CTAs, every CTA taking an equal share of the (row group,
 * frame) units -- the fastest layout when one sweep has the GPU to itself.  k > 0: enough
 * CTAs that none takes more than k units, so kernels that other streams launch meanwhile
 * (several reconstructions served at once) interleave with the pass CTA by CTA.  Applies to
 * launches made (or captured into CUDA graphs) after the call.  No reference counterpart:
 * the reference's kernels are one-shot grids. */
int ptx_set_units_per_cta(int units);

/* The same bound for launches made (or captured) by the calling host thread only, overriding
 * the process-wide value for that thread; units < 0 drops the override.  A server thread that
 * captures bounded sweeps uses it so that neither the host program's own sweeps nor another
 * server's captures see its bound.  No reference counterpart. */
int ptx_set_thread_units_per_cta(int units);

/* The bound in force for the calling thread's launches (its own, else the process-wide one). */
int ptx_get_units_per_cta(void);

/* Copy `bytes` from host memory `src` (pageable or page-locked) to device memory `dst`
 * (current device) in stream order on `stream`.  Up to 256 KiB the bytes are copied at the
 * call into a page-locked ring owned by the library (so `src` may be reused as soon as the
 * call returns) and a kernel reads them over the bus: a small per-step input such as a scan
 * is then neither queued on a copy engine behind another stream's large transfer nor
 * blocking the host as a pageable copy would.  Larger inputs, and calls on a stream that is
 * being captured into a CUDA graph (whose copy node must re-read `src` on every replay),
 * take cudaMemcpyAsync.  No reference counterpart: the reference moves scans with torch's
 * `.to(device)`. */
int ptx_stage_host_bytes(void* dst, const void* src, size_t bytes, void* stream);

/* Optional per-kernel CUDA-event timing: when enabled every launch is bracketed by an
 * event pair on its stream.  ptx_profile_read synchronises on the recorded events and
 * returns the accumulated device time and timed launches of one kernel kind
 * (ids 0 .. ptx_profile_kinds()-1, named by ptx_profile_name). */
int ptx_profile_enable(int on);
int ptx_profile_reset(void);
int ptx_profile_kinds(void);
int ptx_profile_read(int kernel_id, double* total_ms, long long* launches);
const char* ptx_profile_name(int kernel_id);

/* 1 if `n` is a supported transform length (n = 2^a 3^b 5^c, 2 <= n <= 1024). */
int ptx_fft_supported(int n);

/* Which kernels serve line length `n` in the conventional passes: 1 for the power-of-two
 * register FFT (16 .. 1024), 2 for the mixed-radix register FFT (the 2^a 3^b 5^c lengths
 * 6 .. 1000 that are not powers of two), 3 for the runtime-plan shared-memory FFT (the
 * remaining supported lengths 2 .. 8), 0 for an unsupported length.  Host-only query. */
int ptx_fft_engine(int n);

/* Build the twiddle table for length n on the current device now (it is otherwise
 * built on first use, which must not happen inside a CUDA graph capture). */
int ptx_fft_prepare(int n);

/* ---- conventional ptychography --------------------------------------------------
 * Operator  A[b] = |fftshift(fft2(sample[y_b:y_b+ph, x_b:x_b+pw] * probe))|.
 * Replaces `_C.forward` / `_C.backward` of base_extension.cpp:21-60 and the torch path
 * of python/ptychoX/base/ops.py:41-107.
 */

/* Minimum workspace for the base entry points (frames processed per launch = as many
 * as fit; `batch` caps what is useful). */
size_t ptx_base_workspace_bytes(int probe_h, int probe_w, int batch);

/* Forward.  far_field: complex64 [batch, ph, pw], the fftshifted far field (may be
 * NULL when not needed); amplitude: float32 [batch, ph, pw].
 * Replaces base_extension.cpp:21-32 (ptychox_base_forward_cuda, base_kernel.cu:302-329). */
int ptx_base_forward(const float* sample, int sample_h, int sample_w,
                     const float* probe, int probe_h, int probe_w,
                     const int64_t* positions_xy, int batch,
                     float* far_field, float* amplitude,
                     void* workspace, size_t workspace_bytes, void* stream);

/* Adjoint of the forward for an upstream gradient grad_output (float32 [batch, ph, pw]):
 * grad_sample (complex64 [H, W]) and grad_probe (complex64 [ph, pw]) are OVERWRITTEN.
 * far_field is the array written by ptx_base_forward; the object patches are re-read
 * from `sample` instead of being saved.
 * Replaces base_extension.cpp:34-60 (ptychox_base_backward_cuda, base_kernel.cu:331-357). */
int ptx_base_backward(const float* grad_output, const float* far_field,
                      const float* sample, int sample_h, int sample_w,
                      const float* probe, int probe_h, int probe_w,
                      const int64_t* positions_xy, int batch,
                      float* grad_sample, float* grad_probe,
                      void* workspace, size_t workspace_bytes, void* stream);

/* Fused sweep: forward, amplitude-MSE loss against uint16 counts, adjoint.
 * loss (device double[1]) = mean((A - sqrt(scale * I))^2) accumulated in FP64;
 * grad_sample / grad_probe are OVERWRITTEN with dloss/d(sample, probe).
 * Equivalent to F.mse_loss(ptychoX_base(...), observed).backward()
 * (python/train_ptychography.py:549-557) with observed = sqrt(float32(I) * scale). */
int ptx_base_sweep(const float* sample, int sample_h, int sample_w,
                   const float* probe, int probe_h, int probe_w,
                   const int64_t* positions_xy, int batch,
                   const uint16_t* measured, float scale,
                   double* loss, float* grad_sample, float* grad_probe,
                   void* workspace, size_t workspace_bytes, void* stream);

/* ptx_base_sweep for square 32-, 64- or 128-point probes (PTX_ERR_UNSUPPORTED_SIZE
 * otherwise), same arguments and results: one CTA runs the whole sweep of a frame in shared
 * memory (gather, row and column DFTs with the loss epilogue, inverse DFTs, gradient
 * scatter), so a sweep is the prologue and one launch, with no scratch frames in HBM (the
 * workspace still holds the count-decode table and the error word).  The Python operators
 * use it for such probes. */
int ptx_base_sweep_small(const float* sample, int sample_h, int sample_w,
                         const float* probe, int probe_h, int probe_w,
                         const int64_t* positions_xy, int batch,
                         const uint16_t* measured, float scale,
                         double* loss, float* grad_sample, float* grad_probe,
                         void* workspace, size_t workspace_bytes, void* stream);

/* Status word of the last conventional call (ptx_base_forward / _backward / _sweep /
 * _sweep_small) that used `workspace`: the kernels check every scan window on the device,
 * skip a frame whose window leaves the object and set bit 0 of the word (the reference reads
 * such windows out of bounds, base_kernel.cu:108-125; its torch path raises only for windows
 * past the far edge).  This call copies the 4-byte word in stream order on `stream` to
 * `status` (device memory or page-locked host memory: no host synchronisation), so a caller
 * with device-resident positions learns of a bad window without copying the positions to
 * the host.  Read it after the stream has reached the copy and map it with ptx_status_code. */
int ptx_workspace_status(const void* workspace, unsigned* status, void* stream);
/* PTX_ERR_OUT_OF_BOUNDS when bit 0 of a status word is set, else PTX_OK. */
int ptx_status_code(unsigned status);

/* ---- conventional ptychography at sub-pixel scan positions -------------------------
 * No reference counterpart: the reference crops integer windows only
 * (python/ptychoX/base/ops.py:61-62, base_extension.cpp:30 demands int64).  positions_xy
 * holds float64 (x, y) pairs; each frame takes the window at the rounded corner
 * (x0, y0) = floor(p + 1/2) and shifts it by the fraction (dx, dy) = p - (x0, y0) in
 * [-1/2, 1/2) with the Fourier phase ramp of the reference's shift_phase_ramp
 * (coded/ops.py:157-171) applied to the patch:
 *   S = ifft2(fft2(O[y0:y0+ph, x0:x0+pw]) exp(2 pi i (dx kx / pw + dy ky / ph))),
 *   A = |fftshift(fft2(S * probe))|
 * (kx, ky the signed integer frequencies).  At integer positions S is the plain window.
 * Probe sides: powers of two in [16, 1024] (PTX_ERR_UNSUPPORTED_SIZE otherwise).  Windows that
 * leave the object are skipped and flagged in the status word (ptx_workspace_status).
 * Workspace: ptx_base_subpix_workspace_bytes (tables of the per-frame ramps, and two scratch
 * frames per frame processed at once). */
size_t ptx_base_subpix_workspace_bytes(int probe_h, int probe_w, int batch);

/* Forward: far_field (complex64 [batch, ph, pw], fftshifted, may be NULL) and amplitude. */
int ptx_base_subpix_forward(const float* sample, int sample_h, int sample_w,
                            const float* probe, int probe_h, int probe_w,
                            const double* positions_xy, int batch,
                            float* far_field, float* amplitude,
                            void* workspace, size_t workspace_bytes, void* stream);

/* Adjoint for grad_output (float32 [batch, ph, pw]) from the forward's far field;
 * grad_sample and grad_probe are OVERWRITTEN. */
int ptx_base_subpix_backward(const float* grad_output, const float* far_field,
                             const float* sample, int sample_h, int sample_w,
                             const float* probe, int probe_h, int probe_w,
                             const double* positions_xy, int batch,
                             float* grad_sample, float* grad_probe,
                             void* workspace, size_t workspace_bytes, void* stream);

/* Fused sweep: mean((A - sqrt(scale * I))^2) in FP64 and its gradients (OVERWRITTEN), as
 * ptx_base_sweep on the sub-pixel operator (five passes: column shift of the gathered
 * window, row shift x probe x row DFT, the column loss pass, the row adjoint with the probe
 * gradient, the column adjoint with the object scatter). */
int ptx_base_subpix_sweep(const float* sample, int sample_h, int sample_w,
                          const float* probe, int probe_h, int probe_w,
                          const double* positions_xy, int batch,
                          const uint16_t* measured, float scale,
                          double* loss, float* grad_sample, float* grad_probe,
                          void* workspace, size_t workspace_bytes, void* stream);

/* ---- Fourier ptychography --------------------------------------------------------
 * Operator  A[b] = |ifft2(fftshift(S[window_b] * pupil))|, S = fft2(object), window_b the
 * (lh x lw) block at rows (ly+r+H/2) % H, columns (lx+c+W/2) % W of S.
 * All four sides must be powers of two in [4, 1024].
 * Replaces `_C.forward` / `_C.backward` of fpm_extension.cpp:21-60 and the torch path of
 * python/ptychoX/fpm/ops.py:38-124.
 */
size_t ptx_fpm_workspace_bytes(int object_h, int object_w, int low_h, int low_w, int batch);

/* Forward.  spectrum (OUT, complex64 [H, W]) = fft2(object), kept by the caller for the
 * backward; image (complex64 [batch, lh, lw], may be NULL) and amplitude (float32).
 * Replaces fpm_extension.cpp:21-32 (ptychox_fpm_forward_cuda, fpm_kernel.cu:233-273). */
int ptx_fpm_forward(const float* object, int object_h, int object_w,
                    const float* pupil, int low_h, int low_w,
                    const int64_t* led_indices_xy, int batch,
                    float* spectrum, float* image, float* amplitude,
                    void* workspace, size_t workspace_bytes, void* stream);

/* Adjoint for grad_output (float32 [batch, lh, lw]); image and spectrum as written by the
 * forward.  grad_object (complex64 [H, W]) and grad_pupil are OVERWRITTEN.
 * Replaces fpm_extension.cpp:34-60 (ptychox_fpm_backward_cuda, fpm_kernel.cu:275-317). */
int ptx_fpm_backward(const float* grad_output, const float* image, const float* spectrum,
                     int object_h, int object_w, const float* pupil, int low_h, int low_w,
                     const int64_t* led_indices_xy, int batch,
                     float* grad_object, float* grad_pupil,
                     void* workspace, size_t workspace_bytes, void* stream);

/* Fused sweep: mean((A - sqrt(scale * I))^2) in FP64 and its gradients (OVERWRITTEN),
 * as F.mse_loss(ptychoX_fourier(...), observed).backward() (python/train_fpm.py:255-263). */
int ptx_fpm_sweep(const float* object, int object_h, int object_w,
                  const float* pupil, int low_h, int low_w,
                  const int64_t* led_indices_xy, int batch,
                  const uint16_t* measured, float scale,
                  double* loss, float* grad_object, float* grad_pupil,
                  void* workspace, size_t workspace_bytes, void* stream);

/* ---- coded and near-field ptychography ------------------------------------------
 * Operator  x_b = ifft2(fft2(O) T1 R_b),  s_b = ifft2(fft2(x_b M) T2),
 * A_b = sqrt(avgpool_ds |s_b|^2),  R_b = exp(2 pi i (dx_b fx + dy_b fy)) with signed
 * integer frequencies and shifts_xy float32 [batch, 2] (dx, dy) in units of the field side.
 * transfer_1 = NULL gives near-field ptychography (T1 = 1).  Square fields, n a power of
 * two in [16, 1024]; downsample must divide n (and 8).
 * Replaces `_C.forward` / `_C.backward` of coded_extension.cpp:26-88 and the torch path
 * of python/ptychoX/coded/ops.py:22-171; near-field replaces the MATLAB operator
 * adPtychoX_nearf (fwd_adPtychoX_nearf.cu, bwd_adPtychoX_nearf.cu) with the exact
 * RMS-pool gradient.
 */
size_t ptx_coded_workspace_bytes(int n, int batch);

/* Forward: x_forward, sensor (complex64 [batch, n, n], saved for the backward) and
 * amplitude (float32 [batch, n/ds, n/ds]).  Replaces coded_kernel.cu:283-345. */
int ptx_coded_forward(const float* object, const float* coded_surface,
                      const float* transfer_1, const float* transfer_2, int n,
                      const float* shifts_xy, int batch, int downsample,
                      float* x_forward, float* sensor, float* amplitude,
                      void* workspace, size_t workspace_bytes, void* stream);

/* Adjoint for grad_output (float32 [batch, n/ds, n/ds]) from the saved forward arrays
 * (x_forward 16-byte aligned); grad_object and grad_coded (complex64 [n, n]) are OVERWRITTEN.
 * Replaces coded_kernel.cu:347-424. */
int ptx_coded_backward(const float* grad_output, const float* x_forward, const float* sensor,
                       const float* amplitude, const float* coded_surface,
                       const float* transfer_1, const float* transfer_2, int n,
                       const float* shifts_xy, int batch, int downsample,
                       float* grad_object, float* grad_coded,
                       void* workspace, size_t workspace_bytes, void* stream);

/* Fused sweep: mean((A - sqrt(scale * I))^2) in FP64 (I uint16 [batch, n/ds, n/ds]) and
 * its gradients (OVERWRITTEN), as F.mse_loss(ptychoX_coded(...), observed).backward()
 * (python/train_coded.py:225-237). */
int ptx_coded_sweep(const float* object, const float* coded_surface,
                    const float* transfer_1, const float* transfer_2, int n,
                    const float* shifts_xy, int batch, int downsample,
                    const uint16_t* measured, float scale,
                    double* loss, float* grad_object, float* grad_coded,
                    void* workspace, size_t workspace_bytes, void* stream);

/* Sweep with the periodic finite-difference data loss of python/train_coded.py:101-107
 * (`fd_loss`, the `--loss fd-isotropic` / `fd-anisotropic` options of train_coded.py:237)
 * in place of the MSE: D = A - sqrt(scale * I), dx / dy the periodic forward differences
 * of D along x / y, loss = sum sqrt(dx^2 + dy^2 + 1e-5) (isotropic != 0) or
 * sum |dx| + |dy|, summed (not averaged) in FP64; gradients OVERWRITTEN.  The loss couples
 * neighbouring pixels, so the pooled amplitudes are materialised: the sweep runs the
 * forward passes (keeping x and the sensor fields), a stencil pass for dL/dA, and the
 * adjoint passes, all inside the workspace (ptx_coded_fd_workspace_bytes). */
size_t ptx_coded_fd_workspace_bytes(int n, int batch, int downsample);
int ptx_coded_sweep_fd(const float* object, const float* coded_surface,
                       const float* transfer_1, const float* transfer_2, int n,
                       const float* shifts_xy, int batch, int downsample,
                       const uint16_t* measured, float scale, int isotropic,
                       double* loss, float* grad_object, float* grad_coded,
                       void* workspace, size_t workspace_bytes, void* stream);

/* General coded / near-field sweep.  loss_kind: PTX_LOSS_MSE (as ptx_coded_sweep),
 * PTX_LOSS_FD_ISOTROPIC / PTX_LOSS_FD_ANISOTROPIC (as ptx_coded_sweep_fd).  grad_shifts
 * (double [batch, 2], may be NULL) receives dL/d(shifts_xy): the shifts enter only through
 * the phase ramp R_b, so dL/d(dx_b, dy_b) = -2 pi sum_k (fx, fy) Im(conj(G_b) u_b) with
 * u_b = fft2(O) T1 R_b and G_b its gradient -- what autograd gives through the reference's
 * torch formulation (python/ptychoX/coded/ops.py:157-171; its CUDA operator returns no
 * shift gradient).  Workspace: ptx_coded_sweep_ex_workspace_bytes. */
#define PTX_LOSS_MSE 0
#define PTX_LOSS_FD_ISOTROPIC 1
#define PTX_LOSS_FD_ANISOTROPIC 2
size_t ptx_coded_sweep_ex_workspace_bytes(int n, int batch, int downsample, int loss_kind);
int ptx_coded_sweep_ex(const float* object, const float* coded_surface,
                       const float* transfer_1, const float* transfer_2, int n,
                       const float* shifts_xy, int batch, int downsample,
                       const uint16_t* measured, float scale, int loss_kind,
                       double* loss, float* grad_object, float* grad_coded, double* grad_shifts,
                       void* workspace, size_t workspace_bytes, void* stream);

/* ---- optimiser step -------------------------------------------------------------
 * Adam on a complex64 parameter with torch.optim.Adam semantics (the reference drivers'
 * optimiser, python/train_ptychography.py:500-507): the (re, im) pairs are independent
 * reals, m = lerp(m, g, 1-b1), v = b2 v + (1-b2) g^2,
 * p -= lr/(1-b1^t) * m / (sqrt(v)/sqrt(1-b2^t) + eps); then an optional projection:
 * PTX_CONSTRAIN_UNIT_AMPLITUDE (|z| <= 1, phase kept; the MATLAB scripts' object clamp)
 * or PTX_CONSTRAIN_REAL_NONNEGATIVE (z -> max(Re z, 0); train_coded.py:242-244).
 * `state` is 16 bytes of device memory, zeroed before the first step; it holds the step
 * count, so the call can be captured in a CUDA graph and replayed.  exp_avg and
 * exp_avg_sq are complex64-shaped (n_complex pairs) and zero at the start.  All four
 * arrays must be 16-byte aligned. */
#define PTX_CONSTRAIN_NONE 0
#define PTX_CONSTRAIN_UNIT_AMPLITUDE 1
#define PTX_CONSTRAIN_REAL_NONNEGATIVE 2
int ptx_adam_step(float* param, const float* grad, float* exp_avg, float* exp_avg_sq,
                  size_t n_complex, void* state, float lr, float beta1, float beta2, float eps,
                  int constraint, void* stream);

/* Allocation-free fused sweep, for callers that cannot allocate device memory: a host
 * program that loads this library as a plug-in and keeps the GPU memory pool to itself,
 * or an acquisition loop that must not take the device-wide synchronisation of a
 * cudaMalloc/cudaFree mid-scan.  No counterpart in the reference (which allocates every
 * temporary with torch::empty / torch::zeros, base_kernel.cu:250-251,281-282).
 * Same arguments and results as ptx_base_sweep minus the workspace: the scratch frames
 * live in a fixed PTX_NOALLOC_SCRATCH_BYTES device array that every GPU loading the
 * library holds until exit.  ptx_base_workspace_bytes(probe_h, probe_w, 1) (one frame of
 * ph x pw rounded up to 16 columns, 8 bytes each, plus a 256 KiB table and 256 bytes)
 * must fit in it, else PTX_ERR_WORKSPACE.  The first call on a device looks up the
 * array's device address (make it before any CUDA graph capture).  All calls share the
 * array: calls that overlap on the GPU race and must be serialised by the caller. */
#define PTX_NOALLOC_SCRATCH_BYTES (8u * 1024u * 1024u)
int ptx_base_sweep_noalloc(const float* sample, int sample_h, int sample_w,
                           const float* probe, int probe_h, int probe_w,
                           const int64_t* positions_xy, int batch,
                           const uint16_t* measured, float scale,
                           double* loss, float* grad_sample, float* grad_probe, void* stream);

/* ---- reconstruction server (continuous batching of whole reconstructions) ---------- */

/* The reference drivers' training loop (python/train_ptychography.py:473-603, train_fpm.py,
 * train_coded.py: per iteration a sweep, F.mse_loss and torch.optim.Adam with betas
 * (0.9, 0.999), eps 1e-16) served natively for many problems at once.  Requests are copied
 * at submit; a scheduler thread admits them first come first served while their resident
 * bytes fit the HBM budget, keeps each admitted reconstruction on the device (one
 * stream-ordered allocation), captures one iteration (fused sweep + one Adam step of each
 * parameter) as a CUDA graph with the persistent passes bounded to 8 units per CTA, and
 * replays the iterations of all active reconstructions concurrently on per-reconstruction
 * streams (older ones at higher priority).  Two threads: the scheduler thread only queues
 * graph replays and polls events (it never waits on the device); an admission thread does
 * the blocking work -- allocation, upload, the warm-up sweep, capture, and the read-back of
 * finished reconstructions -- off the scheduler's path.  The 8-unit bound is the capturing
 * thread's own (ptx_set_thread_units_per_cta): the process-wide setting and the sweeps of
 * other host threads are untouched.  A request with target_ratio > 0 stops at a fixed error:
 * once a completed iteration's loss is at most target_ratio times the initial loss (the
 * sweep at obj0 / aux0), no further iteration is queued.  Python:
 * ptychox_b200.native_server. */
#define PTX_MODALITY_CONVENTIONAL 0
#define PTX_MODALITY_FOURIER 1
#define PTX_MODALITY_CODED 2
#define PTX_MODALITY_NEARFIELD 3

typedef struct ptx_recon_request {
  int modality;            /* PTX_MODALITY_* */
  int obj_h, obj_w;        /* object (conventional), object spectrum side (Fourier), field (coded) */
  int aux_h, aux_w;        /* probe / pupil / coded surface or probe field (coded: = object) */
  int batch;               /* positions, LEDs or shifts */
  int downsample;          /* coded and near-field */
  int iters;               /* iterations: one sweep and one Adam step of each parameter */
  float scale;             /* observed amplitude = sqrt(scale * count) */
  float lr_obj, lr_aux;    /* Adam learning rates */
  int constrain_obj, constrain_aux;  /* PTX_CONSTRAIN_* projection after each step */
  const float* obj0;       /* host, interleaved complex64 [obj_h][obj_w] */
  const float* aux0;       /* host, complex64 [aux_h][aux_w] */
  const void* scan;        /* host: int64 [batch][2] positions / LED corners, float32 [batch][2] shifts */
  const uint16_t* measured;  /* host counts [batch][aux_h][aux_w], coded [batch][n/ds][n/ds] */
  const float* transfer_1; /* host complex64 [n][n] (coded; NULL otherwise) */
  const float* transfer_2; /* host complex64 [n][n] (coded and near-field) */
  float target_ratio;      /* > 0: stop once loss <= target_ratio * initial loss; 0: run all iters */
} ptx_recon_request;

/* Start a server on `device`; hbm_budget 0 = 70% of the free device memory. */
int ptx_server_create(int device, size_t hbm_budget, int max_active, void** server);
/* Queue a reconstruction (its arrays are copied at the call); *id identifies it.  A request
 * whose resident bytes exceed the budget is refused with PTX_ERR_WORKSPACE, a conventional
 * scan whose windows leave the object with PTX_ERR_OUT_OF_BOUNDS. */
int ptx_server_submit(void* server, const ptx_recon_request* request, long long* id);
/* Non-blocking.  *done = 1 when the reconstruction has finished: the final parameters are
 * copied to object_out / aux_out (host, as obj0 / aux0; either may be NULL), the loss of its
 * last sweep to *final_loss and submit-to-finish seconds to *latency_s, and the request is
 * forgotten.  A failed request returns its error code (and is forgotten). */
int ptx_server_poll(void* server, long long id, int* done, double* final_loss, double* latency_s,
                    float* object_out, float* aux_out);
/* ptx_server_poll that also reports the iterations the reconstruction ran (*iterations, may
 * be NULL): iters, or fewer when its error target was met. */
int ptx_server_poll_ex(void* server, long long id, int* done, double* final_loss, double* latency_s,
                       int* iterations, float* object_out, float* aux_out);
/* Cancel queued requests, finish the active ones, stop the scheduler and free the server. */
int ptx_server_destroy(void* server);

/* ---- sub-pixel registration (positional tracking of coded / near-field scans) ---- */

/* Workspace of ptx_reg_upsampled_peak (0 when usfac <= 2). */
size_t ptx_reg_workspace_bytes(int batch, int rows, int cols, int usfac);

/* The matrix-multiply DFT refinement of dftregistration (matlab/Examples/Near-field
 * Ptychography/+misc/dftregistration.m:102-121 with dftups :150-185) for `batch` images:
 * `cross_power` [batch][rows][cols] interleaved complex64 holds buf2ft .* conj(buf1ft);
 * `row_center` / `col_center` (int32 [batch], device) the initial estimate times usfac
 * (round(shift * usfac)).  The inverse DFT of each cross-power spectrum is evaluated on the
 * n x n patch (n = ceil(1.5 usfac)) of the grid upsampled by usfac whose element
 * (fix(n / 2), fix(n / 2)) sits at the estimate; `peak_rc` (int32 [batch][2]) receives the
 * zero-based (row, col) of the first maximum of |CC| in column-major order (MATLAB's
 * find(..., 1, 'first')) and `peak_cc` (interleaved complex128 [batch]) CC there,
 * CC = conj(dftups); the upsampled DFT is summed in FP64.  The refined shift is
 * estimate + (peak - fix(n / 2)) / usfac.  3 <= usfac <= 100000. */
int ptx_reg_upsampled_peak(const float* cross_power, int batch, int rows, int cols, int usfac,
                           const int* row_center, const int* col_center, int* peak_rc, double* peak_cc,
                           void* workspace, size_t workspace_bytes, void* stream);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif /* PTYCHOX_H_ */
