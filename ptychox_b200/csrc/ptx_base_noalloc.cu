// Allocation-free variant of the conventional fused sweep.
//
// Some hosts cannot hand this library device memory for its scratch frames: an
// acquisition or instrument-control program that loads the library as a plug-in and
// owns the GPU memory pool without exposing an allocator to plug-ins, or a scan loop
// that must never take the device-wide synchronisation a cudaMalloc/cudaFree can cause
// in the middle of an acquisition.  ptx_base_sweep_noalloc serves them: its scratch is
// the file-scope device array below, so the call allocates nothing.  The caller still
// owns and passes every input and output.
//
// Limits and rules:
//   - the array holds kNoallocScratchBytes (8 MiB) on every GPU that loads this library,
//     until the process exits; one probe frame (rounded up to 16 columns) plus the
//     256 KiB count-decode table and a 256-byte header must fit in it, otherwise the call
//     returns PTX_ERR_WORKSPACE;
//   - in host code the array's name is not a device address, so the first call on each
//     device looks the address up with cudaGetSymbolAddress (with that device current)
//     and caches it; ptx_clear_cache drops the cached addresses (a device reset or a new
//     primary context gives the array a new address), so the next call looks them up
//     again; make that first call (and the first after a ptx_clear_cache) before any CUDA
//     graph capture;
//   - all calls share the one array: the error word at its start is cleared by each
//     call and every frame is rewritten before it is read, but calls that overlap on the
//     GPU (different streams, or different host threads on one device) race on it and
//     must be serialised by the caller.
#include <cuda_runtime.h>

#include <mutex>

#include "ptx_internal.h"

namespace ptx {
namespace {

constexpr size_t kNoallocScratchBytes = PTX_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (looked up once per device).
int noalloc_scratch(void** out) {
  int dev = 0;
  if (int st = cuda_status(cudaGetDevice(&dev), "cudaGetDevice")) return st;
  if (dev < 0 || dev >= kMaxDevices) return set_error(PTX_ERR_INVALID_ARGUMENT, "device %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* ptr = nullptr;
    if (int st = cuda_status(cudaGetSymbolAddress(&ptr, g_noalloc_scratch), "cudaGetSymbolAddress(scratch)")) {
      return st;
    }
    g_noalloc_ptr[dev] = ptr;
  }
  *out = g_noalloc_ptr[dev];
  return PTX_OK;
}

}  // namespace

void clear_noalloc_cache() {
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  for (void*& p : g_noalloc_ptr) p = nullptr;
}

}  // namespace ptx

extern "C" int ptx_base_sweep_noalloc(const float* sample, int sample_h, int sample_w, const float* probe,
                                      int probe_h, int probe_w, const int64_t* positions_xy, int batch,
                                      const uint16_t* measured, float scale, double* loss, float* grad_sample,
                                      float* grad_probe, void* stream) {
  using namespace ptx;
  if (probe_h <= 0 || probe_w <= 0) return set_error(PTX_ERR_INVALID_ARGUMENT, "non-positive probe shape");
  const size_t need = ptx_base_workspace_bytes(probe_h, probe_w, 1);  // header, decode table, one frame
  if (need > kNoallocScratchBytes) {
    return set_error(PTX_ERR_WORKSPACE,
                     "a %d x %d probe frame needs %zu bytes of scratch; ptx_base_sweep_noalloc has a fixed "
                     "%zu-byte scratch (use ptx_base_sweep with a caller workspace)",
                     probe_h, probe_w, need, kNoallocScratchBytes);
  }
  void* scratch = nullptr;
  if (int st = noalloc_scratch(&scratch)) return st;
  return ptx_base_sweep(sample, sample_h, sample_w, probe, probe_h, probe_w, positions_xy, batch, measured, scale,
                        loss, grad_sample, grad_probe, scratch, kNoallocScratchBytes, stream);
}
