// Library core: error reporting, FFT line plans and their FP64-derived twiddle tables.
//
// The reference keeps a process-global cuFFT plan cache keyed by (device, batch, h, w)
// behind a mutex (python/ptychoX/csrc/base_kernel.cu:19-91).  Here a "plan" is only the
// radix sequence of one line length plus its twiddle table; tables live in a static
// device pool (one per device), are filled once per (device, length) with a
// synchronous copy, and are shared by every transform of that length.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <cstdarg>
#include <cstdio>
#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "ptx_internal.h"
#include "ptx_mixfft.cuh"

namespace ptx {

namespace {

constexpr int kPoolEntries = 1 << 17;  // 1 MB of float2 per device
__device__ float2 g_twiddle_pool[kPoolEntries];

thread_local std::string g_last_error;

std::mutex g_plan_mutex;
std::map<int, int> g_table_offset;                       // n -> offset of n's tables in the pool
int g_pool_used = 0;
std::map<std::pair<int, int>, LinePlan> g_plans;         // (device, n) -> plan

bool factor_235(int n, int* a, int* b, int* c) {
  *a = *b = *c = 0;
  if (n < 2) return false;
  while (n % 2 == 0) { n /= 2; ++*a; }
  while (n % 3 == 0) { n /= 3; ++*b; }
  while (n % 5 == 0) { n /= 5; ++*c; }
  return n == 1;
}

// Radix sequence: the power-of-two part in ceil(a/4) balanced stages of radix 16/8/4/2,
// then one stage per factor 3 and 5.
int make_radices(int n, int* radix) {
  int a, b, c;
  if (!factor_235(n, &a, &b, &c)) return -1;
  int ns = 0;
  if (a > 0) {
    const int stages = (a + 3) / 4;
    int left = a;
    for (int s = 0; s < stages; ++s) {
      const int bits = (left + (stages - s) - 1) / (stages - s);  // ceil(left / remaining)
      radix[ns++] = 1 << bits;
      left -= bits;
    }
  }
  for (int i = 0; i < b; ++i) radix[ns++] = 3;
  for (int i = 0; i < c; ++i) radix[ns++] = 5;
  return ns;
}

}  // namespace

int set_error(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int cuda_status(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return PTX_OK;
  return set_error(PTX_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

bool size_supported(int n) {
  int a, b, c;
  if (n < 2 || n > 1024) return false;
  if (!factor_235(n, &a, &b, &c)) return false;
  int radix[kMaxStages];
  return make_radices(n, radix) <= kMaxStages;
}

int get_line_plan(int n, LinePlan* out) {
  if (!size_supported(n)) {
    return set_error(PTX_ERR_UNSUPPORTED_SIZE,
                     "transform length %d is not supported (needs 2^a 3^b 5^c, 2..1024)", n);
  }
  int dev = 0;
  if (int st = cuda_status(cudaGetDevice(&dev), "cudaGetDevice")) return st;
  std::lock_guard<std::mutex> lock(g_plan_mutex);
  auto key = std::make_pair(dev, n);
  auto it = g_plans.find(key);
  if (it != g_plans.end()) {
    *out = it->second;
    return PTX_OK;
  }
  LinePlan p{};
  p.n = n;
  p.threads = (n + kValuesPerThread - 1) / kValuesPerThread;
  int radix[kMaxStages];
  p.nstages = make_radices(n, radix);
  p.radices = 0;
  for (int s = 0; s < p.nstages; ++s) p.radices |= static_cast<unsigned long long>(radix[s]) << (5 * s);
  // the natural table (n entries), then the two layouts of the mixed-radix engine's
  // inter-step twiddles (n entries each; every supported length has them: the generic-length
  // FPM kernels run powers of two on that engine too)
  const int mix_b = mix::split_b(n);
  const int entries = mix_b ? 3 * n : n;
  int offset;
  auto ot = g_table_offset.find(n);
  if (ot == g_table_offset.end()) {
    const int span = (entries + 31) / 32 * 32;
    if (g_pool_used + span > kPoolEntries) {
      return set_error(PTX_ERR_UNSUPPORTED_SIZE, "twiddle pool exhausted (call ptx_clear_cache)");
    }
    offset = g_pool_used;
    g_pool_used += span;
    g_table_offset[n] = offset;
  } else {
    offset = ot->second;
  }
  std::vector<float2> table(entries);
  const double two_pi = 6.283185307179586476925286766559;
  for (int m = 0; m < n; ++m) {
    const double ang = two_pi * static_cast<double>(m) / static_cast<double>(n);
    table[m] = make_float2(static_cast<float>(std::cos(ang)), static_cast<float>(-std::sin(ang)));
  }
  if (mix_b) {
    const int a = n / mix_b;
    for (int t = 0; t < mix_b; ++t) {
      for (int u = 0; u < a; ++u) {
        const float2 w = table[(t * u) % n];
        table[n + u * mix_b + t] = w;
        table[2 * n + t * a + u] = w;
      }
    }
  }
  if (int st = cuda_status(cudaMemcpyToSymbol(g_twiddle_pool, table.data(), sizeof(float2) * entries,
                                              sizeof(float2) * offset, cudaMemcpyHostToDevice),
                           "twiddle upload")) {
    return st;
  }
  void* base = nullptr;
  if (int st = cuda_status(cudaGetSymbolAddress(&base, g_twiddle_pool), "cudaGetSymbolAddress")) {
    return st;
  }
  p.tw = reinterpret_cast<const float2*>(base) + offset;
  p.mix_twt = mix_b ? p.tw + n : nullptr;
  p.mix_twi = mix_b ? p.tw + 2 * n : nullptr;
  g_plans[key] = p;
  *out = p;
  return PTX_OK;
}

namespace {
std::mutex g_smem_mutex;
std::map<std::pair<int, const void*>, int> g_smem_cap;  // (device, kernel) -> cap already set
}  // namespace

int ensure_smem(const void* kernel, int bytes) {
  // the default 48 KB cap covers a kernel's static shared memory too (block reductions
  // keep up to a few hundred bytes there): raise the cap for anything within 1 KB of it
  if (bytes + 1024 <= 48 * 1024) return PTX_OK;
  int dev = 0;
  if (int st = cuda_status(cudaGetDevice(&dev), "cudaGetDevice")) return st;
  const auto key = std::make_pair(dev, kernel);
  {
    std::lock_guard<std::mutex> lock(g_smem_mutex);
    auto it = g_smem_cap.find(key);
    if (it != g_smem_cap.end() && it->second >= bytes) return PTX_OK;
  }
  if (int st = cuda_status(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes),
                           "cudaFuncSetAttribute(MaxDynamicSharedMemorySize)")) {
    return st;
  }
  std::lock_guard<std::mutex> lock(g_smem_mutex);
  int& cap = g_smem_cap[key];
  cap = std::max(cap, bytes);
  return PTX_OK;
}

void clear_smem_cache() {
  std::lock_guard<std::mutex> lock(g_smem_mutex);
  g_smem_cap.clear();
}

bool pdl_enabled() {
  static const bool on = [] {
    const char* v = std::getenv("PTYCHOX_PDL");
    return !(v && v[0] == '0');
  }();
  return on;
}

RowShape row_shape(const LinePlan& p, int rows_available) {
  RowShape s;
  int lines = 256 / p.threads;
  if (lines < 1) lines = 1;
  if (lines > rows_available) lines = rows_available;
  if (lines < 1) lines = 1;
  s.lines = lines;
  s.threads = ((lines * p.threads + 31) / 32) * 32;
  s.smem = lines * line_pitch(p.n) * static_cast<int>(sizeof(float2));
  return s;
}

ColShape col_shape(const LinePlan& p) {
  ColShape s;
  s.cols = kTile;
  while (s.cols > 1 && s.cols * p.threads > 512) s.cols /= 2;
  s.threads = ((s.cols * p.threads + 31) / 32) * 32;
  s.smem = s.cols * line_pitch(p.n) * static_cast<int>(sizeof(float2));
  return s;
}

namespace {
const char* const kKernelNames[kNumKernelIds] = {
    "base_rows_forward", "base_cols", "base_rows_adjoint", "fpm_rows_forward", "fpm_cols",
    "fpm_rows_adjoint", "fft2_rows", "fft2_cols", "coded_rows", "coded_cols", "misc",
    "subpix_cols",      "subpix_rows"};

struct Profiler {
  std::mutex mu;
  bool on = false;
  std::vector<cudaEvent_t> pool;
  struct Pending { int id; cudaEvent_t a, b; };
  std::vector<Pending> pending;
  cudaEvent_t open_start[kNumKernelIds] = {};
  double total_ms[kNumKernelIds] = {};
  long long timed[kNumKernelIds] = {};
};
Profiler g_prof;
std::atomic<long long> g_launches[kNumKernelIds];

cudaEvent_t take_event() {
  if (!g_prof.pool.empty()) {
    cudaEvent_t e = g_prof.pool.back();
    g_prof.pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}
}  // namespace

void prof_begin(int id, cudaStream_t s) {
  g_launches[id].fetch_add(1, std::memory_order_relaxed);
  if (!g_prof.on) return;
  std::lock_guard<std::mutex> lock(g_prof.mu);
  cudaEvent_t e = take_event();
  cudaEventRecord(e, s);
  g_prof.open_start[id] = e;
}

void prof_end(int id, cudaStream_t s) {
  if (!g_prof.on) return;
  std::lock_guard<std::mutex> lock(g_prof.mu);
  if (!g_prof.open_start[id]) return;
  cudaEvent_t e = take_event();
  cudaEventRecord(e, s);
  g_prof.pending.push_back({id, g_prof.open_start[id], e});
  g_prof.open_start[id] = nullptr;
}

int sm_count() {
  int dev = 0, n = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) {
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  }
  return n > 0 ? n : 148;
}

struct ResidentKey {
  int dev, threads, smem;
  const void* kernel;
  bool operator<(const ResidentKey& o) const {
    return std::tie(dev, threads, smem, kernel) < std::tie(o.dev, o.threads, o.smem, o.kernel);
  }
};
std::mutex g_resident_mutex;
std::map<ResidentKey, int> g_resident;

int resident_ctas(const void* kernel, int threads, int smem) {
  int dev = 0;
  cudaGetDevice(&dev);
  const ResidentKey key{dev, threads, smem, kernel};
  {
    std::lock_guard<std::mutex> lock(g_resident_mutex);
    auto it = g_resident.find(key);
    if (it != g_resident.end()) return it->second;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess) {
    cudaGetLastError();
    per_sm = 1;
  }
  const int n = std::max(1, per_sm) * sm_count();
  std::lock_guard<std::mutex> lock(g_resident_mutex);
  g_resident[key] = n;
  return n;
}

std::atomic<int> g_units_per_cta{0};
thread_local int t_units_per_cta = -1;  // this thread's bound (-1: the process-wide one)

int units_per_cta() {
  return t_units_per_cta >= 0 ? t_units_per_cta : g_units_per_cta.load(std::memory_order_relaxed);
}

int set_thread_units_per_cta(int units) {
  const int prev = t_units_per_cta;
  t_units_per_cta = units < 0 ? -1 : units;
  return prev;
}

int persistent_grid(const void* kernel, int threads, int smem, long long units) {
  long long grid = std::min<long long>(units, resident_ctas(kernel, threads, smem));
  const int k = units_per_cta();
  if (k > 0) grid = std::max(grid, (units + k - 1) / k);
  return static_cast<int>(std::max<long long>(1, std::min<long long>(grid, std::max<long long>(units, 1))));
}

// Device copy of page-locked host memory, read over the bus with loads that never hit a
// stale cached line of system memory (ld.global.cv).  Grid-stride; 8-byte words when both
// ends are 8-byte aligned, bytes otherwise.
__global__ void stage_host_kernel(unsigned char* __restrict__ dst, const unsigned char* __restrict__ src,
                                  size_t bytes) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t i0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (((reinterpret_cast<uintptr_t>(dst) | reinterpret_cast<uintptr_t>(src)) & 7) == 0) {
    const size_t n8 = bytes / 8;
    auto* d8 = reinterpret_cast<unsigned long long*>(dst);
    const auto* s8 = reinterpret_cast<const unsigned long long*>(src);
    for (size_t i = i0; i < n8; i += stride) d8[i] = __ldcv(s8 + i);
    for (size_t i = n8 * 8 + i0; i < bytes; i += stride) dst[i] = __ldcv(src + i);
  } else {
    for (size_t i = i0; i < bytes; i += stride) dst[i] = __ldcv(src + i);
  }
}

// ---- staging ring for small host inputs -------------------------------------------------
// One page-locked, device-mapped ring of kStageRingBytes per device.  stage_host copies the
// caller's bytes into the next span of the ring (the caller may reuse its memory at once),
// launches stage_host_kernel to read the span into `dst` on the stream and records the
// span's event after it.  A span is reused only after its event has completed (normally
// long before the ring wraps round to it; otherwise the host waits on that event).  The
// whole sequence runs under one lock, so every span in the ring has its event recorded.
constexpr size_t kStageRingBytes = 1u << 20;
constexpr size_t kStageMaxBytes = kStageRingBytes / 4;  // larger inputs take cudaMemcpyAsync

struct StageRing {
  unsigned char* host = nullptr;
  unsigned char* device = nullptr;
  size_t head = 0;
  struct Span {
    size_t off, len;
    cudaEvent_t done;
  };
  std::deque<Span> live;
  std::vector<cudaEvent_t> spare;
};
std::mutex g_stage_mutex;
std::map<int, StageRing> g_stage;

// PTX_OK with *staged = false when the ring cannot take the copy (too large, or no ring on
// this device): the caller copies instead.
int stage_host(void* dst, const void* src, size_t bytes, cudaStream_t s, bool* staged) {
  *staged = false;
  if (bytes > kStageMaxBytes) return PTX_OK;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return cuda_status(cudaGetLastError(), "cudaGetDevice");
  std::lock_guard<std::mutex> lock(g_stage_mutex);
  StageRing& r = g_stage[dev];
  if (!r.host) {
    void* h = nullptr;
    if (cudaHostAlloc(&h, kStageRingBytes, cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess) {
      cudaGetLastError();
      return PTX_OK;
    }
    void* d = nullptr;
    if (cudaHostGetDevicePointer(&d, h, 0) != cudaSuccess || !d) {
      cudaGetLastError();
      cudaFreeHost(h);
      return PTX_OK;
    }
    r.host = static_cast<unsigned char*>(h);
    r.device = static_cast<unsigned char*>(d);
  }
  // retire completed spans from the oldest end, then wait for any live span the new one overlaps
  while (!r.live.empty()) {
    if (cudaEventQuery(r.live.front().done) != cudaSuccess) {
      cudaGetLastError();
      break;
    }
    r.spare.push_back(r.live.front().done);
    r.live.pop_front();
  }
  const size_t off = r.head + bytes > kStageRingBytes ? 0 : r.head;
  for (const StageRing::Span& sp : r.live) {
    if (sp.off < off + bytes && off < sp.off + sp.len && cudaEventSynchronize(sp.done) != cudaSuccess) {
      return cuda_status(cudaGetLastError(), "staging ring wait");
    }
  }
  cudaEvent_t ev = nullptr;
  if (!r.spare.empty()) {
    ev = r.spare.back();
    r.spare.pop_back();
  } else if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
    return cuda_status(cudaGetLastError(), "cudaEventCreate");
  }
  std::memcpy(r.host + off, src, bytes);
  const size_t words = (bytes + 7) / 8;
  const unsigned grid = static_cast<unsigned>(std::min<size_t>((words + 255) / 256, 1024));
  prof_begin(kMiscKernel, s);
  stage_host_kernel<<<grid, 256, 0, s>>>(static_cast<unsigned char*>(dst), r.device + off, bytes);
  prof_end(kMiscKernel, s);
  const cudaError_t launched = cudaGetLastError();
  const cudaError_t recorded = launched == cudaSuccess ? cudaEventRecord(ev, s) : launched;
  if (recorded != cudaSuccess) {
    r.spare.push_back(ev);
    return cuda_status(recorded, "ptx_stage_host_bytes launch");
  }
  r.live.push_back({off, bytes, ev});
  r.head = (off + bytes + 15) / 16 * 16;
  *staged = true;
  return PTX_OK;
}

}  // namespace ptx

extern "C" {

int ptx_stage_host_bytes(void* dst, const void* src, size_t bytes, void* stream) {
  if (bytes == 0) return PTX_OK;
  if (!dst || !src) return ptx::set_error(PTX_ERR_INVALID_ARGUMENT, "null pointer argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // a stream being captured into a CUDA graph gets a copy node that re-reads `src` on every
  // replay (a ring span would be filled once, at capture, and later reused)
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &capture) != cudaSuccess) {
    cudaGetLastError();
    capture = cudaStreamCaptureStatusActive;
  }
  bool staged = false;
  if (capture == cudaStreamCaptureStatusNone) {
    if (int st = ptx::stage_host(dst, src, bytes, s, &staged)) return st;
  }
  if (staged) return PTX_OK;
  return ptx::cuda_status(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, s), "ptx_stage_host_bytes copy");
}

int ptx_set_units_per_cta(int units) {
  if (units < 0) return ptx::set_error(PTX_ERR_INVALID_ARGUMENT, "units per CTA must be >= 0");
  ptx::g_units_per_cta.store(units, std::memory_order_relaxed);
  return PTX_OK;
}

int ptx_set_thread_units_per_cta(int units) {
  ptx::set_thread_units_per_cta(units);
  return PTX_OK;
}

int ptx_get_units_per_cta(void) { return ptx::units_per_cta(); }

int ptx_version(void) { return 200; }  // 0.2.0

const char* ptx_last_error(void) { return ptx::g_last_error.c_str(); }

int ptx_clear_cache(void) {
  std::lock_guard<std::mutex> lock(ptx::g_plan_mutex);
  // Table offsets stay assigned: a table is rebuilt with identical contents at the same
  // place, so kernels still in flight never see another length's table.
  ptx::g_plans.clear();
  ptx::clear_noalloc_cache();
  ptx::clear_smem_cache();
  return PTX_OK;
}

long long ptx_launch_count(void) {
  long long n = 0;
  for (int i = 0; i < ptx::kNumKernelIds; ++i) n += ptx::g_launches[i].load(std::memory_order_relaxed);
  return n;
}

int ptx_profile_enable(int on) {
  std::lock_guard<std::mutex> lock(ptx::g_prof.mu);
  ptx::g_prof.on = on != 0;
  return PTX_OK;
}

int ptx_profile_reset(void) {
  std::lock_guard<std::mutex> lock(ptx::g_prof.mu);
  for (auto& p : ptx::g_prof.pending) {
    ptx::g_prof.pool.push_back(p.a);
    ptx::g_prof.pool.push_back(p.b);
  }
  ptx::g_prof.pending.clear();
  for (int i = 0; i < ptx::kNumKernelIds; ++i) {
    ptx::g_prof.total_ms[i] = 0.0;
    ptx::g_prof.timed[i] = 0;
  }
  return PTX_OK;
}

int ptx_profile_read(int kernel_id, double* total_ms, long long* launches) {
  if (kernel_id < 0 || kernel_id >= ptx::kNumKernelIds || !total_ms || !launches) {
    return ptx::set_error(PTX_ERR_INVALID_ARGUMENT, "bad kernel id");
  }
  std::lock_guard<std::mutex> lock(ptx::g_prof.mu);
  for (auto& p : ptx::g_prof.pending) {
    if (int st = ptx::cuda_status(cudaEventSynchronize(p.b), "cudaEventSynchronize")) return st;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, p.a, p.b);
    ptx::g_prof.total_ms[p.id] += ms;
    ptx::g_prof.timed[p.id] += 1;
    ptx::g_prof.pool.push_back(p.a);
    ptx::g_prof.pool.push_back(p.b);
  }
  ptx::g_prof.pending.clear();
  *total_ms = ptx::g_prof.total_ms[kernel_id];
  *launches = ptx::g_prof.timed[kernel_id];
  return PTX_OK;
}

int ptx_profile_kinds(void) { return ptx::kNumKernelIds; }

const char* ptx_profile_name(int kernel_id) {
  if (kernel_id < 0 || kernel_id >= ptx::kNumKernelIds) return "";
  return ptx::kKernelNames[kernel_id];
}

int ptx_fft_supported(int n) { return ptx::size_supported(n) ? 1 : 0; }

int ptx_fft_engine(int n) {
  if (!ptx::size_supported(n)) return 0;
  if (n >= 16 && (n & (n - 1)) == 0) return 1;
  return ptx::mix_ops(n) ? 2 : 3;
}

int ptx_fft_prepare(int n) {
  ptx::LinePlan p;
  return ptx::get_line_plan(n, &p);
}

}  // extern "C"
