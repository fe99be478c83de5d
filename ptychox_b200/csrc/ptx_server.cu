// Reconstruction server: continuous batching of whole reconstructions on one GPU.
//
// The native counterpart of the reference drivers' training loop run for many problems at
// once (python/train_ptychography.py:473-603, train_fpm.py, train_coded.py: a sweep per
// iteration, F.mse_loss, torch.optim.Adam).  A request carries one problem (object,
// probe / pupil / coded surface, scan, counts, schedule); the server copies it at submit,
// admits requests first come first served while their resident bytes fit the HBM budget,
// and keeps each admitted reconstruction's state on the device: parameters, gradients,
// Adam moments, counts, scan and workspace in one allocation from the server's own
// stream-ordered pool (kept mapped between reconstructions).  One iteration
// (fused sweep + one Adam step of each parameter) is captured once per reconstruction as a
// CUDA graph, with the persistent passes bounded to 8 units per CTA at capture so the
// kernels of concurrent reconstructions interleave CTA by CTA.  Two threads share the work:
//   - the scheduler thread only replays: each tick it queues the next iteration of every
//     active reconstruction on that reconstruction's stream (older reconstructions on
//     higher-priority streams, at most two iterations queued per stream) and polls events,
//     so it never waits on the device;
//   - the admission thread does everything that blocks: it admits queued requests first
//     come first served within the budget and slot count (allocation, upload, a warm-up
//     sweep that also gives the initial loss, capture, instantiation) and hands the ready
//     reconstruction to the scheduler, and it reads back and frees finished ones.
// A request may stop early at a fixed error: once the loss of a completed iteration falls
// to target_ratio times the initial loss, no further iteration is queued (the iterations
// already queued still run).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "ptx_internal.h"

namespace ptx {
namespace {

using Clock = std::chrono::steady_clock;

constexpr size_t kServerWorkspaceCap = 512ull << 20;  // workspace per reconstruction (longer scans chunk)
constexpr int kServerUnitsPerCta = 8;
constexpr int kServerMaxInflight = 2;
constexpr float kAdamBeta1 = 0.9f, kAdamBeta2 = 0.999f, kAdamEps = 1e-16f;

size_t align256(size_t v) { return (v + 255) / 256 * 256; }

struct Request {
  long long id = 0;
  ptx_recon_request d{};
  std::vector<unsigned char> obj0, aux0, scan, meas, t1, t2;
  size_t ws_bytes = 0, bytes = 0;
  Clock::time_point submitted, finished;
  int status = 0;  // 0 queued, 1 active, 2 done, < 0: -(error code)
  double final_loss = NAN;
  int iterations = 0;  // iterations run (fewer than d.iters when the error target was met)
  std::vector<unsigned char> obj_out, aux_out;
};

struct Slot {
  Request* req = nullptr;
  cudaStream_t stream = nullptr;
  void* base = nullptr;
  float *obj = nullptr, *aux = nullptr, *g_obj = nullptr, *g_aux = nullptr;
  float *m_obj = nullptr, *v_obj = nullptr, *m_aux = nullptr, *v_aux = nullptr;
  void *st_obj = nullptr, *st_aux = nullptr, *scan = nullptr, *ws = nullptr;
  uint16_t* meas = nullptr;
  float *t1 = nullptr, *t2 = nullptr;
  double* loss = nullptr;
  cudaGraphExec_t exec = nullptr;
  int launched = 0;
  int limit = 0;                // iterations to queue (d.iters, or fewer once the target is met)
  double target = -1.0;         // stop once a completed iteration's loss is <= target
  double* loss_host = nullptr;  // page-locked: each replay copies its sweep loss here
  std::deque<cudaEvent_t> inflight;
  std::vector<cudaEvent_t> spare;
  cudaEvent_t done = nullptr;
};

struct Server {
  int device = 0;
  size_t budget = 0;
  int max_active = 8;
  // the server's own stream-ordered pool: memory freed by a finished reconstruction stays
  // mapped for the next one instead of returning to the system at every synchronisation
  cudaMemPool_t pool = nullptr;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Request*> queued;
  std::map<long long, std::unique_ptr<Request>> requests;
  long long next_id = 1;
  bool stop = false;
  // hand-over between the threads (under mu): reconstructions ready to run, finished ones
  // to read back, the slots and bytes held by admitted (or admitting) reconstructions
  std::deque<Slot> ready, finished;
  int slots_held = 0;
  size_t used = 0;
  bool scheduler_done = false;
  std::thread scheduler, admitter;
};

size_t obj_elems(const ptx_recon_request& d) { return (size_t)d.obj_h * d.obj_w; }
size_t aux_elems(const ptx_recon_request& d) { return (size_t)d.aux_h * d.aux_w; }
size_t count_elems(const ptx_recon_request& d) {
  if (d.modality == PTX_MODALITY_CODED || d.modality == PTX_MODALITY_NEARFIELD) {
    const size_t m = (size_t)(d.obj_h / d.downsample);
    return (size_t)d.batch * m * m;
  }
  return (size_t)d.batch * aux_elems(d);
}
bool coded_like(const ptx_recon_request& d) {
  return d.modality == PTX_MODALITY_CODED || d.modality == PTX_MODALITY_NEARFIELD;
}

size_t workspace_for(const ptx_recon_request& d) {
  if (d.modality == PTX_MODALITY_CONVENTIONAL) {
    const size_t frame = (size_t)num_tiles(d.aux_w) * kTile * d.aux_h * sizeof(float2);
    const size_t full = ptx_base_workspace_bytes(d.aux_h, d.aux_w, d.batch);
    return std::min(full, std::max(256 + frame, kServerWorkspaceCap));
  }
  if (d.modality == PTX_MODALITY_FOURIER) {
    const size_t full = ptx_fpm_workspace_bytes(d.obj_h, d.obj_w, d.aux_h, d.aux_w, d.batch);
    const size_t fixed = ptx_fpm_workspace_bytes(d.obj_h, d.obj_w, d.aux_h, d.aux_w, 1);
    return std::min(full, std::max(fixed, kServerWorkspaceCap));
  }
  const size_t full = ptx_coded_workspace_bytes(d.obj_h, d.batch);
  const size_t fixed = ptx_coded_workspace_bytes(d.obj_h, 1);
  return std::min(full, std::max(fixed, kServerWorkspaceCap));
}

// Resident bytes of an admitted reconstruction: the one allocation admit() carves up.
size_t slot_bytes(const Request& r) {
  const size_t po = align256(obj_elems(r.d) * sizeof(float2)), pa = align256(aux_elems(r.d) * sizeof(float2));
  return 4 * (po + pa)  // parameters, gradients and the two Adam moments of each
         + 3 * 256      // the two Adam states and the loss
         + align256(r.scan.size()) + align256(r.meas.size()) + align256(r.t1.size()) + align256(r.t2.size()) +
         align256(r.ws_bytes);
}

int run_sweep(const Slot& s) {
  const ptx_recon_request& d = s.req->d;
  if (d.modality == PTX_MODALITY_CONVENTIONAL) {
    // one CTA per frame for square 32 / 64 / 128 probes; for 128^2 frames only from 96 frames
    // up (one such CTA takes ~30 us per wave of frames, the three passes ~11 us + 0.21 us per
    // frame on a B200)
    const bool small = d.aux_h == d.aux_w &&
                       (d.aux_w == 32 || d.aux_w == 64 || (d.aux_w == 128 && d.batch >= 96));
    return (small ? ptx_base_sweep_small : ptx_base_sweep)(
        s.obj, d.obj_h, d.obj_w, s.aux, d.aux_h, d.aux_w, static_cast<const int64_t*>(s.scan), d.batch, s.meas,
        d.scale, s.loss, s.g_obj, s.g_aux, s.ws, s.req->ws_bytes, s.stream);
  }
  if (d.modality == PTX_MODALITY_FOURIER) {
    return ptx_fpm_sweep(s.obj, d.obj_h, d.obj_w, s.aux, d.aux_h, d.aux_w, static_cast<const int64_t*>(s.scan),
                         d.batch, s.meas, d.scale, s.loss, s.g_obj, s.g_aux, s.ws, s.req->ws_bytes, s.stream);
  }
  return ptx_coded_sweep(s.obj, s.aux, d.modality == PTX_MODALITY_CODED ? s.t1 : nullptr, s.t2, d.obj_h,
                         static_cast<const float*>(s.scan), d.batch, d.downsample, s.meas, d.scale, s.loss, s.g_obj,
                         s.g_aux, s.ws, s.req->ws_bytes, s.stream);
}

int run_iteration(const Slot& s) {
  const ptx_recon_request& d = s.req->d;
  if (int st = run_sweep(s)) return st;
  if (int st = ptx_adam_step(s.obj, s.g_obj, s.m_obj, s.v_obj, obj_elems(d), s.st_obj, d.lr_obj, kAdamBeta1,
                             kAdamBeta2, kAdamEps, d.constrain_obj, s.stream)) {
    return st;
  }
  return ptx_adam_step(s.aux, s.g_aux, s.m_aux, s.v_aux, aux_elems(d), s.st_aux, d.lr_aux, kAdamBeta1, kAdamBeta2,
                       kAdamEps, d.constrain_aux, s.stream);
}

void release(Slot& s) {
  if (s.stream) cudaStreamSynchronize(s.stream);
  if (s.loss_host) cudaFreeHost(s.loss_host);
  for (cudaEvent_t e : s.inflight) cudaEventDestroy(e);
  for (cudaEvent_t e : s.spare) cudaEventDestroy(e);
  s.inflight.clear();
  s.spare.clear();
  if (s.done) cudaEventDestroy(s.done);
  if (s.exec) cudaGraphExecDestroy(s.exec);
  if (s.base) cudaFreeAsync(s.base, s.stream);
  if (s.stream) {
    cudaStreamSynchronize(s.stream);
    cudaStreamDestroy(s.stream);
  }
  s = Slot{};
  cudaGetLastError();
}

// Allocate, upload, warm up and capture one reconstruction; PTX_OK or an error code.
int admit(Slot& s, Request* r, int priority, cudaMemPool_t pool) {
  s.req = r;
  const ptx_recon_request& d = r->d;
  if (cudaStreamCreateWithPriority(&s.stream, cudaStreamNonBlocking, priority) != cudaSuccess) {
    return cuda_status(cudaGetLastError(), "server stream");
  }
  const size_t po = align256(obj_elems(d) * sizeof(float2)), pa = align256(aux_elems(d) * sizeof(float2));
  const size_t total = slot_bytes(*r);
  if (cudaMallocFromPoolAsync(&s.base, total, pool, s.stream) != cudaSuccess) {
    return cuda_status(cudaGetLastError(), "server alloc");
  }
  char* p = static_cast<char*>(s.base);
  auto take = [&](size_t n) {
    char* q = p;
    p += align256(n);
    return q;
  };
  s.obj = reinterpret_cast<float*>(take(po));
  s.aux = reinterpret_cast<float*>(take(pa));
  s.g_obj = reinterpret_cast<float*>(take(po));
  s.g_aux = reinterpret_cast<float*>(take(pa));
  s.m_obj = reinterpret_cast<float*>(take(po));
  s.v_obj = reinterpret_cast<float*>(take(po));
  s.m_aux = reinterpret_cast<float*>(take(pa));
  s.v_aux = reinterpret_cast<float*>(take(pa));
  s.st_obj = take(256);
  s.st_aux = take(256);
  s.loss = reinterpret_cast<double*>(take(256));
  s.scan = take(r->scan.size());
  s.meas = reinterpret_cast<uint16_t*>(take(r->meas.size()));
  if (!r->t1.empty()) s.t1 = reinterpret_cast<float*>(take(r->t1.size()));
  if (!r->t2.empty()) s.t2 = reinterpret_cast<float*>(take(r->t2.size()));
  s.ws = take(r->ws_bytes);
  cudaStream_t st = s.stream;
  cudaMemcpyAsync(s.obj, r->obj0.data(), r->obj0.size(), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s.aux, r->aux0.data(), r->aux0.size(), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s.scan, r->scan.data(), r->scan.size(), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s.meas, r->meas.data(), r->meas.size(), cudaMemcpyHostToDevice, st);
  if (s.t1) cudaMemcpyAsync(s.t1, r->t1.data(), r->t1.size(), cudaMemcpyHostToDevice, st);
  if (s.t2) cudaMemcpyAsync(s.t2, r->t2.data(), r->t2.size(), cudaMemcpyHostToDevice, st);
  // Adam moments (contiguous m_obj .. v_aux), their states and the loss start at zero
  cudaMemsetAsync(s.m_obj, 0, 2 * po + 2 * pa + 3 * 256, st);
  if (cudaGetLastError() != cudaSuccess) return cuda_status(cudaGetLastError(), "server upload");
  if (cudaMallocHost(&s.loss_host, sizeof(double)) != cudaSuccess) {
    return cuda_status(cudaGetLastError(), "server host loss");
  }
  *s.loss_host = NAN;
  // one sweep outside the capture builds the FFT plans and kernel attributes; at the initial
  // parameters it is also the first iteration's sweep, whose loss sets the error target
  if (int e = run_sweep(s)) return e;
  double loss0 = NAN;
  cudaMemcpyAsync(&loss0, s.loss, sizeof(double), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return cuda_status(cudaGetLastError(), "server warm-up");
  s.limit = d.iters;
  s.target = d.target_ratio > 0.f ? (double)d.target_ratio * loss0 : -1.0;
  // the bound applies to this (scheduler) thread's launches only: another server's
  // scheduler, or the host program's own sweeps, keep theirs
  const int saved_units = set_thread_units_per_cta(kServerUnitsPerCta);
  cudaGraph_t graph = nullptr;
  int status = cuda_status(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "server capture");
  if (!status) {
    status = run_iteration(s);
    if (!status && s.target >= 0.0) {
      status = cuda_status(cudaMemcpyAsync(s.loss_host, s.loss, sizeof(double), cudaMemcpyDeviceToHost, st),
                           "server loss copy");
    }
    const cudaError_t end = cudaStreamEndCapture(st, &graph);
    if (!status && end != cudaSuccess) status = cuda_status(end, "server capture end");
  }
  set_thread_units_per_cta(saved_units);
  if (!status && cudaGraphInstantiate(&s.exec, graph, 0) != cudaSuccess) {
    status = cuda_status(cudaGetLastError(), "server graph instantiate");
  }
  if (graph) cudaGraphDestroy(graph);
  if (status) return status;
  if (cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming) != cudaSuccess) {
    return cuda_status(cudaGetLastError(), "server event");
  }
  return PTX_OK;
}

// Queue the next iteration unless kServerMaxInflight are still queued or the schedule is
// complete; true if launched.  With an error target, a completed iteration whose loss (copied
// to loss_host by the replay) is at or below it ends the schedule: the iterations already
// queued run and `done` is recorded behind them.
bool launch_next(Slot& s, int* err) {
  bool completed = false;
  while (!s.inflight.empty() && cudaEventQuery(s.inflight.front()) == cudaSuccess) {
    s.spare.push_back(s.inflight.front());
    s.inflight.pop_front();
    completed = true;
  }
  cudaGetLastError();
  if (completed && s.target >= 0.0 && s.launched < s.limit) {
    const double seen = *static_cast<volatile double*>(s.loss_host);
    if (seen <= s.target) {
      s.limit = s.launched;
      cudaEventRecord(s.done, s.stream);
    }
  }
  if (s.launched >= s.limit || (int)s.inflight.size() >= kServerMaxInflight) return false;
  if (cudaGraphLaunch(s.exec, s.stream) != cudaSuccess) {
    *err = cuda_status(cudaGetLastError(), "server graph launch");
    return false;
  }
  cudaEvent_t ev = nullptr;
  if (!s.spare.empty()) {
    ev = s.spare.back();
    s.spare.pop_back();
  } else if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
    *err = cuda_status(cudaGetLastError(), "server event");
    return false;
  }
  cudaEventRecord(ev, s.stream);
  s.inflight.push_back(ev);
  if (++s.launched == s.limit) cudaEventRecord(s.done, s.stream);
  return true;
}

// Read back a finished reconstruction; PTX_OK or an error code.
int collect(Slot& s) {
  Request* r = s.req;
  r->obj_out.resize(r->obj0.size());
  r->aux_out.resize(r->aux0.size());
  cudaMemcpyAsync(r->obj_out.data(), s.obj, r->obj_out.size(), cudaMemcpyDeviceToHost, s.stream);
  cudaMemcpyAsync(r->aux_out.data(), s.aux, r->aux_out.size(), cudaMemcpyDeviceToHost, s.stream);
  double loss = NAN;
  cudaMemcpyAsync(&loss, s.loss, sizeof(double), cudaMemcpyDeviceToHost, s.stream);
  if (cudaStreamSynchronize(s.stream) != cudaSuccess) return cuda_status(cudaGetLastError(), "server read-back");
  r->final_loss = loss;
  r->iterations = s.launched;
  return PTX_OK;
}

// Scheduler thread: replays only.  Takes ready reconstructions, queues one iteration per
// active reconstruction per tick, and passes finished (or failed) ones to the admission
// thread; it never synchronises with the device.
void schedule(Server* sv) {
  cudaSetDevice(sv->device);
  std::vector<Slot> active;
  for (;;) {
    {
      std::lock_guard<std::mutex> lock(sv->mu);
      while (!sv->ready.empty()) {
        active.push_back(sv->ready.front());
        sv->ready.pop_front();
      }
    }
    bool progressed = false;
    for (Slot& s : active) {
      int err = 0;
      progressed |= launch_next(s, &err);
      if (err) {
        std::lock_guard<std::mutex> lock(sv->mu);
        s.req->status = -err;
      }
    }
    for (size_t i = 0; i < active.size();) {
      Slot& s = active[i];
      bool failed;
      {
        std::lock_guard<std::mutex> lock(sv->mu);
        failed = s.req->status < 0;
      }
      if (!failed && !(s.launched == s.limit && cudaEventQuery(s.done) == cudaSuccess)) {
        cudaGetLastError();
        ++i;
        continue;
      }
      {
        std::lock_guard<std::mutex> lock(sv->mu);
        sv->finished.push_back(s);
      }
      sv->cv.notify_all();
      active.erase(active.begin() + i);
      progressed = true;
    }
    std::unique_lock<std::mutex> lock(sv->mu);
    if (sv->stop && sv->queued.empty() && sv->ready.empty() && active.empty() && sv->slots_held == 0) break;
    if (active.empty() && sv->ready.empty()) {
      sv->cv.wait_for(lock, std::chrono::milliseconds(5));
    } else if (!progressed) {
      lock.unlock();
      std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
  }
  std::lock_guard<std::mutex> lock(sv->mu);
  sv->scheduler_done = true;
  sv->cv.notify_all();
}

// Admission thread: everything that waits on the device.  Reads back and frees finished
// reconstructions (returning their bytes and slot), then admits queued requests first come
// first served within the budget and slot count, one at a time, and hands each ready
// reconstruction to the scheduler.
void admit_loop(Server* sv) {
  cudaSetDevice(sv->device);
  int least = 0, greatest = 0;
  cudaDeviceGetStreamPriorityRange(&least, &greatest);
  for (;;) {
    Slot done_slot;
    bool have_done = false;
    Request* r = nullptr;
    int prio = greatest;
    {
      std::unique_lock<std::mutex> lock(sv->mu);
      for (;;) {
        if (sv->stop) {
          for (Request* q : sv->queued) {
            q->status = -PTX_ERR_INVALID_ARGUMENT;  // cancelled
            q->finished = Clock::now();
          }
          sv->queued.clear();
        }
        if (!sv->finished.empty()) {
          done_slot = sv->finished.front();
          sv->finished.pop_front();
          have_done = true;
          break;
        }
        if (!sv->queued.empty() && sv->slots_held < sv->max_active &&
            (sv->used + sv->queued.front()->bytes <= sv->budget || sv->slots_held == 0)) {
          r = sv->queued.front();
          sv->queued.pop_front();
          r->status = 1;
          sv->used += r->bytes;
          prio = std::max(greatest, std::min(least, greatest + sv->slots_held));
          ++sv->slots_held;
          break;
        }
        if (sv->scheduler_done) return;
        sv->cv.wait_for(lock, std::chrono::milliseconds(5));
      }
    }
    if (have_done) {
      Request* q = done_slot.req;
      bool failed;
      {
        std::lock_guard<std::mutex> lock(sv->mu);
        failed = q->status < 0;
      }
      const int e = failed ? 0 : collect(done_slot);
      release(done_slot);
      {
        std::lock_guard<std::mutex> lock(sv->mu);
        q->status = failed ? q->status : (e ? -e : 2);
        q->finished = Clock::now();
        sv->used -= q->bytes;
        --sv->slots_held;
      }
      sv->cv.notify_all();
      continue;
    }
    Slot s;
    const int e = admit(s, r, prio, sv->pool);
    if (e) {
      release(s);
      std::lock_guard<std::mutex> lock(sv->mu);
      r->status = -e;
      r->finished = Clock::now();
      sv->used -= r->bytes;
      --sv->slots_held;
      sv->cv.notify_all();
      continue;
    }
    {
      std::lock_guard<std::mutex> lock(sv->mu);
      sv->ready.push_back(s);
    }
    sv->cv.notify_all();
  }
}

int validate(const ptx_recon_request& d) {
  if (d.modality < PTX_MODALITY_CONVENTIONAL || d.modality > PTX_MODALITY_NEARFIELD) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "unknown modality %d", d.modality);
  }
  if (d.obj_h <= 0 || d.obj_w <= 0 || d.aux_h <= 0 || d.aux_w <= 0 || d.batch <= 0 || d.iters <= 0) {
    return set_error(PTX_ERR_INVALID_ARGUMENT, "non-positive shape, batch or iteration count");
  }
  if (!d.obj0 || !d.aux0 || !d.scan || !d.measured) return set_error(PTX_ERR_INVALID_ARGUMENT, "null pointer argument");
  if (!(d.scale > 0.f)) return set_error(PTX_ERR_INVALID_ARGUMENT, "scale must be positive");
  if (coded_like(d)) {
    if (d.obj_h != d.obj_w || d.aux_h != d.obj_h || d.aux_w != d.obj_w) {
      return set_error(PTX_ERR_INVALID_ARGUMENT, "coded / near-field fields must be square and of one size");
    }
    if (d.downsample <= 0 || d.obj_h % d.downsample) {
      return set_error(PTX_ERR_INVALID_ARGUMENT, "downsample must divide the field side");
    }
    if (!d.transfer_2 || (d.modality == PTX_MODALITY_CODED && !d.transfer_1)) {
      return set_error(PTX_ERR_INVALID_ARGUMENT, "missing transfer function");
    }
  }
  if (!(d.target_ratio >= 0.f)) return set_error(PTX_ERR_INVALID_ARGUMENT, "target_ratio must be >= 0");
  for (int c : {d.constrain_obj, d.constrain_aux}) {
    if (c < PTX_CONSTRAIN_NONE || c > PTX_CONSTRAIN_REAL_NONNEGATIVE) {
      return set_error(PTX_ERR_INVALID_ARGUMENT, "unknown constraint %d", c);
    }
  }
  return PTX_OK;
}

template <typename T>
void copy_in(std::vector<unsigned char>& dst, const T* src, size_t bytes) {
  dst.resize(bytes);
  if (bytes) std::memcpy(dst.data(), src, bytes);
}

}  // namespace
}  // namespace ptx

using namespace ptx;

extern "C" {

int ptx_server_create(int device, size_t hbm_budget, int max_active, void** server) {
  if (!server) return set_error(PTX_ERR_INVALID_ARGUMENT, "null pointer argument");
  *server = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
    cudaGetLastError();
    return set_error(PTX_ERR_INVALID_ARGUMENT, "no CUDA device %d", device);
  }
  if (max_active <= 0) return set_error(PTX_ERR_INVALID_ARGUMENT, "max_active must be positive");
  auto* sv = new Server();
  sv->device = device;
  sv->max_active = max_active;
  if (hbm_budget == 0) {
    size_t free_b = 0, total_b = 0;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    cudaMemGetInfo(&free_b, &total_b);
    cudaSetDevice(prev);
    hbm_budget = free_b / 10 * 7;
  }
  sv->budget = hbm_budget;
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  if (cudaMemPoolCreate(&sv->pool, &props) != cudaSuccess) {
    delete sv;
    return cuda_status(cudaGetLastError(), "server memory pool");
  }
  unsigned long long keep = ~0ull;
  cudaMemPoolSetAttribute(sv->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  sv->scheduler = std::thread(schedule, sv);
  sv->admitter = std::thread(admit_loop, sv);
  *server = sv;
  return PTX_OK;
}

int ptx_server_submit(void* server, const ptx_recon_request* request, long long* id) {
  if (!server || !request || !id) return set_error(PTX_ERR_INVALID_ARGUMENT, "null pointer argument");
  auto* sv = static_cast<Server*>(server);
  const ptx_recon_request& d = *request;
  if (int st = validate(d)) return st;
  auto r = std::make_unique<Request>();
  r->d = d;
  const size_t no = obj_elems(d) * sizeof(float2), na = aux_elems(d) * sizeof(float2);
  copy_in(r->obj0, d.obj0, no);
  copy_in(r->aux0, d.aux0, na);
  copy_in(r->scan, static_cast<const unsigned char*>(d.scan), (size_t)d.batch * 2 * (coded_like(d) ? 4 : 8));
  copy_in(r->meas, d.measured, count_elems(d) * sizeof(uint16_t));
  if (coded_like(d)) {
    if (d.modality == PTX_MODALITY_CODED) copy_in(r->t1, d.transfer_1, no);
    copy_in(r->t2, d.transfer_2, no);
  }
  if (d.modality == PTX_MODALITY_CONVENTIONAL) {
    // windows must lie inside the object, as the Python operators check on the host
    const int64_t* pos = reinterpret_cast<const int64_t*>(r->scan.data());
    for (int b = 0; b < d.batch; ++b) {
      const int64_t x = pos[2 * b], y = pos[2 * b + 1];
      if (x < 0 || y < 0 || x + d.aux_w > d.obj_w || y + d.aux_h > d.obj_h) {
        return set_error(PTX_ERR_OUT_OF_BOUNDS, "position %d: a %d x %d window at (%lld, %lld) leaves the %d x %d object",
                         b, d.aux_h, d.aux_w, (long long)x, (long long)y, d.obj_h, d.obj_w);
      }
    }
  }
  r->d.obj0 = r->d.aux0 = r->d.transfer_1 = r->d.transfer_2 = nullptr;
  r->d.scan = nullptr;
  r->d.measured = nullptr;
  r->ws_bytes = workspace_for(d);
  r->bytes = slot_bytes(*r);
  if (r->bytes > sv->budget) {
    return set_error(PTX_ERR_WORKSPACE, "request needs %zu resident bytes, more than the %zu-byte budget", r->bytes,
                     sv->budget);
  }
  r->submitted = Clock::now();
  {
    std::lock_guard<std::mutex> lock(sv->mu);
    if (sv->stop) return set_error(PTX_ERR_INVALID_ARGUMENT, "server is shutting down");
    r->id = sv->next_id++;
    *id = r->id;
    sv->queued.push_back(r.get());
    sv->requests[r->id] = std::move(r);
  }
  sv->cv.notify_all();
  return PTX_OK;
}

int ptx_server_poll(void* server, long long id, int* done, double* final_loss, double* latency_s, float* object_out,
                    float* aux_out) {
  return ptx_server_poll_ex(server, id, done, final_loss, latency_s, nullptr, object_out, aux_out);
}

int ptx_server_poll_ex(void* server, long long id, int* done, double* final_loss, double* latency_s, int* iterations,
                       float* object_out, float* aux_out) {
  if (!server || !done) return set_error(PTX_ERR_INVALID_ARGUMENT, "null pointer argument");
  auto* sv = static_cast<Server*>(server);
  std::lock_guard<std::mutex> lock(sv->mu);
  auto it = sv->requests.find(id);
  if (it == sv->requests.end()) return set_error(PTX_ERR_INVALID_ARGUMENT, "unknown request %lld", id);
  Request& r = *it->second;
  *done = 0;
  if (r.status == 0 || r.status == 1) return PTX_OK;
  if (r.status < 0) {
    const int code = -r.status;
    sv->requests.erase(it);
    return set_error(code, "request %lld failed (status %d)", id, code);
  }
  *done = 1;
  if (final_loss) *final_loss = r.final_loss;
  if (latency_s) *latency_s = std::chrono::duration<double>(r.finished - r.submitted).count();
  if (iterations) *iterations = r.iterations;
  if (object_out) std::memcpy(object_out, r.obj_out.data(), r.obj_out.size());
  if (aux_out) std::memcpy(aux_out, r.aux_out.data(), r.aux_out.size());
  sv->requests.erase(it);
  return PTX_OK;
}

int ptx_server_destroy(void* server) {
  if (!server) return PTX_OK;
  auto* sv = static_cast<Server*>(server);
  {
    std::lock_guard<std::mutex> lock(sv->mu);
    sv->stop = true;
  }
  sv->cv.notify_all();
  if (sv->scheduler.joinable()) sv->scheduler.join();
  if (sv->admitter.joinable()) sv->admitter.join();
  if (sv->pool) cudaMemPoolDestroy(sv->pool);
  delete sv;
  return PTX_OK;
}

}  // extern "C"
