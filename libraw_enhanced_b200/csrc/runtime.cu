// runtime.cu -- multi-image execution on one GPU: the batch runner (many
// images per call, pipelined over several streams, optionally one CUDA graph
// per batch), its autotuner, and the request server (continuous batching
// under a device-memory budget).
//
// Neither exists in the reference, whose accelerator develops one image per
// synchronous call (core/accelerator.cpp, core/libraw_wrapper.cpp:1477-1853).
// Each image still runs the reference's per-image chain (develop_device in
// pipeline.cu); only the scheduling around it is new:
//   * a lane = one stream, one workspace arena and resident device buffers
//     for a mosaic and a result; a lane runs its images in order, lanes run
//     concurrently, so uploads and downloads of one lane overlap the kernels
//     of another (copy engines and SMs work at the same time);
//   * images are assigned to lanes largest-first onto the least-loaded lane;
//   * the batch runner can capture the whole batch (every lane's copies and
//     kernels, forked from and joined to one stream) as one CUDA graph and
//     replay it while the batch signature repeats;
//   * the server admits queued requests onto idle lanes while the resident
//     bytes of all lanes stay within the budget, and signals completion from
//     a host callback on the lane stream.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <mutex>
#include <numeric>
#include <thread>
#include <unordered_map>

#include "lre_internal.h"

namespace lre {
namespace {

using Clock = std::chrono::steady_clock;

double ms_since(Clock::time_point t0, Clock::time_point t1) {
  return std::chrono::duration<double, std::milli>(t1 - t0).count();
}

size_t out_bytes_of(const lre_image& im) {
  return im.width * im.height * 3 * (im.params.output_bits == 16 ? 2 : 4);
}
size_t mosaic_bytes_of(const lre_image& im) { return im.width * im.height * 4; }

// Device bytes one image holds on a lane: mosaic + result + chain workspace.
size_t image_device_bytes(const lre_image& im) {
  return ((mosaic_bytes_of(im) + 4095) & ~size_t(4095)) + ((out_bytes_of(im) + 4095) & ~size_t(4095)) +
         ((develop_ws_bytes(im.params, im.width, im.height) + 255) & ~size_t(255));
}

struct Lane {
  Context* c = nullptr;
  void* d_mos = nullptr;
  size_t mos_cap = 0;
  void* d_out = nullptr;
  size_t out_cap = 0;
  cudaEvent_t join = nullptr;

  size_t resident() const { return mos_cap + out_cap + c->ws.capacity(); }
};

lre_status lane_open(Lane& l, int device, const Tuning& t) {
  lre_ctx* ctx = nullptr;
  lre_status st = lre_create(device, &ctx);
  if (st != LRE_OK) return st;
  l.c = reinterpret_cast<Context*>(ctx);
  l.c->tune = t;
  if (cudaEventCreateWithFlags(&l.join, cudaEventDisableTiming) != cudaSuccess) return LRE_ERR_CUDA;
  return LRE_OK;
}

void lane_close(Lane& l) {
  if (!l.c) return;
  cudaSetDevice(l.c->device);
  cudaStreamSynchronize(l.c->stream);
  if (l.d_mos) cudaFree(l.d_mos);
  if (l.d_out) cudaFree(l.d_out);
  if (l.join) cudaEventDestroy(l.join);
  lre_destroy(reinterpret_cast<lre_ctx*>(l.c));
  l = Lane();
}

// Grow the lane's resident buffers and workspace to hold `im` (host mode
// needs the mosaic/result buffers; device mode only the workspace).
lre_status lane_fit(Lane& l, const lre_image& im, bool host_mode) {
  Context* c = l.c;
  if (host_mode) {
    LRE_TRY(ensure_buffer(c, &l.d_mos, &l.mos_cap, mosaic_bytes_of(im)));
    LRE_TRY(ensure_buffer(c, &l.d_out, &l.out_cap, out_bytes_of(im)));
  }
  LRE_CUDA_TRY(c, c->ws.reserve(develop_ws_bytes(im.params, im.width, im.height), c->stream));
  return LRE_OK;
}

void lane_release(Lane& l) {
  cudaStreamSynchronize(l.c->stream);
  if (l.d_mos) cudaFree(l.d_mos);
  if (l.d_out) cudaFree(l.d_out);
  l.d_mos = l.d_out = nullptr;
  l.mos_cap = l.out_cap = 0;
  l.c->ws.release();
}

// Enqueue one image on a lane (buffers already fitted).
lre_status lane_enqueue(Lane& l, const lre_image& im, bool host_mode) {
  Context* c = l.c;
  if (!host_mode) return develop_device(c, im.mosaic, im.out, im.width, im.height, im.params);
  LRE_CUDA_TRY(c, cudaMemcpyAsync(l.d_mos, im.mosaic, mosaic_bytes_of(im), cudaMemcpyHostToDevice, c->stream));
  LRE_TRY(develop_device(c, reinterpret_cast<const float*>(l.d_mos), l.d_out, im.width, im.height, im.params));
  LRE_CUDA_TRY(c, cudaMemcpyAsync(im.out, l.d_out, out_bytes_of(im), cudaMemcpyDeviceToHost, c->stream));
  return LRE_OK;
}

// Page-lock pageable host buffers for the duration of a call.
struct HostPins {
  std::vector<void*> pinned;
  cudaError_t pin(const void* p, size_t bytes) {
    cudaPointerAttributes a;
    cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) cudaGetLastError();
    if (e == cudaSuccess && a.type != cudaMemoryTypeUnregistered) return cudaSuccess;
    e = cudaHostRegister(const_cast<void*>(p), bytes, cudaHostRegisterDefault);
    if (e == cudaErrorHostMemoryAlreadyRegistered) {
      cudaGetLastError();
      return cudaSuccess;
    }
    if (e == cudaSuccess) pinned.push_back(const_cast<void*>(p));
    return e;
  }
  void release() {
    for (void* p : pinned) cudaHostUnregister(p);
    pinned.clear();
  }
  ~HostPins() { release(); }
};

// Largest-first onto the least-loaded lane; returns per-lane image lists in
// execution order.
std::vector<std::vector<size_t>> assign_lanes(const lre_image* im, size_t n, int lanes) {
  std::vector<size_t> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
    return im[a].width * im[a].height > im[b].width * im[b].height;
  });
  std::vector<std::vector<size_t>> out(lanes);
  std::vector<size_t> load(lanes, 0);
  for (size_t i : order) {
    int best = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    out[best].push_back(i);
    load[best] += im[i].width * im[i].height;
  }
  return out;
}

}  // namespace

// ------------------------------------------------------------------ batch
struct Batch {
  lre_batch_config cfg{};
  Tuning tune;
  int lanes = 3;
  bool tuned = false;
  std::vector<Lane> L;
  cudaStream_t main = nullptr;
  cudaEvent_t fork = nullptr;
  std::string err;
  std::vector<unsigned char> sig;
  cudaGraphExec_t exec = nullptr;
  uint64_t graph_launches = 0;

  lre_status fail_msg(lre_status st, const std::string& m) {
    err = m;
    return st;
  }
};

namespace {

lre_status batch_set_lanes(Batch* b, int lanes) {
  lanes = std::max(1, std::min(lanes, 8));
  while ((int)b->L.size() > lanes) {
    lane_close(b->L.back());
    b->L.pop_back();
  }
  while ((int)b->L.size() < lanes) {
    b->L.emplace_back();
    lre_status st = lane_open(b->L.back(), b->cfg.device, b->tune);
    if (st != LRE_OK) {
      b->L.pop_back();
      return b->fail_msg(st, "batch: cannot create a lane context");
    }
  }
  for (auto& l : b->L) l.c->tune = b->tune;
  b->lanes = lanes;
  return LRE_OK;
}

void drop_graph(Batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;
  b->sig.clear();
}

std::vector<unsigned char> batch_signature(const Batch* b, const lre_image* im, size_t n, bool host_mode) {
  std::vector<unsigned char> s;
  auto put = [&](const void* p, size_t k) {
    const unsigned char* q = reinterpret_cast<const unsigned char*>(p);
    s.insert(s.end(), q, q + k);
  };
  put(&n, sizeof(n));
  put(&b->lanes, sizeof(int));
  put(&b->tune, sizeof(Tuning));
  put(&host_mode, sizeof(bool));
  for (size_t i = 0; i < n; i++) put(&im[i], sizeof(lre_image));
  return s;
}

// Enqueue every image on its lane; the caller synchronises (eager) or ends
// the capture (graph).
lre_status enqueue_all(Batch* b, const lre_image* im, const std::vector<std::vector<size_t>>& plan, bool host_mode,
                       uint64_t* launches) {
  uint64_t before = 0;
  for (auto& l : b->L) before += l.c->launches.load();
  // round-robin over lanes so every stream receives work early
  size_t maxlen = 0;
  for (auto& p : plan) maxlen = std::max(maxlen, p.size());
  for (size_t k = 0; k < maxlen; k++) {
    for (int li = 0; li < b->lanes; li++) {
      if (k >= plan[li].size()) continue;
      lre_status st = lane_enqueue(b->L[li], im[plan[li][k]], host_mode);
      if (st != LRE_OK) return b->fail_msg(st, std::string("batch: ") + b->L[li].c->last_error);
    }
  }
  uint64_t after = 0;
  for (auto& l : b->L) after += l.c->launches.load();
  *launches = after - before;
  return LRE_OK;
}

lre_status run_eager(Batch* b, const lre_image* im, size_t n, bool host_mode, uint64_t* launches) {
  auto plan = assign_lanes(im, n, b->lanes);
  for (int li = 0; li < b->lanes; li++)
    for (size_t i : plan[li]) {
      lre_status st = lane_fit(b->L[li], im[i], host_mode);
      if (st != LRE_OK) return b->fail_msg(st, std::string("batch: ") + b->L[li].c->last_error);
    }
  LRE_TRY(enqueue_all(b, im, plan, host_mode, launches));
  for (auto& l : b->L) {
    cudaError_t e = cudaStreamSynchronize(l.c->stream);
    if (e != cudaSuccess) return b->fail_msg(LRE_ERR_CUDA, std::string("batch: ") + cudaGetErrorString(e));
  }
  return LRE_OK;
}

lre_status run_graph(Batch* b, const lre_image* im, size_t n, bool host_mode, int* graph_state, uint64_t* launches) {
  std::vector<unsigned char> sig = batch_signature(b, im, n, host_mode);
  if (!b->exec || sig != b->sig) {
    drop_graph(b);
    auto plan = assign_lanes(im, n, b->lanes);
    for (int li = 0; li < b->lanes; li++)
      for (size_t i : plan[li]) {
        lre_status st = lane_fit(b->L[li], im[i], host_mode);
        if (st != LRE_OK) return b->fail_msg(st, std::string("batch: ") + b->L[li].c->last_error);
      }
    for (auto& l : b->L) cudaStreamSynchronize(l.c->stream);
    cudaError_t e = cudaStreamBeginCapture(b->main, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return b->fail_msg(LRE_ERR_CUDA, std::string("batch: begin capture: ") + cudaGetErrorString(e));
    cudaEventRecord(b->fork, b->main);
    for (auto& l : b->L) cudaStreamWaitEvent(l.c->stream, b->fork, 0);
    lre_status st = enqueue_all(b, im, plan, host_mode, launches);
    for (auto& l : b->L) {
      cudaEventRecord(l.join, l.c->stream);
      cudaStreamWaitEvent(b->main, l.join, 0);
    }
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(b->main, &g);
    if (st != LRE_OK) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      return st;
    }
    if (e != cudaSuccess || !g) return b->fail_msg(LRE_ERR_CUDA, std::string("batch: end capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      b->exec = nullptr;
      return b->fail_msg(LRE_ERR_CUDA, std::string("batch: instantiate: ") + cudaGetErrorString(e));
    }
    b->sig = std::move(sig);
    b->graph_launches = *launches;
    *graph_state = 1;
  } else {
    *launches = b->graph_launches;
    *graph_state = 2;
  }
  cudaError_t e = cudaGraphLaunch(b->exec, b->main);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->main);
  if (e != cudaSuccess) return b->fail_msg(LRE_ERR_CUDA, std::string("batch: graph launch: ") + cudaGetErrorString(e));
  return LRE_OK;
}

// ---------------------------------------------------------------- autotune
// Times the kernel-shape choices on the batch's largest image (device
// resident on lane 0) and, for host-buffer batches, the lane count on the
// first images of the batch; keeps the fastest of each.
float time_stream(cudaStream_t s, const std::function<lre_status()>& fn, int reps, lre_status* st) {
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  *st = fn();  // warm-up
  cudaEventRecord(e0, s);
  for (int i = 0; i < reps && *st == LRE_OK; i++) *st = fn();
  cudaEventRecord(e1, s);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ms / reps;
}

lre_status autotune(Batch* b, const lre_image* im, size_t n, bool host_mode) {
  size_t big = 0;
  for (size_t i = 1; i < n; i++)
    if (im[i].width * im[i].height > im[big].width * im[big].height) big = i;
  const lre_image& ref = im[big];
  Lane& l = b->L[0];
  Context* c = l.c;
  const size_t w = ref.width, h = ref.height;
  const size_t rgb = ((w * h * 12) + 255) & ~size_t(255);
  // lane 0 holds: mosaic, two RGB planes, and the stage workspace after them
  lre_image dev = ref;
  float *d_mos = nullptr, *d_a = nullptr, *d_b = nullptr;
  if (cudaMalloc(&d_mos, w * h * 4) != cudaSuccess || cudaMalloc(&d_a, rgb) != cudaSuccess ||
      cudaMalloc(&d_b, rgb) != cudaSuccess) {
    cudaFree(d_mos);
    cudaFree(d_a);
    cudaFree(d_b);
    cudaGetLastError();
    return b->fail_msg(LRE_ERR_OUT_OF_MEMORY, "batch autotune: cannot allocate the trial buffers");
  }
  auto cleanup = [&]() {
    cudaStreamSynchronize(c->stream);
    cudaFree(d_mos);
    cudaFree(d_a);
    cudaFree(d_b);
  };
  cudaMemcpyAsync(d_mos, ref.mosaic, w * h * 4, host_mode ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, c->stream);
  {
    lre_develop_params all = ref.params;  // room for every stage that is timed
    all.defringe = 1;
    all.axial_ca_correction = 1;
    LRE_CUDA_TRY(c, c->ws.reserve(develop_ws_bytes(all, w, h), c->stream));
  }
  c->ws.reset();
  lre_status st = launch_amaze(c, d_mos, 1, d_a, w, h, ref.params.filters == LRE_FILTERS_XTRANS ? 0x94949494u : ref.params.filters,
                               ref.params.cam_mul, ref.params.maximum_value);
  c->ws.reset();
  if (st != LRE_OK) {
    cleanup();
    return b->fail_msg(st, "batch autotune: " + c->last_error);
  }
  const lre_develop_params& p = ref.params;
  Tuning best = b->tune;
  // guided filter variants
  {
    const int cand[4][2] = {{128, 128}, {128, 64}, {64, 128}, {64, 64}};
    float best_ms = 1e30f;
    float* dmax = c->d_scalars + 1;
    for (auto& v : cand) {
      c->tune.axial_strip = v[0];
      c->tune.axial_rows = v[1];
      float ms = time_stream(c->stream, [&]() -> lre_status {
        const size_t mark = c->ws.used();
        LRE_TRY(launch_channel_max(c, d_a, w * h, 1, dmax, true));
        lre_status s2 = launch_axial_ca(c, d_a, d_b, w, h, p.axial_ca_radius, p.axial_ca_epsilon, p.axial_ca_strength, dmax);
        c->ws.rewind(mark);
        return s2;
      }, 2, &st);
      if (st != LRE_OK) break;
      if (ms < best_ms) {
        best_ms = ms;
        best.axial_strip = v[0];
        best.axial_rows = v[1];
      }
    }
  }
  // defringe blur tile
  if (st == LRE_OK) {
    float best_ms = 1e30f;
    for (int t : {32, 64}) {
      c->tune.blur_tile = t;
      float ms = time_stream(c->stream, [&]() -> lre_status {
        const size_t mark = c->ws.used();
        lre_status s2 = launch_defringe(c, d_a, d_b, w, h, p.defringe_radius, p.defringe_edge_threshold,
                                        p.defringe_chroma_threshold, p.defringe_strength, p.defringe_green != 0,
                                        p.defringe_green_strength, nullptr);
        c->ws.rewind(mark);
        return s2;
      }, 2, &st);
      if (st != LRE_OK) break;
      if (ms < best_ms) {
        best_ms = ms;
        best.blur_tile = t;
      }
    }
  }
  cleanup();
  if (st != LRE_OK) return b->fail_msg(st, "batch autotune: " + c->last_error);
  b->tune = best;
  for (auto& ln : b->L) ln.c->tune = best;
  // lane count: eager runs of the first images (host mode only: the lanes
  // exist to overlap copies with kernels)
  if (host_mode && b->cfg.lanes <= 0 && n >= 4) {
    const size_t k = std::min<size_t>(n, 8);
    double best_ms = 1e30;
    int best_l = b->lanes;
    for (int lanes : {2, 3, 4}) {
      LRE_TRY(batch_set_lanes(b, lanes));
      uint64_t lc = 0;
      auto t0 = Clock::now();
      LRE_TRY(run_eager(b, im, k, host_mode, &lc));
      double ms = ms_since(t0, Clock::now());
      if (ms < best_ms) {
        best_ms = ms;
        best_l = lanes;
      }
    }
    LRE_TRY(batch_set_lanes(b, best_l));
  }
  b->tuned = true;
  return LRE_OK;
}

lre_status batch_validate(Batch* b, const lre_image* im, size_t n) {
  if (!im && n) return b->fail_msg(LRE_ERR_INVALID_ARGUMENT, "batch: null image array");
  for (size_t i = 0; i < n; i++) {
    if (!im[i].mosaic || !im[i].out) return b->fail_msg(LRE_ERR_INVALID_ARGUMENT, "batch: null buffer in image " + std::to_string(i));
    lre_status st = develop_validate(b->L[0].c, &im[i].params, im[i].width, im[i].height);
    if (st != LRE_OK) return b->fail_msg(st, "batch: image " + std::to_string(i) + ": " + b->L[0].c->last_error);
  }
  return LRE_OK;
}

lre_status batch_run(Batch* b, const lre_image* im, size_t n, lre_batch_stats* stats, bool host_mode) {
  auto t0 = Clock::now();
  cudaSetDevice(b->cfg.device);
  LRE_TRY(batch_validate(b, im, n));
  lre_batch_stats s{};
  if (n == 0) {
    if (stats) *stats = s;
    return LRE_OK;
  }
  HostPins pins;
  if (host_mode) {
    for (size_t i = 0; i < n; i++) {
      if (pins.pin(im[i].mosaic, mosaic_bytes_of(im[i])) != cudaSuccess ||
          pins.pin(im[i].out, out_bytes_of(im[i])) != cudaSuccess)
        return b->fail_msg(LRE_ERR_OUT_OF_MEMORY, "batch: cannot page-lock host buffer of image " + std::to_string(i));
    }
  }
  if (b->cfg.autotune && !b->tuned) {
    auto ta = Clock::now();
    drop_graph(b);
    LRE_TRY(autotune(b, im, n, host_mode));
    s.tune_ms = ms_since(ta, Clock::now());
  }
  uint64_t launches = 0;
  // A captured graph keeps the host addresses of its copies; host buffers
  // that this call page-locks are unlocked again on return, so a graph is
  // only built (and replayed) when every host buffer was already
  // page-locked by the caller.
  if (b->cfg.use_graph && (!host_mode || pins.pinned.empty())) {
    LRE_TRY(run_graph(b, im, n, host_mode, &s.graph, &launches));
  } else {
    LRE_TRY(run_eager(b, im, n, host_mode, &launches));
  }
  s.lanes = b->lanes;
  s.launches = launches;
  s.ms = ms_since(t0, Clock::now());
  if (stats) *stats = s;
  return LRE_OK;
}

}  // namespace

// ------------------------------------------------------------------ server
struct Request {
  uint64_t ticket = 0;
  lre_image img{};
  size_t bytes = 0;
  lre_decode_fn decode = nullptr;  // fills img.mosaic on a decode thread first
  void* user = nullptr;
  Clock::time_point t_submit, t_ready, t_admit, t_done;  // t_ready: joined the device queue
  lre_status status = LRE_OK;
  int lane = -1;
  bool done = false;
  HostPins pins;
};

struct Server {
  lre_server_config cfg{};
  std::vector<Lane> L;
  std::vector<Request*> running;  // per lane
  std::vector<char> finished;     // per lane: completion callback fired
  std::mutex mu;
  std::condition_variable cv_sched, cv_done;
  std::deque<Request*> queue;     // ready for a lane
  std::deque<Request*> decode_q;  // waiting for a decode thread
  int decoding = 0;               // decode callbacks running
  std::condition_variable cv_decode;
  std::vector<std::thread> decoders;
  std::unordered_map<uint64_t, Request*> reqs;
  uint64_t next_ticket = 1;
  size_t resident = 0, peak = 0;
  bool stop = false;
  std::thread sched;
  std::string err;
  Context vctx;  // holds validation messages of submit (never launches)
};

namespace {

struct DoneArg {
  Server* s;
  int lane;
};

void CUDART_CB on_lane_done(void* p) {
  DoneArg* a = static_cast<DoneArg*>(p);
  {
    std::lock_guard<std::mutex> lk(a->s->mu);
    a->s->finished[a->lane] = 1;
  }
  a->s->cv_sched.notify_one();
  delete a;
}

size_t server_resident(const Server* s) {
  size_t r = 0;
  for (auto& l : s->L) r += l.resident();
  return r;
}

// Completes finished lanes; caller holds the lock.
void reap(Server* s) {
  for (size_t li = 0; li < s->L.size(); li++) {
    if (!s->finished[li] || !s->running[li]) continue;
    Request* r = s->running[li];
    cudaError_t e = cudaStreamQuery(s->L[li].c->stream);
    if (e != cudaSuccess && e != cudaErrorNotReady) r->status = LRE_ERR_CUDA;
    r->t_done = Clock::now();
    r->done = true;
    s->running[li] = nullptr;
    s->finished[li] = 0;
    s->cv_done.notify_all();
  }
}

void scheduler(Server* s) {
  cudaSetDevice(s->cfg.device);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    reap(s);
    bool any_running = std::any_of(s->running.begin(), s->running.end(), [](Request* r) { return r != nullptr; });
    if (s->stop && s->queue.empty() && !any_running && s->decode_q.empty() && s->decoding == 0) break;
    // admit FIFO while a lane is idle and the budget holds
    bool admitted = false;
    while (!s->queue.empty()) {
      int li = -1;
      for (size_t k = 0; k < s->L.size(); k++)
        if (!s->running[k]) {
          li = (int)k;
          break;
        }
      if (li < 0) break;
      Request* r = s->queue.front();
      Lane& l = s->L[li];
      const size_t cur = server_resident(s);
      size_t need = cur - l.resident() + std::max(l.resident(), r->bytes);
      if (need > s->cfg.device_budget_bytes) {
        // free the buffers of idle lanes (other than li) and retry
        for (size_t k = 0; k < s->L.size(); k++)
          if (!s->running[k] && (int)k != li && s->L[k].resident()) lane_release(s->L[k]);
        need = server_resident(s) - l.resident() + std::max(l.resident(), r->bytes);
        if (need > s->cfg.device_budget_bytes) {
          if (l.resident() > r->bytes) lane_release(l);
          need = server_resident(s) - l.resident() + std::max(l.resident(), r->bytes);
        }
        if (need > s->cfg.device_budget_bytes) break;  // wait for a running request to finish
      }
      s->queue.pop_front();
      r->t_admit = Clock::now();
      r->lane = li;
      s->running[li] = r;
      admitted = true;
      lk.unlock();
      lre_status st = lane_fit(l, r->img, true);
      if (st == LRE_OK) st = lane_enqueue(l, r->img, true);
      if (st == LRE_OK) {
        DoneArg* a = new DoneArg{s, li};
        if (cudaLaunchHostFunc(l.c->stream, on_lane_done, a) != cudaSuccess) {
          delete a;
          st = LRE_ERR_CUDA;
        }
      }
      if (st != LRE_OK) cudaStreamSynchronize(l.c->stream);  // no completion callback is pending
      lk.lock();
      s->resident = server_resident(s);
      s->peak = std::max(s->peak, s->resident);
      if (st != LRE_OK) {
        r->status = st;
        r->t_done = Clock::now();
        r->done = true;
        s->running[li] = nullptr;
        s->err = l.c->last_error;
        s->cv_done.notify_all();
      }
    }
    if (!admitted) s->cv_sched.wait(lk);
  }
}

// Decode thread: runs queued decode callbacks (FIFO) outside the lock and
// moves each decoded request to the device queue.  Drains its queue before
// it stops, so destroying the server finishes every submitted request.
void decoder(Server* s) {
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    s->cv_decode.wait(lk, [&] { return s->stop || !s->decode_q.empty(); });
    if (s->decode_q.empty()) break;  // stopping, nothing left
    Request* r = s->decode_q.front();
    s->decode_q.pop_front();
    s->decoding++;
    lk.unlock();
    const lre_status st = r->decode(r->user, const_cast<float*>(r->img.mosaic), r->img.width, r->img.height);
    lk.lock();
    s->decoding--;
    r->t_ready = Clock::now();
    if (st != LRE_OK) {
      r->status = st;
      r->t_admit = r->t_done = r->t_ready;
      r->done = true;
      s->err = "server: the decode callback returned an error";
      s->cv_done.notify_all();
    } else {
      s->queue.push_back(r);
    }
    s->cv_sched.notify_one();
  }
}

// Validation, budget check and page-locking shared by both submit forms.
lre_status prepare_request(Server* s, const lre_image* img, Request** out) {
  if (!img->mosaic || !img->out) {
    std::lock_guard<std::mutex> lk(s->mu);
    s->err = "server: null buffer";
    return LRE_ERR_INVALID_ARGUMENT;
  }
  {
    std::lock_guard<std::mutex> lk(s->mu);
    lre_status st = develop_validate(&s->vctx, &img->params, img->width, img->height);
    if (st != LRE_OK) {
      s->err = "server: " + s->vctx.last_error;
      return st;
    }
  }
  Request* r = new Request();
  r->img = *img;
  r->bytes = image_device_bytes(*img);
  if (r->bytes > s->cfg.device_budget_bytes) {
    delete r;
    std::lock_guard<std::mutex> lk(s->mu);
    s->err = "server: request needs more device memory than the budget";
    return LRE_ERR_BUSY;
  }
  cudaSetDevice(s->cfg.device);
  if (r->pins.pin(img->mosaic, mosaic_bytes_of(*img)) != cudaSuccess ||
      r->pins.pin(img->out, out_bytes_of(*img)) != cudaSuccess) {
    delete r;
    std::lock_guard<std::mutex> lk(s->mu);
    s->err = "server: cannot page-lock the request's host buffers";
    return LRE_ERR_OUT_OF_MEMORY;
  }
  r->t_submit = r->t_ready = Clock::now();
  *out = r;
  return LRE_OK;
}

// Tickets the request and queues it (device queue, or the decode queue when
// it has a decode callback).
lre_status enqueue_request(Server* s, Request* r, uint64_t* ticket) {
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) {
      delete r;
      return LRE_ERR_BUSY;
    }
    r->ticket = s->next_ticket++;
    s->reqs[r->ticket] = r;
    (r->decode ? s->decode_q : s->queue).push_back(r);
    *ticket = r->ticket;
  }
  if (r->decode) s->cv_decode.notify_one();
  else s->cv_sched.notify_one();
  return LRE_OK;
}

}  // namespace

}  // namespace lre

using lre::Batch;
using lre::Context;
using lre::Server;

extern "C" {

lre_status lre_set_tuning(lre_ctx* ctx, const lre_tuning* t) {
  Context* c = reinterpret_cast<Context*>(ctx);
  if (!c || !t) return LRE_ERR_INVALID_ARGUMENT;
  if ((t->axial_strip != 128 && t->axial_strip != 64) || (t->axial_rows != 128 && t->axial_rows != 64) ||
      (t->blur_tile != 32 && t->blur_tile != 64))
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "set_tuning: axial_strip 128|64, axial_rows 128|64, blur_tile 32|64");
  c->tune.axial_strip = t->axial_strip;
  c->tune.axial_rows = t->axial_rows;
  c->tune.blur_tile = t->blur_tile;
  return LRE_OK;
}

lre_status lre_get_tuning(const lre_ctx* ctx, lre_tuning* t) {
  const Context* c = reinterpret_cast<const Context*>(ctx);
  if (!c || !t) return LRE_ERR_INVALID_ARGUMENT;
  t->lanes = 1;
  t->axial_strip = c->tune.axial_strip;
  t->axial_rows = c->tune.axial_rows;
  t->blur_tile = c->tune.blur_tile;
  return LRE_OK;
}

lre_status lre_batch_create(const lre_batch_config* cfg, lre_batch** out) {
  if (!cfg || !out) return LRE_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return LRE_ERR_NO_DEVICE;
  }
  if (cfg->device < 0 || cfg->device >= n) return LRE_ERR_INVALID_ARGUMENT;
  cudaSetDevice(cfg->device);
  Batch* b = new Batch();
  b->cfg = *cfg;
  if (cudaStreamCreateWithFlags(&b->main, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess) {
    delete b;
    return LRE_ERR_CUDA;
  }
  lre_status st = lre::batch_set_lanes(b, cfg->lanes > 0 ? cfg->lanes : 3);
  if (st != LRE_OK) {
    lre_batch_destroy(reinterpret_cast<lre_batch*>(b));
    return st;
  }
  *out = reinterpret_cast<lre_batch*>(b);
  return LRE_OK;
}

void lre_batch_destroy(lre_batch* bp) {
  Batch* b = reinterpret_cast<Batch*>(bp);
  if (!b) return;
  cudaSetDevice(b->cfg.device);
  lre::drop_graph(b);
  for (auto& l : b->L) lre::lane_close(l);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->main) cudaStreamDestroy(b->main);
  delete b;
}

const char* lre_batch_last_error(const lre_batch* bp) {
  const Batch* b = reinterpret_cast<const Batch*>(bp);
  return b ? b->err.c_str() : "null batch";
}

lre_status lre_batch_run(lre_batch* bp, const lre_image* images, size_t n, lre_batch_stats* stats) {
  Batch* b = reinterpret_cast<Batch*>(bp);
  if (!b) return LRE_ERR_INVALID_ARGUMENT;
  return lre::batch_run(b, images, n, stats, true);
}

lre_status lre_dev_batch_run(lre_batch* bp, const lre_image* images, size_t n, lre_batch_stats* stats) {
  Batch* b = reinterpret_cast<Batch*>(bp);
  if (!b) return LRE_ERR_INVALID_ARGUMENT;
  return lre::batch_run(b, images, n, stats, false);
}

lre_status lre_batch_get_tuning(const lre_batch* bp, lre_tuning* t) {
  const Batch* b = reinterpret_cast<const Batch*>(bp);
  if (!b || !t) return LRE_ERR_INVALID_ARGUMENT;
  t->lanes = b->lanes;
  t->axial_strip = b->tune.axial_strip;
  t->axial_rows = b->tune.axial_rows;
  t->blur_tile = b->tune.blur_tile;
  return LRE_OK;
}

lre_status lre_batch_set_tuning(lre_batch* bp, const lre_tuning* t) {
  Batch* b = reinterpret_cast<Batch*>(bp);
  if (!b || !t) return LRE_ERR_INVALID_ARGUMENT;
  if ((t->axial_strip != 128 && t->axial_strip != 64) || (t->axial_rows != 128 && t->axial_rows != 64) ||
      (t->blur_tile != 32 && t->blur_tile != 64) || t->lanes < 1 || t->lanes > 8)
    return b->fail_msg(LRE_ERR_INVALID_ARGUMENT, "batch_set_tuning: lanes 1..8, axial_strip 128|64, axial_rows 128|64, blur_tile 32|64");
  cudaSetDevice(b->cfg.device);
  lre::drop_graph(b);
  b->tune.axial_strip = t->axial_strip;
  b->tune.axial_rows = t->axial_rows;
  b->tune.blur_tile = t->blur_tile;
  b->tuned = true;
  return lre::batch_set_lanes(b, t->lanes);
}

lre_status lre_server_create(const lre_server_config* cfg, lre_server** out) {
  if (!cfg || !out) return LRE_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return LRE_ERR_NO_DEVICE;
  }
  if (cfg->device < 0 || cfg->device >= n) return LRE_ERR_INVALID_ARGUMENT;
  cudaSetDevice(cfg->device);
  Server* s = new Server();
  s->cfg = *cfg;
  if (s->cfg.lanes <= 0) s->cfg.lanes = 4;
  s->cfg.lanes = std::min(s->cfg.lanes, 16);
  if (s->cfg.device_budget_bytes == 0) s->cfg.device_budget_bytes = size_t(150) * 1000 * 1000 * 1000;
  s->L.resize(s->cfg.lanes);
  for (auto& l : s->L) {
    lre_status st = lre::lane_open(l, cfg->device, lre::Tuning());
    if (st != LRE_OK) {
      for (auto& q : s->L) lre::lane_close(q);
      delete s;
      return st;
    }
  }
  s->running.assign(s->cfg.lanes, nullptr);
  s->finished.assign(s->cfg.lanes, 0);
  if (s->cfg.decode_threads <= 0) s->cfg.decode_threads = 2;
  s->cfg.decode_threads = std::min(s->cfg.decode_threads, 16);
  s->sched = std::thread(lre::scheduler, s);
  for (int i = 0; i < s->cfg.decode_threads; i++) s->decoders.emplace_back(lre::decoder, s);
  *out = reinterpret_cast<lre_server*>(s);
  return LRE_OK;
}

void lre_server_destroy(lre_server* sp) {
  Server* s = reinterpret_cast<Server*>(sp);
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_sched.notify_all();
  s->cv_decode.notify_all();
  for (auto& t : s->decoders) t.join();  // the decode queue is drained first
  if (s->sched.joinable()) s->sched.join();
  cudaSetDevice(s->cfg.device);
  for (auto& l : s->L) lre::lane_close(l);
  for (auto& kv : s->reqs) delete kv.second;
  delete s;
}

const char* lre_server_last_error(const lre_server* sp) {
  const Server* s = reinterpret_cast<const Server*>(sp);
  return s ? s->err.c_str() : "null server";
}

lre_status lre_server_submit(lre_server* sp, const lre_image* img, uint64_t* ticket) {
  Server* s = reinterpret_cast<Server*>(sp);
  if (!s || !img || !ticket) return LRE_ERR_INVALID_ARGUMENT;
  lre::Request* r = nullptr;
  LRE_TRY(lre::prepare_request(s, img, &r));
  return lre::enqueue_request(s, r, ticket);
}

lre_status lre_server_submit_decode(lre_server* sp, const lre_image* img, lre_decode_fn decode, void* user,
                                    uint64_t* ticket) {
  Server* s = reinterpret_cast<Server*>(sp);
  if (!s || !img || !ticket || !decode) return LRE_ERR_INVALID_ARGUMENT;
  lre::Request* r = nullptr;
  LRE_TRY(lre::prepare_request(s, img, &r));
  r->decode = decode;
  r->user = user;
  return lre::enqueue_request(s, r, ticket);
}

lre_status lre_server_wait(lre_server* sp, uint64_t ticket, double timeout_ms, lre_request_stats* stats) {
  Server* s = reinterpret_cast<Server*>(sp);
  if (!s) return LRE_ERR_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return LRE_ERR_INVALID_ARGUMENT;
  lre::Request* r = it->second;
  auto ready = [&]() { return r->done; };
  if (timeout_ms < 0) {
    s->cv_done.wait(lk, ready);
  } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), ready)) {
    return LRE_ERR_TIMEOUT;
  }
  if (stats) {
    stats->status = r->status;
    stats->lane = r->lane;
    stats->queue_ms = lre::ms_since(r->t_ready, r->t_admit);
    stats->run_ms = lre::ms_since(r->t_admit, r->t_done);
    stats->total_ms = lre::ms_since(r->t_submit, r->t_done);
    stats->device_bytes = r->bytes;
    stats->decode_ms = r->decode ? lre::ms_since(r->t_submit, r->t_ready) : 0.0;
  }
  lre_status st = r->status;
  s->reqs.erase(it);
  lk.unlock();
  delete r;  // unpins its host buffers
  return st;
}

lre_status lre_server_memory(const lre_server* sp, size_t* in_use, size_t* peak) {
  const Server* s = reinterpret_cast<const Server*>(sp);
  if (!s) return LRE_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(const_cast<Server*>(s)->mu);
  if (in_use) *in_use = s->resident;
  if (peak) *peak = s->peak;
  return LRE_OK;
}

}  // extern "C"
