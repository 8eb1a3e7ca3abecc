// host_stage.cu -- host <-> device copies for the host-buffer entry points.
//
// The reference's accelerator takes ImageBuffer / ImageBufferFloat over
// ordinary (pageable) host memory (core/accelerator.h:59-80; its Metal path
// wraps page-aligned vectors without a copy).  A cudaMemcpy from pageable
// memory goes through the driver's own small staging buffer, one piece at a
// time, and runs far below the PCIe rate.  Page-locking the caller's buffer
// on every call (cudaHostRegister) costs about as much as the copy.
//
// So a pageable buffer of more than a few MB is copied through a ring of
// pinned chunks owned by the context: the DMA of one chunk overlaps the host
// memcpy of the next, and each host memcpy is split over a small pool of
// worker threads (one thread alone moves ~10 GB/s, below the link).
//   * host -> device: memcpy into a free chunk, then an async DMA on the
//     caller's stream; returns once every chunk has been enqueued (the
//     caller's buffer may be reused at once, as after a pageable
//     cudaMemcpyAsync);
//   * device -> host: DMAs into up to kRing chunks ahead, each memcpy'd out
//     as its event completes; returns when the data is in the caller's
//     buffer.
// Page-locked (or registered) buffers and small copies take the direct
// cudaMemcpyAsync path.
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "lre_internal.h"

namespace lre {

namespace {

constexpr size_t kChunk = size_t(16) << 20;   // bytes per pinned chunk
constexpr int kRing = 4;                      // pinned chunks per context
constexpr size_t kDirectBelow = size_t(4) << 20;  // small copies: direct

}  // namespace

// Worker pool that splits one memcpy over its threads.
class HostStager {
 public:
  explicit HostStager(int threads) {
    for (int i = 0; i < threads; i++) workers_.emplace_back([this, i] { run(i); });
  }
  ~HostStager() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
    for (int k = 0; k < kRing; k++) {
      if (ev_[k]) cudaEventDestroy(ev_[k]);
      if (buf_[k]) cudaFreeHost(buf_[k]);
    }
  }

  // Pinned ring on the current device (allocated once).
  cudaError_t ensure_ring() {
    if (buf_[0]) return cudaSuccess;
    for (int k = 0; k < kRing; k++) {
      cudaError_t e = cudaHostAlloc(&buf_[k], kChunk, cudaHostAllocDefault);
      if (e != cudaSuccess) return e;
      e = cudaEventCreateWithFlags(&ev_[k], cudaEventDisableTiming);
      if (e != cudaSuccess) return e;
      busy_[k] = false;
    }
    return cudaSuccess;
  }

  // memcpy(dst, src, n) over the calling thread and the workers.
  void copy(void* dst, const void* src, size_t n) {
    const int parts = (int)workers_.size() + 1;
    const size_t piece = ((n + parts - 1) / parts + 63) & ~size_t(63);
    {
      std::lock_guard<std::mutex> lk(mu_);
      job_dst_ = static_cast<char*>(dst);
      job_src_ = static_cast<const char*>(src);
      job_n_ = n;
      job_piece_ = piece;
      pending_ = (int)workers_.size();
      gen_++;
    }
    cv_.notify_all();
    const size_t n0 = std::min(n, piece);  // part 0 on the calling thread
    if (n0) std::memcpy(dst, src, n0);
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [this] { return pending_ == 0; });
  }

  char* buf(int k) { return static_cast<char*>(buf_[k]); }
  cudaEvent_t ev(int k) { return ev_[k]; }
  bool busy_[kRing] = {false, false, false, false};

 private:
  void run(int idx) {
    unsigned long long seen = 0;
    for (;;) {
      char* d;
      const char* s;
      size_t n, piece;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
        d = job_dst_;
        s = job_src_;
        n = job_n_;
        piece = job_piece_;
      }
      const size_t lo = std::min(n, piece * (size_t)(idx + 1)), hi = std::min(n, lo + piece);
      if (hi > lo) std::memcpy(d + lo, s + lo, hi - lo);
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (--pending_ == 0) done_cv_.notify_one();
      }
    }
  }

  std::vector<std::thread> workers_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  bool stop_ = false;
  unsigned long long gen_ = 0;
  int pending_ = 0;
  char* job_dst_ = nullptr;
  const char* job_src_ = nullptr;
  size_t job_n_ = 0, job_piece_ = 0;
  void* buf_[kRing] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t ev_[kRing] = {nullptr, nullptr, nullptr, nullptr};
};

void destroy_stager(Context* c) {
  delete c->stager;
  c->stager = nullptr;
}

namespace {

bool is_pageable(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return a.type == cudaMemoryTypeUnregistered;
}

lre_status stager(Context* c, HostStager** out) {
  if (!c->stager) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    c->stager = new HostStager((int)std::min(7u, hw > 1 ? hw / 2 : 0u));
  }
  LRE_CUDA_TRY(c, c->stager->ensure_ring());
  *out = c->stager;
  return LRE_OK;
}

}  // namespace

lre_status copy_h2d(Context* c, void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes < kDirectBelow || !is_pageable(src)) {
    LRE_CUDA_TRY(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    return LRE_OK;
  }
  HostStager* st;
  LRE_TRY(stager(c, &st));
  int k = 0;
  for (size_t off = 0; off < bytes; off += kChunk, k = (k + 1) % kRing) {
    const size_t n = std::min(kChunk, bytes - off);
    if (st->busy_[k]) LRE_CUDA_TRY(c, cudaEventSynchronize(st->ev(k)));  // its previous DMA is done
    st->copy(st->buf(k), static_cast<const char*>(src) + off, n);
    LRE_CUDA_TRY(c, cudaMemcpyAsync(static_cast<char*>(dst) + off, st->buf(k), n, cudaMemcpyHostToDevice, s));
    LRE_CUDA_TRY(c, cudaEventRecord(st->ev(k), s));
    st->busy_[k] = true;
  }
  return LRE_OK;
}

lre_status copy_d2h(Context* c, void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes < kDirectBelow || !is_pageable(dst)) {
    LRE_CUDA_TRY(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
    LRE_CUDA_TRY(c, cudaStreamSynchronize(s));
    return LRE_OK;
  }
  HostStager* st;
  LRE_TRY(stager(c, &st));
  const size_t nchunks = (bytes + kChunk - 1) / kChunk;
  // chunk j uses ring slot j % kRing; a slot still holding an upload's data
  // is reused only after that DMA has finished
  auto issue = [&](size_t j) -> lre_status {
    const int k = (int)(j % kRing);
    if (st->busy_[k]) LRE_CUDA_TRY(c, cudaEventSynchronize(st->ev(k)));
    const size_t off = j * kChunk, n = std::min(kChunk, bytes - off);
    LRE_CUDA_TRY(c, cudaMemcpyAsync(st->buf(k), static_cast<const char*>(src) + off, n, cudaMemcpyDeviceToHost, s));
    LRE_CUDA_TRY(c, cudaEventRecord(st->ev(k), s));
    st->busy_[k] = true;
    return LRE_OK;
  };
  for (size_t j = 0; j < std::min(nchunks, (size_t)kRing); j++) LRE_TRY(issue(j));
  for (size_t j = 0; j < nchunks; j++) {
    const int k = (int)(j % kRing);
    LRE_CUDA_TRY(c, cudaEventSynchronize(st->ev(k)));
    const size_t off = j * kChunk, n = std::min(kChunk, bytes - off);
    st->copy(static_cast<char*>(dst) + off, st->buf(k), n);
    st->busy_[k] = false;
    if (j + kRing < nchunks) LRE_TRY(issue(j + kRing));
  }
  return LRE_OK;
}

}  // namespace lre
