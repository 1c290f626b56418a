// Staged copies between pageable host arrays and the device (hos_stage.h).
//
// A pageable cudaMemcpyAsync is staged by the driver through its own pinned
// buffers with one host thread; the reference's driver passes its whole
// packed state (two complex fields, 16.8 MB at 1024^2) this way twice per
// sol_update_RK call.  Here the host side of the staging is split over
// several threads and overlapped with the copy engine, chunk by chunk.
#include <algorithm>
#include <condition_variable>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <system_error>
#include <thread>
#include <vector>

#include "hos_stage.h"

namespace hos {
namespace {

constexpr size_t STAGE_MIN = 1u << 20;    // smaller copies go straight to the driver
constexpr size_t PART_MIN = 256u << 10;   // smallest piece one copy thread takes

int env_int(const char* name, int dflt) {
  const char* s = getenv(name);
  return (s && *s) ? atoi(s) : dflt;
}

// ------------------------------------------------------------ copy threads
// A job is a list of parts; every thread (the caller's included) claims the
// next part under the lock, copies it without the lock and counts it done.
// The pool lives until the process ends and its threads are detached: no
// join at exit, and a process forked from this one (which has none of the
// threads) still finishes every copy on the caller's thread.
class CopyPool {
 public:
  void copy(unsigned char* dst, const unsigned char* src, size_t bytes) {
    const int nt = threads();
    size_t parts = std::min<size_t>((size_t)nt, std::max<size_t>(1, bytes / PART_MIN));
    if (parts <= 1) {
      memcpy(dst, src, bytes);
      return;
    }
    std::lock_guard<std::mutex> job(job_m_);  // one job at a time
    start(nt - 1);
    size_t piece = (bytes + parts - 1) / parts;
    piece = (piece + 4095) & ~(size_t)4095;
    parts = (bytes + piece - 1) / piece;
    {
      std::lock_guard<std::mutex> lk(m_);
      dst_ = dst;
      src_ = src;
      bytes_ = bytes;
      piece_ = piece;
      nparts_ = parts;
      next_ = 0;
      done_ = 0;
      gen_++;
    }
    cv_.notify_all();
    work(gen_);
    std::unique_lock<std::mutex> lk(m_);
    done_cv_.wait(lk, [&] { return done_ == nparts_; });
  }

 private:
  int threads() {
    if (nthreads_ == 0) {
      const int hw = (int)std::thread::hardware_concurrency();
      nthreads_ = std::max(1, env_int("HOS_COPY_THREADS", std::min(8, std::max(1, hw))));
    }
    return nthreads_;
  }

  void start(int workers) {
    std::lock_guard<std::mutex> lk(m_);
    while (started_ < workers) {
      const unsigned long long g = gen_;
      try {
        std::thread([this, g] { loop(g); }).detach();
      } catch (const std::system_error&) {
        return;  // no more threads: the caller's thread takes the parts
      }
      started_++;
    }
  }

  [[noreturn]] void loop(unsigned long long seen) {
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(m_);
        cv_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
      }
      work(seen);
    }
  }

  // Copies parts of job `g` until none is left (or a newer job replaced it).
  void work(unsigned long long g) {
    for (;;) {
      unsigned char* d;
      const unsigned char* s;
      size_t n;
      {
        std::lock_guard<std::mutex> lk(m_);
        if (gen_ != g || next_ >= nparts_) return;
        const size_t off = next_ * piece_;
        next_++;
        d = dst_ + off;
        s = src_ + off;
        n = std::min(piece_, bytes_ - off);
      }
      memcpy(d, s, n);
      bool last;
      {
        std::lock_guard<std::mutex> lk(m_);
        last = ++done_ == nparts_;
      }
      if (last) done_cv_.notify_all();
    }
  }

  std::mutex job_m_;
  std::mutex m_;
  std::condition_variable cv_, done_cv_;
  int started_ = 0;
  int nthreads_ = 0;
  unsigned long long gen_ = 0;
  unsigned char* dst_ = nullptr;
  const unsigned char* src_ = nullptr;
  size_t bytes_ = 0, piece_ = 0, nparts_ = 0, next_ = 0, done_ = 0;
};

CopyPool& pool() {
  static CopyPool* p = new CopyPool;  // never destroyed (see above)
  return *p;
}

// ------------------------------------------------------------ staging buffers
struct Stager {
  std::mutex m;
  size_t chunk = 0;
  unsigned char* pin[2] = {nullptr, nullptr};
  bool failed = false;  // pinned allocation failed: copies go to the driver
  std::vector<cudaEvent_t> ev;  // two per device, created on first use
};

Stager& stager() {
  static Stager* s = new Stager;  // lives until the process ends, like the pinned buffers
  return *s;
}

bool staging_on() {
  static const int on = env_int("HOS_STAGE", 1);
  return on != 0;
}

// Whether p is host memory the driver knows nothing about (pageable).
bool pageable(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeUnregistered;
}

bool is_device(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice;
}

// The staging buffers and this device's two events (the caller holds s.m).
cudaError_t prepare(Stager& s, cudaEvent_t* ev) {
  if (!s.pin[0]) {
    const int kb = std::max(64, env_int("HOS_STAGE_CHUNK_KB", 2048));
    s.chunk = (size_t)kb << 10;
    for (int b = 0; b < 2; b++) {
      if (cudaHostAlloc((void**)&s.pin[b], s.chunk, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        if (b == 1) cudaFreeHost(s.pin[0]);
        s.pin[0] = s.pin[1] = nullptr;
        s.failed = true;
        return cudaErrorMemoryAllocation;
      }
    }
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if ((int)s.ev.size() < 2 * (dev + 1)) s.ev.resize(2 * (dev + 1), nullptr);
  for (int b = 0; b < 2; b++) {
    cudaEvent_t& x = s.ev[2 * dev + b];
    if (!x) {
      e = cudaEventCreateWithFlags(&x, cudaEventDisableTiming);
      if (e != cudaSuccess) {
        x = nullptr;
        return e;
      }
    }
    ev[b] = x;
  }
  return cudaSuccess;
}

#define ST_CK(x)                         \
  do {                                   \
    const cudaError_t e_ = (x);          \
    if (e_ != cudaSuccess) return e_;    \
  } while (0)

// Pageable host -> device.  Each buffer is refilled only after the copy
// engine has drained it; the last chunks are drained before returning so the
// buffers are free for the next caller.
cudaError_t staged_h2d(Stager& s, const cudaEvent_t* ev, unsigned char* dst, const unsigned char* src, size_t bytes,
                       cudaStream_t st) {
  const size_t C = s.chunk;
  const size_t nch = (bytes + C - 1) / C;
  for (size_t i = 0; i < nch; i++) {
    const int b = (int)(i & 1);
    const size_t off = i * C, n = std::min(C, bytes - off);
    if (i >= 2) ST_CK(cudaEventSynchronize(ev[b]));
    pool().copy(s.pin[b], src + off, n);
    ST_CK(cudaMemcpyAsync(dst + off, s.pin[b], n, cudaMemcpyHostToDevice, st));
    ST_CK(cudaEventRecord(ev[b], st));
  }
  for (size_t i = nch >= 2 ? nch - 2 : 0; i < nch; i++) ST_CK(cudaEventSynchronize(ev[i & 1]));
  return cudaSuccess;
}

// Device -> pageable host: chunk i+1 is in flight while the host threads
// copy chunk i out of the other buffer.
cudaError_t staged_d2h(Stager& s, const cudaEvent_t* ev, unsigned char* dst, const unsigned char* src, size_t bytes,
                       cudaStream_t st) {
  const size_t C = s.chunk;
  const size_t nch = (bytes + C - 1) / C;
  auto issue = [&](size_t i) -> cudaError_t {
    const int b = (int)(i & 1);
    const size_t off = i * C, n = std::min(C, bytes - off);
    cudaError_t e = cudaMemcpyAsync(s.pin[b], src + off, n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(ev[b], st);
    return e;
  };
  ST_CK(issue(0));
  for (size_t i = 0; i < nch; i++) {
    const int b = (int)(i & 1);
    const size_t off = i * C, n = std::min(C, bytes - off);
    if (i + 1 < nch) ST_CK(issue(i + 1));
    ST_CK(cudaEventSynchronize(ev[b]));
    pool().copy(dst + off, s.pin[b], n);
  }
  return cudaSuccess;
}

}  // namespace

void par_memcpy(void* dst, const void* src, size_t bytes) {
  pool().copy(static_cast<unsigned char*>(dst), static_cast<const unsigned char*>(src), bytes);
}

cudaError_t host_copy(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (bytes >= STAGE_MIN && staging_on()) {
    const bool up = pageable(src) && is_device(dst);
    const bool down = !up && pageable(dst) && is_device(src);
    if (up || down) {
      Stager& s = stager();
      std::lock_guard<std::mutex> lk(s.m);
      cudaEvent_t ev[2];
      if (!s.failed && prepare(s, ev) == cudaSuccess) {
        if (up)
          return staged_h2d(s, ev, static_cast<unsigned char*>(dst), static_cast<const unsigned char*>(src), bytes, st);
        return staged_d2h(s, ev, static_cast<unsigned char*>(dst), static_cast<const unsigned char*>(src), bytes, st);
      }
    }
  }
  return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, st);
}

}  // namespace hos
