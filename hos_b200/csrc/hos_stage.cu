// Staged copies between pageable host arrays and the device (hos_stage.h).
//
// A pageable cudaMemcpyAsync is staged by the driver through its own pinned
// buffers with one host thread; the reference's driver passes its whole
// packed state (two complex fields, 16.8 MB at 1024^2) this way twice per
// sol_update_RK call.  Here the host side of the staging is split over
// several threads and overlapped with the copy engine: host to device, the
// threads fill one half of the pinned buffer while the copy engine empties
// the other; device to host, every part's device copy is queued at once and
// the threads copy each part out as soon as it has landed.
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <pthread.h>
#include <system_error>
#include <thread>
#include <vector>

#include "hos_stage.h"

namespace hos {
namespace {

constexpr size_t STAGE_MIN = 1u << 20;     // smaller copies go straight to the driver
constexpr size_t WINDOW_MAX = 64u << 20;   // largest pinned buffer; longer copies go window by window

int env_int(const char* name, int dflt) {
  const char* s = getenv(name);
  return (s && *s) ? atoi(s) : dflt;
}

// ------------------------------------------------------------ copy threads
// A job is `nparts` parts, claimed in index order by the pool's threads and
// by the caller's thread; work(k) does part k.
// The caller's thread claims parts too, so a job finishes even with no copy
// thread running.  The pool lives until the process ends and its threads
// are detached: no join at exit; a process forked from this one has none of
// the threads and starts its own.
class CopyPool {
 public:
  // In a forked child: the copy threads did not come along.
  void forget_threads() { started_ = 0; }

  void run(size_t nparts, const std::function<void(size_t)>& work) {
    std::lock_guard<std::mutex> job(job_m_);  // one job at a time
    start(threads() - 1);
    unsigned long long g;
    {
      std::lock_guard<std::mutex> lk(m_);
      work_ = &work;
      nparts_ = nparts;
      next_ = 0;
      done_ = 0;
      g = ++gen_;
    }
    cv_.notify_all();
    while (take_one(g)) {
    }
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

  // Starts copy threads up to `workers`; returns how many run.
  int start(int workers) {
    std::lock_guard<std::mutex> lk(m_);
    while (started_ < workers) {
      const unsigned long long g = gen_;
      try {
        std::thread([this, g] { loop(g); }).detach();
      } catch (const std::system_error&) {
        break;  // no more threads: the others take the parts
      }
      started_++;
    }
    return started_;
  }

  [[noreturn]] void loop(unsigned long long seen) {
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(m_);
        cv_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
      }
      while (take_one(seen)) {
      }
    }
  }

  // Claims and does one part of job g; false when none is left (or a newer
  // job replaced it).
  bool take_one(unsigned long long g) {
    size_t k;
    const std::function<void(size_t)>* w;
    {
      std::lock_guard<std::mutex> lk(m_);
      if (gen_ != g || next_ >= nparts_) return false;
      k = next_++;
      w = work_;
    }
    (*w)(k);
    bool last;
    {
      std::lock_guard<std::mutex> lk(m_);
      last = ++done_ == nparts_;
    }
    if (last) done_cv_.notify_all();
    return true;
  }

  std::mutex job_m_;
  std::mutex m_;
  std::condition_variable cv_, done_cv_;
  int started_ = 0;
  int nthreads_ = 0;
  unsigned long long gen_ = 0;
  const std::function<void(size_t)>* work_ = nullptr;
  size_t nparts_ = 0, next_ = 0, done_ = 0;
};

CopyPool* g_pool = nullptr;

CopyPool& pool() {
  static CopyPool* p = [] {
    g_pool = new CopyPool;  // never destroyed (see above)
    // a forked child has none of the parent's threads: it starts its own
    pthread_atfork(nullptr, nullptr, [] { g_pool->forget_threads(); });
    return g_pool;
  }();
  return *p;
}

// ------------------------------------------------------------ staging buffer
struct Stager {
  std::mutex m;
  unsigned char* pin = nullptr;  // pinned buffer of `cap` bytes
  size_t cap = 0;
  bool failed = false;           // pinned allocation failed: copies go to the driver
  std::vector<std::vector<cudaEvent_t>> ev;  // per device: one per part of a window, created on first use
};

Stager& stager() {
  static Stager* s = new Stager;  // lives until the process ends, like the pinned buffer
  return *s;
}

bool staging_on() {
  static const int on = env_int("HOS_STAGE", 1);
  return on != 0;
}

size_t part_bytes() {
  static const size_t p = (size_t)std::max(64, env_int("HOS_STAGE_CHUNK_KB", 1024)) << 10;
  return p;
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

// A pinned buffer for a copy of `bytes` (at most WINDOW_MAX) and `nparts`
// events of the current device (the caller holds s.m; every earlier copy
// through the buffer has finished).
cudaError_t prepare(Stager& s, size_t bytes, size_t nparts, int* dev, cudaEvent_t** evs) {
  const size_t need = std::min(bytes, WINDOW_MAX);
  if (s.cap < need) {
    if (s.pin) cudaFreeHost(s.pin);
    s.pin = nullptr;
    s.cap = 0;
    if (cudaHostAlloc((void**)&s.pin, need, cudaHostAllocPortable) != cudaSuccess) {
      cudaGetLastError();
      s.pin = nullptr;
      s.failed = true;
      return cudaErrorMemoryAllocation;
    }
    s.cap = need;
  }
  cudaError_t e = cudaGetDevice(dev);
  if (e != cudaSuccess) return e;
  if ((int)s.ev.size() <= *dev) s.ev.resize(*dev + 1);
  std::vector<cudaEvent_t>& v = s.ev[*dev];
  while (v.size() < nparts) {
    cudaEvent_t x;
    e = cudaEventCreateWithFlags(&x, cudaEventDisableTiming);
    if (e != cudaSuccess) return e;
    v.push_back(x);
  }
  *evs = v.data();
  return cudaSuccess;
}

#define ST_CK(x)                         \
  do {                                   \
    const cudaError_t e_ = (x);          \
    if (e_ != cudaSuccess) return e_;    \
  } while (0)

// Pageable host -> device in chunks of two parts, through two halves of the
// pinned buffer: all threads copy chunk i into one half (each a slice of it)
// while the copy engine moves chunk i-1 out of the other.  (A part per thread
// with the copy engine fed part by part measured slower: one thread's memcpy
// is a fraction of the host's bandwidth.)  The last copies have finished when
// the call returns, so the buffer is free for the next caller.
cudaError_t staged_h2d(Stager& s, unsigned char* dst, const unsigned char* src, size_t bytes, cudaStream_t st) {
  const size_t C = 2 * part_bytes();
  int dev = 0;
  cudaEvent_t* evs = nullptr;
  ST_CK(prepare(s, std::max(bytes, 2 * C), 2, &dev, &evs));
  const size_t nch = (bytes + C - 1) / C;
  for (size_t i = 0; i < nch; i++) {
    const int b = (int)(i & 1);
    unsigned char* half = s.pin + b * C;
    const size_t off = i * C, n = std::min(C, bytes - off);
    if (i >= 2) ST_CK(cudaEventSynchronize(evs[b]));
    const size_t slice = std::max<size_t>(128u << 10, (n + 7) / 8);
    const size_t nsl = (n + slice - 1) / slice;
    const std::function<void(size_t)> work = [&](size_t k) {
      const size_t o = k * slice;
      memcpy(half + o, src + off + o, std::min(slice, n - o));
    };
    pool().run(nsl, work);
    ST_CK(cudaMemcpyAsync(dst + off, half, n, cudaMemcpyHostToDevice, st));
    ST_CK(cudaEventRecord(evs[b], st));
  }
  for (size_t i = nch >= 2 ? nch - 2 : 0; i < nch; i++) ST_CK(cudaEventSynchronize(evs[i & 1]));
  return cudaSuccess;
}

// Device -> pageable host, window by window: every part's device copy is
// queued first, each followed by an event; a thread that takes part k waits
// for its event and copies it out while the later parts are still in flight.
cudaError_t staged_d2h(Stager& s, unsigned char* dst, const unsigned char* src, size_t bytes, cudaStream_t st) {
  const size_t P = part_bytes();
  const size_t npmax = (std::min(bytes, WINDOW_MAX) + P - 1) / P;
  int dev = 0;
  cudaEvent_t* evs = nullptr;
  ST_CK(prepare(s, bytes, npmax, &dev, &evs));
  for (size_t w0 = 0; w0 < bytes; w0 += s.cap) {
    const size_t wb = std::min(s.cap, bytes - w0);
    const size_t np = (wb + P - 1) / P;
    for (size_t k = 0; k < np; k++) {
      const size_t off = k * P;
      ST_CK(cudaMemcpyAsync(s.pin + off, src + w0 + off, std::min(P, wb - off), cudaMemcpyDeviceToHost, st));
      ST_CK(cudaEventRecord(evs[k], st));
    }
    std::atomic<int> err{(int)cudaSuccess};
    const std::function<void(size_t)> work = [&](size_t k) {
      cudaError_t e = cudaSetDevice(dev);
      if (e == cudaSuccess) e = cudaEventSynchronize(evs[k]);
      if (e != cudaSuccess) {
        err.store((int)e);
        return;
      }
      const size_t off = k * P;
      memcpy(dst + w0 + off, s.pin + off, std::min(P, wb - off));
    };
    pool().run(np, work);
    if (err.load() != (int)cudaSuccess) return (cudaError_t)err.load();
  }
  return cudaSuccess;
}

}  // namespace

cudaError_t host_copy(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (bytes >= STAGE_MIN && staging_on()) {
    const bool up = pageable(src) && is_device(dst);
    const bool down = !up && pageable(dst) && is_device(src);
    if (up || down) {
      Stager& s = stager();
      std::lock_guard<std::mutex> lk(s.m);
      if (!s.failed) {
        cudaError_t e = up ? staged_h2d(s, static_cast<unsigned char*>(dst), static_cast<const unsigned char*>(src),
                                        bytes, st)
                           : staged_d2h(s, static_cast<unsigned char*>(dst), static_cast<const unsigned char*>(src),
                                        bytes, st);
        if (e != cudaErrorMemoryAllocation || !s.failed) return e;
        // the pinned buffer could not be had: the driver's path below
      }
    }
  }
  return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, st);
}

}  // namespace hos
