// The persistent ensemble kernel (see hos_persist.h for the scheduling
// rules): every resident block takes work items in list order, waits for
// the member's earlier passes, runs the pass body on the item's blocks and
// counts the item done.
#include <cstdint>
#include <cstdlib>

#include "hos_kernels.cuh"
#include "hos_persist.h"

namespace hos {
namespace {

// ---------------------------------------------------------------- pass bodies
// One non-inlined function per (precision, pass, line length): each keeps
// its own register allocation and the kernel stays small to compile.
template <typename T, int NX, int MODE>
__device__ __noinline__ void pb_xinv(const void* a, int bx, int by, const void* tw, unsigned char* sm) {
  xinv_body<T, NX, 8, MODE>(*static_cast<const XInvArgs*>(a), bx, by, PERSIST_THREADS, tw, sm);
}
template <typename T, int NX, int MODE>
__device__ __noinline__ void pb_xfwd(const void* a, int bx, int by, const void* tw, unsigned char* sm) {
  xfwd_body<T, NX, 8, MODE>(*static_cast<const XFwdArgs*>(a), bx, by, PERSIST_THREADS, tw, sm);
}
template <typename T, int H, int E, int MODE>
__device__ __noinline__ void pb_yinv(const void* a, int bx, int by, const void* tw, const void* twy,
                                     unsigned char* sm) {
  yinv_body<T, H, E, MODE>(*static_cast<const YInvArgs*>(a), bx, by, PERSIST_THREADS, tw, twy, sm);
}
template <typename T, int H, int MODE>
__device__ __noinline__ void pb_yfwd(const void* a, int bx, int by, const void* tw, const void* twy,
                                     unsigned char* sm) {
  yfwd_body<T, H, 8, MODE>(*static_cast<const YFwdArgs*>(a), bx, by, PERSIST_THREADS, tw, twy, sm);
}
__device__ __noinline__ void pb_step_end(const void* a) {
  step_end_body(*static_cast<const StepEndArgs*>(a), PERSIST_THREADS);
}

template <typename T, int S>
__device__ __forceinline__ void run_size(int code, const PTask& k, int bx, int by, unsigned char* sm) {
  constexpr int NX = 64 << S, H = 32 << S;
  switch (code) {
    case PC_XINV_STAGE: pb_xinv<T, NX, XI_STAGE>(k.args, bx, by, k.tw0, sm); break;
    case PC_XFWD_LEVEL: pb_xfwd<T, NX, XF_LEVEL>(k.args, bx, by, k.tw0, sm); break;
    case PC_XFWD_RHS: pb_xfwd<T, NX, XF_RHS>(k.args, bx, by, k.tw0, sm); break;
    case PC_YINV_JOBS: pb_yinv<T, H, 16, YI_JOBS>(k.args, bx, by, k.tw0, k.tw1, sm); break;
    case PC_YINV_JOBS8: pb_yinv<T, H, 8, YI_JOBS>(k.args, bx, by, k.tw0, k.tw1, sm); break;
    case PC_YINV_LEVEL: pb_yinv<T, H, 8, YI_LEVEL>(k.args, bx, by, k.tw0, k.tw1, sm); break;
    case PC_YFWD_LEVEL: pb_yfwd<T, H, YF_LEVEL>(k.args, bx, by, k.tw0, k.tw1, sm); break;
    case PC_YFWD_RHS: pb_yfwd<T, H, YF_RHS>(k.args, bx, by, k.tw0, k.tw1, sm); break;
    default: break;
  }
}

template <typename T>
__device__ __forceinline__ void run_prec(const PTask& k, int bx, int by, unsigned char* sm) {
  const int code = k.body / PERSIST_SIZES, s = k.body % PERSIST_SIZES;
  switch (s) {
    case 0: run_size<T, 0>(code, k, bx, by, sm); break;
    case 1: run_size<T, 1>(code, k, bx, by, sm); break;
    case 2: run_size<T, 2>(code, k, bx, by, sm); break;
    case 3: run_size<T, 3>(code, k, bx, by, sm); break;
    case 4: run_size<T, 4>(code, k, bx, by, sm); break;
    default: run_size<T, 5>(code, k, bx, by, sm); break;
  }
}

__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];\n" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_relaxed(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ long long now_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}

template <int MINB>
__global__ void __launch_bounds__(PERSIST_THREADS, MINB) k_persist(const __grid_constant__ PersistArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ PTask s_task;  // the current item's task, read once by thread 0
  __shared__ int s_item, s_go, s_left;
  __shared__ unsigned long long s_epoch;
  if (threadIdx.x == 0) s_epoch = *a.epoch;  // written by the previous launch's last block
  __syncthreads();
  const unsigned long long epoch = s_epoch;
  int next_it = -1;  // thread 0: the item taken ahead, while the current one runs
  for (;;) {
    if (threadIdx.x == 0) {
      int it = next_it >= 0 ? next_it : (int)atomicAdd(a.head, 1u);
      if (it >= a.nitems || ld_relaxed(a.err)) it = -1;
      int go = 0;
      if (it >= 0) {
        // one load gives the task, the member and the wait target
        const int4 inf = __ldg(&a.item_info[it]);
        s_task = a.tasks[inf.x];
        s_left = a.remaining[inf.y];
        const unsigned long long target = epoch * (unsigned long long)(unsigned)inf.w + (unsigned long long)(unsigned)inf.z;
        unsigned long long seen = ld_acquire(&a.done[inf.y]);
        go = 1;
        if (seen < target) {
          const long long t0 = now_ns();
          while ((seen = ld_acquire(&a.done[inf.y])) < target) {
            if (ld_relaxed(a.err)) {
              go = 0;
              break;
            }
            if (now_ns() - t0 > a.wait_limit_ns) {
              if (atomicCAS(a.err, 0, 1) == 0) {
                a.err_info[0] = it;
                a.err_info[1] = inf.y;
                a.err_info[2] = (long long)target;
                a.err_info[3] = (long long)seen;
              }
              go = 0;
              break;
            }
            __nanosleep(100);
          }
        }
        // take the next item now: the atomic's latency hides behind this
        // item's work (items are still taken, and run, in list order)
        if (go) next_it = (int)atomicAdd(a.head, 1u);
      }
      s_item = it;
      s_go = go;
    }
    // the barrier orders every thread's reads after thread 0's acquire
    __syncthreads();
    const int it = s_item;
    if (it < 0 || !s_go) break;
    const PTask& k = s_task;
    const int local = it - k.first_item;
    const int b0 = local * k.per_item;
    const int nb = k.gx * k.gy;
    const int b1 = min(b0 + k.per_item, nb);
    // a member whose step budget is spent skips its items (they still count
    // as done); the budget only changes in the member's step end, the last
    // task of its step, so every item of one launch sees the same value
    const int left = s_left;
    if (left == 0) {
      // nothing to do
    } else if (k.body == PC_STEP_END * PERSIST_SIZES) {
      pb_step_end(k.args);
      if (left > 0 && threadIdx.x == 0) a.remaining[k.member] = left - 1;
    } else {
      for (int b = b0; b < b1; b++) {
        const int bx = b % k.gx, by = b / k.gx;
        if (k.prec)
          run_prec<float>(k, bx, by, smraw);
        else
          run_prec<double>(k, bx, by, smraw);
        __syncthreads();  // the next block of the item reuses the shared memory
      }
    }
    // the item's writes are visible device-wide before it is counted done:
    // the barrier orders every thread's writes before thread 0's fence,
    // which is cumulative, and the count comes after the fence
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(&a.done[k.member], 1ull);
    }
  }
  // the last block out resets the counters for the next launch
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned int f = atomicAdd(a.finished, 1u);
    if (f == gridDim.x - 1) {
      __threadfence();
      *a.head = 0u;
      *a.finished = 0u;
      if (ld_relaxed(a.err)) {
        for (int m = 0; m < a.nmembers; m++) a.done[m] = 0ull;
        *a.epoch = 0ull;
      } else {
        *a.epoch = epoch + 1ull;
      }
      __threadfence();
    }
  }
}

}  // namespace

const void* persist_fn(int minb) { return minb == 3 ? (const void*)k_persist<3> : (const void*)k_persist<2>; }

cudaError_t persist_launch(const PersistArgs& a, int blocks, size_t smem, cudaStream_t st, int minb) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(PERSIST_THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;  // all blocks resident: a waiting block never waits on an unplaced one
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  if (minb == 3) return cudaLaunchKernelEx(&cfg, k_persist<3>, a);
  return cudaLaunchKernelEx(&cfg, k_persist<2>, a);
}

cudaError_t persist_occupancy(int* blocks_per_sm, size_t smem, int minb) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, persist_fn(minb), PERSIST_THREADS, smem);
}

cudaError_t persist_set_smem(size_t smem, int minb) {
  return cudaFuncSetAttribute(persist_fn(minb), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

}  // namespace hos
