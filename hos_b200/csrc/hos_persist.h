// The persistent ensemble kernel: one launch advances every member of an
// ensemble by one RK step.
//
// The pass sequence of a member's step (the launches hos_step would make:
// build_stage for each stage, then the step end) becomes a list of tasks,
// one per pass.  A task's blocks are the pass's blocks re-shaped for
// PERSIST_THREADS threads (more lines per block; each line's arithmetic is
// unchanged, so results are bitwise those of hos_step) and grouped into work
// items of per_item blocks.  The items of all members form one global list,
// ordered round by round (task 0 of every member, then task 1, ...); the
// resident blocks of the kernel take items from it in that order with an
// atomic counter.  Before it runs an item, a block waits until every item
// of the member's earlier tasks of this step has completed (a per-member
// counter of completed items), which is the stream order of the separate
// launches.  Every item an item waits on comes earlier in the list and was
// taken by a block that is running (the launch is cooperative, so all
// blocks are resident), so the earliest unfinished item can always run.
//
// Waits are bounded: a wait that exceeds the limit sets an error word, and
// every block then stops taking items and returns; the host reports
// HOS_ERR_TIMEOUT.  The last block to finish resets the counters for the
// next launch (after an error it also clears the per-member counts).
#pragma once

#include <cuda_runtime.h>

namespace hos {

constexpr int PERSIST_THREADS = 256;

// Pass codes of the tasks (body = code * PERSIST_SIZES + size index; the
// size index s selects x-line length 64 << s or y-line length 32 << s).
enum PersistCode {
  PC_XINV_STAGE = 0,
  PC_XFWD_LEVEL,
  PC_XFWD_RHS,
  PC_YINV_JOBS,   // the stage y-inverse, 16 elements per thread
  PC_YINV_LEVEL,
  PC_YFWD_LEVEL,
  PC_YFWD_RHS,
  PC_YINV_JOBS8,  // the stage y-inverse with 8 elements per thread (grids too small for 16)
  PC_STEP_END,
  PC_NCODES
};
constexpr int PERSIST_SIZES = 6;  // x lines 64..2048, y lines 32..1024

struct PTask {
  int body;           // code * PERSIST_SIZES + size index (code PC_STEP_END: size 0)
  int prec;           // 0 double, 1 float
  int member;         // ensemble member
  int gx, gy;         // blocks of the pass
  int per_item;       // blocks per work item
  int nitems;         // work items of the task
  int first_item;     // index of the task's first item in the global list
  long long dep;      // items of the member's earlier tasks in one step
  const void* args;   // XInvArgs / XFwdArgs / YInvArgs / YFwdArgs / StepEndArgs (device)
  const void* tw0;    // twiddles: x lines (x passes) or y half lines (y passes)
  const void* tw1;    // y passes: length-ny table
};

struct PersistArgs {
  const PTask* tasks;
  const int4* item_info;             // per item, in list order: task, member, dep of the task, items of the member's step
  int nitems;
  unsigned long long* done;          // per member: items completed, over all launches
  const long long* member_items;     // per member: items of one step
  int nmembers;
  unsigned int* head;                // next item to take
  unsigned int* finished;            // blocks done with this launch
  unsigned long long* epoch;         // launches completed
  int* remaining;                    // per member: steps still to take (-1: no limit); 0 skips the member
  int* err;                          // 0, or 1 after a wait ran out
  long long* err_info;               // [item, member, target, seen] of the first wait that ran out
  long long wait_limit_ns;           // bound of one wait
};

// The kernel is compiled for 2 resident blocks per SM (up to 128 registers a
// thread) and for 3 (up to 80: more warps, the heavier pass bodies spill);
// `minb` selects one.
// Launches one step of the persistent kernel (cooperative launch of
// `blocks` blocks with `smem` bytes of dynamic shared memory).
cudaError_t persist_launch(const PersistArgs& a, int blocks, size_t smem, cudaStream_t st, int minb);
// Resident blocks per SM of the persistent kernel for `smem` bytes.
cudaError_t persist_occupancy(int* blocks_per_sm, size_t smem, int minb);
// Raises the kernel's dynamic shared memory limit to `smem` bytes.
cudaError_t persist_set_smem(size_t smem, int minb);

}  // namespace hos
