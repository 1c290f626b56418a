// Copies between the caller's host arrays and the device.
//
// A large array in pageable host memory (what fftw_alloc / malloc return,
// and what the reference's driver hands to sol_update_RK) is moved through a
// pinned staging buffer in parts: host threads copy the parts, and each part
// crosses to or from the device while the threads work on the next ones.
// Pinned host memory, device memory and small arrays go straight to
// cudaMemcpyAsync.
#pragma once

#include <cstddef>

#include <cuda_runtime.h>

namespace hos {

// Enqueues the copy of `bytes` bytes from src to dst on `st` (either side may
// be host or device memory, as for cudaMemcpyDefault).  A staged copy from
// pageable host memory has read all of src when this returns; a staged copy
// into pageable host memory has written all of dst when this returns.
cudaError_t host_copy(void* dst, const void* src, size_t bytes, cudaStream_t st);

}  // namespace hos
