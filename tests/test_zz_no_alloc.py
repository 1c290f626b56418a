"""hos_fft_2d_noalloc: the allocation-free variant of fft_2d, for callers
that cannot allocate GPU memory (code running under CUDA-graph stream
capture, latency-critical loops where an allocation would synchronise the
device, hosts whose own allocator owns all device memory).

Its output must equal that of the allocating entry point hos_fft_2d, within
the tolerance of the other transform tests, on two calls in a row (the
second reuses the library's fixed scratch array).  This file is collected
last so that a failure here never hides the rest of the suite."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-14


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_noalloc_matches_allocating_fft_twice():
    import torch

    import hos_b200
    from hos_b200 import HosField

    lib = hos_b200.load()
    fn = lib.hos_fft_2d_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    rng = np.random.default_rng(2024)
    # 2048 x 16: one thread per y line (256 lines per block); 16 x 2048 and
    # 2048 x 256: the longest lines the fixed scratch allows in each direction
    for nx, ny in [(256, 128), (1024, 1024), (2048, 16), (16, 2048), (2048, 256)]:
        with HosField(nx, ny) as f:
            xs = [rng.standard_normal((nx, ny)) for _ in range(2)]
            wants = [f.fft_2d(x) for x in xs]  # the existing, allocating entry point
            xins = [torch.from_numpy(x).cuda() for x in xs]
            outs = [torch.zeros((ny // 2 + 1, nx, 2), dtype=torch.float64, device="cuda") for _ in xs]
            stream = torch.cuda.current_stream()
            # a first call loads the library's device code for this entry
            # point (and with it the fixed arrays) if nothing has yet
            warm = torch.zeros_like(outs[0])
            assert fn(ctypes.c_void_p(xins[0].data_ptr()), ctypes.c_void_p(warm.data_ptr()), nx, ny,
                      ctypes.c_void_p(stream.cuda_stream)) == 0, lib.hos_last_error()
            torch.cuda.synchronize()
            free0 = torch.cuda.mem_get_info()[0]
            for call in range(2):
                rc = fn(ctypes.c_void_p(xins[call].data_ptr()), ctypes.c_void_p(outs[call].data_ptr()), nx, ny,
                        ctypes.c_void_p(stream.cuda_stream))
                assert rc == 0, lib.hos_last_error()
            stream.synchronize()
            # nothing was allocated on the device by the two calls (the
            # library's fixed arrays were placed when its code was loaded)
            assert torch.cuda.mem_get_info()[0] == free0
            for call in range(2):
                got = outs[call].cpu().numpy()
                got = got[..., 0] + 1j * got[..., 1]
                assert rel(got, wants[call]) < TOL, (nx, ny, call)


def test_noalloc_rejects_oversized_grid():
    import torch

    import hos_b200

    lib = hos_b200.load()
    fn = lib.hos_fft_2d_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(buf.data_ptr())
    assert fn(p, p, 2048, 2048, None) == 1  # HOS_ERR_ARG: beyond the fixed scratch
    assert b"too large" in lib.hos_last_error()
    assert fn(p, p, 48, 64, None) == 1
