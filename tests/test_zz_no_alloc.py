"""exafmm_b200_direct_static: the direct sum for callers that may not allocate.

Such callers (codes that give all of HBM to their own pool at start-up, or
loops that must never enter the CUDA allocator) cannot create a handle, so
this entry point takes their own device arrays and uses only a fixed scratch
array built into the library.  The test owns the device memory (torch), calls
the entry point through the C ABI twice in a row -- the second call finds the
first call's leftovers in the shared scratch -- and checks both results
against the handle-based exafmm_b200_direct() at the direct-sum tolerance of
the other tests.  It is collected last (file name) and needs no state from
other tests, so it passes alone in a fresh process too.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-13  # relative L2, as test_direct_vs_oracle


def rel_l2(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def test_direct_static_matches_direct_twice():
    import torch

    import minimal_b200
    from minimal_b200 import FMM, drand48_bodies

    lib = minimal_b200.load_library()
    xq = drand48_bodies(30000, 9)
    src = np.zeros((len(xq), 8))
    src[:, :4] = xq
    fmm = FMM()
    fmm.set_bodies(src)
    fmm.build_tree()

    dev = torch.device("cuda", 0)
    d_src = torch.from_numpy(src).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call, (nt, stride) in enumerate([(4000, 7), (1500, 13)]):
        tgt = np.zeros((nt, 8))
        tgt[:, :4] = xq[::stride][:nt]
        want = fmm.direct(tgt)  # existing entry point, handle-based
        d_tgt = torch.from_numpy(tgt).to(dev)  # p, F start at zero
        torch.cuda.synchronize(dev)
        free_before = torch.cuda.mem_get_info(dev)[0]
        rc = lib.exafmm_b200_direct_static(ctypes.c_void_p(d_src.data_ptr()), len(src),
                                           ctypes.c_void_p(d_tgt.data_ptr()), nt, ctypes.c_void_p(stream))
        assert rc == 0, lib.exafmm_b200_last_error(None).decode()
        assert lib.exafmm_b200_last_error(None).decode() == "", "a success leaves no error message"
        torch.cuda.synchronize(dev)
        if call > 0:  # the first call may load the library's module (and its scratch) onto the GPU
            assert torch.cuda.mem_get_info(dev)[0] == free_before, f"call {call}: device memory was allocated"
        got = d_tgt.cpu().numpy()
        assert np.array_equal(got[:, :4], tgt[:, :4]), f"call {call}: positions must be untouched"
        assert rel_l2(got[:, 4], want[:, 4]) < TOL, f"call {call}: potential"
        assert rel_l2(got[:, 5:], want[:, 5:]) < TOL, f"call {call}: force"


def test_direct_static_rejects_oversize_without_launching():
    import torch

    import minimal_b200

    lib = minimal_b200.load_library()
    dev = torch.device("cuda", 0)
    d = torch.zeros((8, 8), dtype=torch.float64, device=dev)
    too_many = 65536 + 1
    rc = lib.exafmm_b200_direct_static(ctypes.c_void_p(d.data_ptr()), 8, ctypes.c_void_p(d.data_ptr()), too_many,
                                       None)
    assert rc == -1
    assert "65536" in lib.exafmm_b200_last_error(None).decode()


def test_direct_static_rejects_a_stream_of_another_device():
    """The scratch address is per device, so the caller's stream must belong
    to the current device: a stream of a second device is refused before
    anything is launched (needs two GPUs; skipped on one)."""
    import torch

    import minimal_b200

    lib = minimal_b200.load_library()
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two GPUs")
    torch.cuda.set_device(0)
    s1 = torch.cuda.Stream(device=1)
    d = torch.zeros((8, 8), dtype=torch.float64, device="cuda:0")
    rc = lib.exafmm_b200_direct_static(ctypes.c_void_p(d.data_ptr()), 8, ctypes.c_void_p(d.data_ptr()), 8,
                                       ctypes.c_void_p(s1.cuda_stream))
    assert rc == -1
    assert "stream" in lib.exafmm_b200_last_error(None).decode()
