"""cbnm_fc_fcd_noalloc, the FC / FCD entry point that allocates no device memory,
against the FC / FCD that cbnm_run_simulations returns for the same BOLD.

Every call goes through the C ABI.  The file name sorts last, so under a full
run the entry point is also exercised after every other test has used the
library.  The variant repeats the arithmetic of the session's FC kernels in the
same order, so the tolerance below is a few ulp.
"""
import ctypes as C

import numpy as np
import pytest

import cases
from cubnm_b200 import _lib, core

RTOL, ATOL = 1e-12, 1e-14
SCRATCH_BYTES = 32 << 20


def _noalloc():
    L = _lib.lib()
    f = L.cbnm_fc_fcd_noalloc
    f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                  C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return L, f


def _simulate(N, nodes, duration_s, window_size, window_step, bold_remove_s, exc_inter):
    args = list(cases.synthetic_args("rWW", N=N, nodes=nodes, duration_s=duration_s, seed=3,
                                     window_size=window_size, window_step=window_step,
                                     bold_remove_s=bold_remove_s))
    args[7] = dict(args[7], exc_interhemispheric=str(int(exc_inter)))
    return core.run_simulations(*args)


# (N, nodes, duration s, window size, window step, BOLD removed s, exc_interhemispheric)
CASES = {
    "default_windows": (24, 100, 60, 10, 2, 30, False),
    "interhemispheric_excluded": (16, 68, 80, 8, 3, 10, True),
    # 200 windows x 4950 pairs = 7.9 MB per simulation: 4 simulations per scratch chunk, 3 chunks
    "several_scratch_chunks": (10, 100, 220, 10, 1, 10, False),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_noalloc_matches_run_simulations_twice(name):
    import torch
    N, nodes, dur, ws, step, rm, exc = CASES[name]
    ref = _simulate(N, nodes, dur, ws, step, rm, exc)
    L, f = _noalloc()
    bold_np = np.ascontiguousarray(ref["sim_bold"]).reshape(N, -1)
    bold_len = bold_np.shape[1] // nodes
    n_vols_remove = rm  # bold_remove_s * 1000 / BOLD_TR with BOLD_TR = 1000 ms
    dev = torch.device("cuda:0")
    bold = torch.from_numpy(bold_np).to(dev)
    fc = torch.empty(ref["sim_fc_trils"].shape, dtype=torch.float64, device=dev)
    fcd = torch.empty(ref["sim_fcd_trils"].shape, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for _ in range(2):  # two calls in a row: nothing may carry over between them
        fc.fill_(float("nan"))
        fcd.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = f(bold.data_ptr(), N, bold_len, nodes, n_vols_remove, ws, step, 1, int(exc),
               fc.data_ptr(), fcd.data_ptr(), stream)
        assert rc == 0, L.cbnm_last_error()
        torch.cuda.synchronize()
        np.testing.assert_allclose(fc.cpu().numpy(), ref["sim_fc_trils"], rtol=RTOL, atol=ATOL)
        np.testing.assert_allclose(fcd.cpu().numpy(), ref["sim_fcd_trils"], rtol=RTOL, atol=ATOL)


@pytest.mark.gpu
def test_noalloc_allocates_no_device_memory():
    """The property the entry point exists for: after a first call (which may load
    the module holding the scratch), further calls leave the device's free memory
    unchanged -- here a call over several scratch chunks, twice."""
    import torch
    N, nodes, dur, ws, step, rm, exc = CASES["several_scratch_chunks"]
    ref = _simulate(N, nodes, dur, ws, step, rm, exc)
    L, f = _noalloc()
    bold = torch.from_numpy(np.ascontiguousarray(ref["sim_bold"]).reshape(N, -1)).to("cuda:0")
    bold_len = bold.shape[1] // nodes
    fc = torch.empty(ref["sim_fc_trils"].shape, dtype=torch.float64, device="cuda:0")
    fcd = torch.empty(ref["sim_fcd_trils"].shape, dtype=torch.float64, device="cuda:0")
    call = lambda: f(bold.data_ptr(), N, bold_len, nodes, rm, ws, step, 1, int(exc), fc.data_ptr(),  # noqa: E731
                     fcd.data_ptr(), None)
    assert call() == 0, L.cbnm_last_error()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        assert call() == 0, L.cbnm_last_error()
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0, (free0, free1)
    np.testing.assert_allclose(fcd.cpu().numpy(), ref["sim_fcd_trils"], rtol=RTOL, atol=ATOL)


@pytest.mark.gpu
def test_noalloc_fc_only_after_fcd_call():
    import torch
    N, nodes, dur, ws, step, rm, exc = CASES["default_windows"]
    ref = _simulate(N, nodes, dur, ws, step, rm, exc)
    L, f = _noalloc()
    bold = torch.from_numpy(np.ascontiguousarray(ref["sim_bold"]).reshape(N, -1)).to("cuda:0")
    bold_len = bold.shape[1] // nodes
    fc = torch.full(ref["sim_fc_trils"].shape, float("nan"), dtype=torch.float64, device="cuda:0")
    fcd = torch.full(ref["sim_fcd_trils"].shape, float("nan"), dtype=torch.float64, device="cuda:0")
    assert f(bold.data_ptr(), N, bold_len, nodes, rm, ws, step, 1, 0, fc.data_ptr(), fcd.data_ptr(), None) == 0
    fc.fill_(float("nan"))
    assert f(bold.data_ptr(), N, bold_len, nodes, rm, ws, step, 1, 0, fc.data_ptr(), None, None) == 0, \
        L.cbnm_last_error()
    torch.cuda.synchronize()
    np.testing.assert_allclose(fc.cpu().numpy(), ref["sim_fc_trils"], rtol=RTOL, atol=ATOL)


def test_noalloc_rejects_sizes_beyond_scratch():
    """Checked on the host before any CUDA call: 1000 nodes x 10 windows of window FCs
    (40 MB) exceed the 32 MiB scratch.  The pointers are never dereferenced."""
    L, f = _noalloc()
    nodes, bold_len = 1000, 60
    fake = C.c_void_p(256)
    rc = f(fake, 4, bold_len, nodes, 30, 10, 2, 1, 0, fake, fake, None)
    assert rc == 1
    msg = L.cbnm_last_error().decode()
    assert "scratch" in msg and str(SCRATCH_BYTES) in msg, msg


def test_noalloc_rejects_bad_configs():
    L, f = _noalloc()
    fake = C.c_void_p(256)
    assert f(fake, 4, 60, 100, 59, 10, 2, 1, 0, fake, fake, None) == 3      # one volume left for FC
    assert f(fake, 4, 60, 99, 30, 10, 2, 1, 1, fake, fake, None) == 3       # odd nodes with exc_interhemispheric
    assert f(fake, 4, 60, 100, 30, 10, 0, 1, 0, fake, fake, None) == 3      # window_step 0
    assert f(fake, 4, 60, 2, 30, 10, 2, 1, 1, fake, fake, None) == 3        # 2 nodes, one per hemisphere: no pair
    assert "no node pairs" in L.cbnm_last_error().decode()
    assert f(fake, 4, 60, 2, 30, 10, 2, 1, 1, fake, None, None) == 3        # the same for FC only
    assert f(None, 4, 60, 100, 30, 10, 2, 1, 0, fake, fake, None) == 1      # no BOLD
    assert "BOLD" in L.cbnm_last_error().decode() or "bold" in L.cbnm_last_error().decode()
