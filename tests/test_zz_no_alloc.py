"""dtb_gain_contract_noalloc through the C ABI.

The entry point serves callers that cannot call cudaMalloc (a host whose device memory
belongs to its own pool allocator, such as a Julia session whose CUDA.jl pool owns the heap,
or a loop that cannot afford an allocator call): its scratch is a static device array. It must
give the same result as dtb_gain_contract, whose scratch the library allocates, on two calls in
a row (the array keeps the previous call's contents), and it must not change the device's free
memory once set up. This file is collected last so that a failure here leaves every other test
already run.
"""
import ctypes

import numpy as np
import pytest

from dtb import _lib

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-12, "f32": 2e-5}


def _call(fn, G, f1, f2, out):
    import torch
    dtype = _lib.DTB_DTYPE_F64 if G.dtype == torch.float64 else _lib.DTB_DTYPE_F32
    s = torch.cuda.current_stream()
    _lib.check(fn(dtype, ctypes.c_void_p(G.data_ptr()), G.shape[0], G.shape[1], G.shape[2],
                  ctypes.c_void_p(f1.data_ptr()), ctypes.c_void_p(f2.data_ptr()),
                  ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(s.cuda_stream)))
    torch.cuda.synchronize()
    return out.cpu().numpy().copy()


def _inputs(shape, tdt, seed):
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    G = (10 ** (-6 * torch.rand(shape, generator=g, device="cuda", dtype=torch.float64))).to(tdt)
    f1 = torch.rand(shape[1], generator=g, device="cuda", dtype=torch.float64).to(tdt)
    f2 = torch.rand(shape[2], generator=g, device="cuda", dtype=torch.float64).to(tdt)
    return G, f1, f2


@pytest.mark.parametrize("dt,shape", [("f64", (128, 128, 128)), ("f32", (256, 512, 256)),
                                      ("f32", (1024, 1024, 1024))])
def test_noalloc_matches_allocating_entry_on_two_calls(cuda, dt, shape):
    import torch
    L = _lib.load()
    tdt = torch.float64 if dt == "f64" else torch.float32
    out = torch.zeros(shape[0], dtype=torch.float64, device="cuda")
    out2 = torch.zeros_like(out)
    # two different inputs back to back: the second call must not see the first call's scratch
    cases = [_inputs(shape, tdt, 1), _inputs(shape, tdt, 2)]
    refs = [_call(L.dtb_gain_contract, *c, out) for c in cases]
    _call(L.dtb_gain_contract_noalloc, *cases[0], out2)  # first call on this device: set-up
    free0 = torch.cuda.mem_get_info()[0]
    got = [_call(L.dtb_gain_contract_noalloc, *c, out2) for c in cases]
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0  # no device memory taken by the calls
    for g, r in zip(got, refs):
        assert np.max(np.abs(g - r)) / np.max(np.abs(r)) <= TOL[dt]
    assert not np.array_equal(got[0], got[1])
    del cases
    torch.cuda.empty_cache()


def test_noalloc_rejects_blocks_beyond_the_static_limit(cuda):
    import torch
    L = _lib.load()
    G = torch.zeros(8, device="cuda", dtype=torch.float32)
    out = torch.zeros(8, device="cuda", dtype=torch.float64)
    p = ctypes.c_void_p(G.data_ptr())
    # n1 + n2 over 16384: refused on the host before any launch
    rc = L.dtb_gain_contract_noalloc(_lib.DTB_DTYPE_F32, p, 8, 16384, 64, p, p, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == _lib.DTB_EINVAL and b"static scratch" in L.dtb_last_error()
    # too many work units: 40000 output rows of a 1-tile contraction
    rc = L.dtb_gain_contract_noalloc(_lib.DTB_DTYPE_F32, p, 40000, 8, 8, p, p, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == _lib.DTB_EINVAL and b"work units" in L.dtb_last_error()


def test_noalloc_reports_a_bounded_wait_that_gave_up(cuda):
    """The allocation-free entry reports a timed-out wait through dtb_gain_contract_status like
    the allocating one; its flag lives in the static array and the next call clears it."""
    import torch
    L = _lib.load()
    G, f1, f2 = _inputs((64, 64, 64), torch.float64, 3)
    out = torch.zeros(64, dtype=torch.float64, device="cuda")
    ref = _call(L.dtb_gain_contract_noalloc, G, f1, f2, out)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.dtb_gain_contract_status(s) == _lib.DTB_OK
    free0 = torch.cuda.mem_get_info()[0]
    _lib.check(L.dtb_selftest_gain_contract_timeout(1, 0.05, s))
    assert L.dtb_gain_contract_status(s) == _lib.DTB_ETIMEOUT
    assert L.dtb_gain_contract_status(s) == _lib.DTB_OK
    _lib.check(L.dtb_selftest_gain_contract_timeout(1, 0.05, s))
    assert np.array_equal(_call(L.dtb_gain_contract_noalloc, G, f1, f2, out), ref)
    assert L.dtb_gain_contract_status(s) == _lib.DTB_OK
    assert torch.cuda.mem_get_info()[0] == free0
