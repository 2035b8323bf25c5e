"""dtb_gain_contract: the gain contraction of one block in the caller's device memory, through
the C ABI, against the FP64 oracle (rel tolerance 1e-12 for FP64 inputs, 2e-5 for FP32)."""
import ctypes

import numpy as np
import pytest

import oracle
from dtb import _lib

pytestmark = pytest.mark.gpu


def _contract(G, f1, f2):
    import torch
    L = _lib.load()
    dtype = _lib.DTB_DTYPE_F64 if G.dtype == torch.float64 else _lib.DTB_DTYPE_F32
    out = torch.zeros(G.shape[0], dtype=torch.float64, device=G.device)
    s = torch.cuda.current_stream()
    _lib.check(L.dtb_gain_contract(dtype, ctypes.c_void_p(G.data_ptr()), G.shape[0], G.shape[1], G.shape[2],
                                   ctypes.c_void_p(f1.data_ptr()), ctypes.c_void_p(f2.data_ptr()),
                                   ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(s.cuda_stream)))
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("dt", ["f64", "f32"])
@pytest.mark.parametrize("shape", [(8, 5, 8), (128, 128, 128), (64, 300, 64), (3, 2048, 256)])
def test_gain_contract_matches_oracle(cuda, dt, shape):
    import torch
    tdt = torch.float64 if dt == "f64" else torch.float32
    g = torch.Generator(device="cuda")
    g.manual_seed(sum(shape))
    G = (10 ** (-6 * torch.rand(shape, generator=g, device="cuda", dtype=torch.float64))).to(tdt)
    f1 = torch.rand(shape[1], generator=g, device="cuda", dtype=torch.float64).to(tdt)
    f2 = torch.rand(shape[2], generator=g, device="cuda", dtype=torch.float64).to(tdt)
    got = _contract(G, f1, f2)
    exp = oracle.gain_rows(G.double().cpu().numpy(), 0, shape[0], f1.double().cpu().numpy(), f2.double().cpu().numpy())
    tol = 1e-12 if dt == "f64" else 2e-5
    assert np.max(np.abs(got - exp)) / np.max(np.abs(exp)) <= tol


def test_gain_contract_rejects_bad_shapes(cuda):
    import torch
    L = _lib.load()
    G = torch.zeros(4, 4, 12, device="cuda", dtype=torch.float32)
    f = torch.zeros(16, device="cuda", dtype=torch.float32)
    out = torch.zeros(4, device="cuda", dtype=torch.float64)
    rc = L.dtb_gain_contract(_lib.DTB_DTYPE_F32, ctypes.c_void_p(G.data_ptr()), 4, 4, 12,
                             ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(f.data_ptr()),
                             ctypes.c_void_p(out.data_ptr()), None)
    assert rc == _lib.DTB_EINVAL  # n2 = 12 is not a multiple of 8
    assert L.dtb_gain_contract(_lib.DTB_DTYPE_F32, None, 4, 4, 16, None, None, None, None) == _lib.DTB_EINVAL


def test_gain_contract_status_reports_a_bounded_wait_that_gave_up(cuda):
    """A timed-out wait of the contraction is reported by dtb_gain_contract_status, once: the
    flag is raised through the same give-up path by a kernel whose wait runs out after 50 ms."""
    import torch
    L = _lib.load()
    G = torch.rand(16, 8, 8, device="cuda", dtype=torch.float64)
    f = torch.rand(8, device="cuda", dtype=torch.float64)
    ref = _contract(G, f, f)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.dtb_gain_contract_status(s) == _lib.DTB_OK
    _lib.check(L.dtb_selftest_gain_contract_timeout(0, 0.05, s))
    assert L.dtb_gain_contract_status(s) == _lib.DTB_ETIMEOUT
    assert b"gave up" in L.dtb_last_error()
    assert L.dtb_gain_contract_status(s) == _lib.DTB_OK  # read and cleared
    # the next contraction starts from a clear flag and is correct
    _lib.check(L.dtb_selftest_gain_contract_timeout(0, 0.05, s))
    assert np.array_equal(_contract(G, f, f), ref)
    assert L.dtb_gain_contract_status(s) == _lib.DTB_OK
