"""apirl_likelihood_noalloc, the entry point for callers that cannot allocate
device memory (their device memory belongs to another allocator, or a
cudaMalloc would stall or fail where they run), checked through the C ABI
against apirl_likelihood on two calls in a row.

This file is named to be collected last; it passes alone in a fresh process
and after the other tests.  Tolerance: 1e-9 relative, the FP64 likelihood
tolerance of the other tests (the two entry points sum in different orders)."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from apirl_b200 import _lib  # noqa: E402


@pytest.fixture(scope="module")
def lib():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return _lib.load()


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_likelihood_matches_allocating_entry_point_twice(lib):
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    g = torch.Generator(device=dev).manual_seed(1)
    cases = [(1_000_003, 0), (9_437_185, 1)]  # odd sizes: partial last chunk
    for n, gt0 in cases:
        est = torch.rand(n, generator=g, device=dev, dtype=torch.float32) * 4.0
        est[::97] = 0.0
        if gt0:
            est[::89] = -0.5  # skipped by the e > 0 rule
        meas = torch.poisson(est.clamp(min=0) * 3.0, generator=g)
        want = torch.zeros(1, dtype=torch.float64, device=dev)
        _lib.check(lib.apirl_likelihood(n, _p(est), _p(meas), gt0, _p(want), stream))
        for _ in range(2):
            got = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
            _lib.check(lib.apirl_likelihood_noalloc(n, _p(est), _p(meas), gt0, _p(got), stream))
            torch.cuda.synchronize()
            w, v = want.item(), got.item()
            assert np.isfinite(v)
            assert abs(v - w) <= 1e-9 * abs(w), (n, gt0, v, w)


def test_noalloc_rejects_sizes_beyond_its_scratch(lib):
    n = int(lib_max())
    st = lib.apirl_likelihood_noalloc(n + 1, ctypes.c_void_p(16), ctypes.c_void_p(16), 0, ctypes.c_void_p(16), None)
    assert st == _lib.APIRL_ERR_INVALID
    assert b"scratch limit" in lib.apirl_last_error()


def lib_max():
    return 65536 * 4096
