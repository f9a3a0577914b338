"""The allocation-free factorisation entry point, bta_pobtaf_noalloc, called
through the C ABI.

Some callers cannot allocate device memory (a host framework's pool allocator
owns the GPU, or a latency-critical loop cannot pay for cudaFree's device-wide
synchronisation).  For them the library keeps its factorisation scratch in a
fixed device array; this test checks that this variant gives the results of
the ordinary handle-based bta_pobtaf, on two calls in a row (the second call
reuses the array the first one left behind), at the largest accepted sizes,
that a non-positive pivot is reported, and that a problem beyond the limits
is refused up front.  It lives in a file of its own that pytest
collects last."""
import ctypes

import numpy as np
import pytest

from golden_util import rel
from oracle import bta_ref

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _dev(*arrs):
    import torch

    return [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in arrs]


def test_noalloc_matches_handle_path_twice():
    import torch

    from dalia_b200 import _lib

    lib = _lib.load()
    h = _lib.handle()
    stream = torch.cuda.current_stream().cuda_stream
    for call, (n, b, a) in enumerate([(4, 200, 5), (3, 300, 6)]):
        rng = np.random.default_rng(40 + call)
        blocks = bta_ref.random_bta(n, b, a, rng)
        ref = _dev(*blocks)
        got = _dev(*blocks)
        info_ref = ctypes.c_int64(-1)
        rc = lib.bta_pobtaf(h.bind_stream(), n, b, a, *[_lib.ptr(t) for t in ref], ctypes.byref(info_ref))
        assert rc == 0 and info_ref.value == 0
        info = ctypes.c_int64(-1)
        rc = lib.bta_pobtaf_noalloc(n, b, a, *[_lib.ptr(t) for t in got], ctypes.byref(info),
                                    ctypes.c_void_p(stream))
        assert rc == 0 and info.value == 0, (rc, info.value)
        torch.cuda.synchronize()
        for r, g in zip(ref, got):
            assert rel(g.cpu().numpy(), r.cpu().numpy()) < TOL


@pytest.mark.parametrize("n,b,a", [(3, 200, 100), (2, 2048, 128), (5, 64, 0)])
def test_noalloc_matches_handle_path_at_its_limits(n, b, a):
    """A wide arrowhead (two 64-row arrow tiles, a two-tile tip) and the
    largest accepted block and arrowhead sizes."""
    import torch

    from dalia_b200 import _lib

    lib = _lib.load()
    h = _lib.handle()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    blocks = bta_ref.random_bta(n, b, a, np.random.default_rng(7 + b + a))
    if a == 0:
        blocks = blocks[:2] + (np.zeros((n, 0, b)), np.zeros((0, 0)))
    ref = _dev(*blocks)
    got = _dev(*blocks)
    ptr = lambda ts: [_lib.ptr(t) if t.numel() else None for t in ts]  # noqa: E731
    info_ref = ctypes.c_int64(-1)
    assert lib.bta_pobtaf(h.bind_stream(), n, b, a, *ptr(ref), ctypes.byref(info_ref)) == 0
    # asynchronous call, then the status read-back of the scratch array
    assert lib.bta_pobtaf_noalloc(n, b, a, *ptr(got), None, stream) == 0
    info = ctypes.c_int64(-1)
    assert lib.bta_noalloc_get_status(ctypes.byref(info), stream) == 0 and info.value == 0
    for r, g in zip(ref, got):
        if r.numel():
            assert rel(g.cpu().numpy(), r.cpu().numpy()) < TOL


def test_noalloc_reports_non_spd_pivot():
    """A matrix that is not positive definite (built on the host: the third
    diagonal entry of the second block made negative) gives BTA_ERR_NOT_SPD
    and the 1-based global index of the failing pivot, both from the call
    itself and, after an asynchronous call, from bta_noalloc_get_status; the
    next good call clears it."""
    import torch

    from dalia_b200 import _lib

    lib = _lib.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    n, b, a = 3, 150, 4
    D, L, Ab, T = bta_ref.random_bta(n, b, a, np.random.default_rng(3))
    D = D.copy()
    D[1, 2, 2] = -abs(D[1, 2, 2]) - 1e3
    for synchronous in (True, False):
        got = _dev(D, L, Ab, T)
        info = ctypes.c_int64(-1)
        if synchronous:
            rc = lib.bta_pobtaf_noalloc(n, b, a, *[_lib.ptr(t) for t in got], ctypes.byref(info), stream)
        else:
            assert lib.bta_pobtaf_noalloc(n, b, a, *[_lib.ptr(t) for t in got], None, stream) == 0
            rc = lib.bta_noalloc_get_status(ctypes.byref(info), stream)
        assert rc == _lib.BTA_ERR_NOT_SPD
        assert info.value == b + 3  # global row b + 2, 1-based
    good = _dev(*bta_ref.random_bta(n, b, a, np.random.default_rng(4)))
    info = ctypes.c_int64(-1)
    assert lib.bta_pobtaf_noalloc(n, b, a, *[_lib.ptr(t) for t in good], ctypes.byref(info), stream) == 0
    assert info.value == 0


def test_noalloc_rejects_sizes_beyond_its_limits():
    import torch

    from dalia_b200 import _lib

    lib = _lib.load()
    assert lib.bta_noalloc_scratch_bytes() == 2 << 20
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = _lib.ptr(dummy)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for n, b, a in [(2, 2049, 6), (2, 4096, 6), (2, 200, 129)]:
        assert lib.bta_pobtaf_noalloc(n, b, a, p, p, p, p, None, stream) == _lib.BTA_ERR_INVALID
