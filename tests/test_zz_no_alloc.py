"""The allocation-free factorisation entry point, bta_pobtaf_noalloc, called
through the C ABI.

Some callers cannot allocate device memory (a host framework's pool allocator
owns the GPU, or a latency-critical loop cannot pay for cudaFree's device-wide
synchronisation).  For them the library keeps its factorisation scratch in a
fixed device array; this test checks that this variant gives the results of
the ordinary handle-based bta_pobtaf, on two calls in a row (the second call
reuses the array the first one left behind), and that a problem too large for
the array is refused up front.  It lives in a file of its own that pytest
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


def test_noalloc_rejects_blocks_beyond_its_scratch():
    import torch

    from dalia_b200 import _lib

    lib = _lib.load()
    assert lib.bta_noalloc_scratch_bytes() == 2 << 20
    n, b, a = 2, 4096, 6
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = _lib.ptr(dummy)
    rc = lib.bta_pobtaf_noalloc(n, b, a, p, p, p, p, None, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == _lib.BTA_ERR_INVALID
