"""ctypes binding of ``libdalia_bta.so`` (C ABI in ``include/dalia_bta.h``).

There is no CPU fallback: every entry point needs the in-tree CUDA library and
a CUDA device, and raises if either is missing.
"""

from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdalia_bta.so")

BTA_OK = 0
BTA_ERR_INVALID = 1
BTA_ERR_CUDA = 2
BTA_ERR_NOT_SPD = 3
BTA_ERR_TIMEOUT = 4
BTA_ERR_ALLOC = 5

# exported symbol -> (restype, argtypes)
_c_void_p = ctypes.c_void_p
_i64 = ctypes.c_int64
_int = ctypes.c_int
_pi64 = ctypes.POINTER(ctypes.c_int64)
_pdbl = ctypes.POINTER(ctypes.c_double)
_dbl = ctypes.c_double

BTA_PREC_FP64 = 0
BTA_PREC_TF32X3 = 1
BTA_PREC_I8SLICE = 2

SIGNATURES = {
    "bta_create": (_int, [ctypes.POINTER(_c_void_p)]),
    "bta_destroy": (_int, [_c_void_p]),
    "bta_set_stream": (_int, [_c_void_p, _c_void_p]),
    "bta_error_string": (ctypes.c_char_p, [_int]),
    "bta_workspace_bytes": (ctypes.c_size_t, [_c_void_p]),
    "bta_pobtaf": (_int, [_c_void_p, _i64, _i64, _i64, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _pi64]),
    "bta_pobtas": (_int, [_c_void_p, _i64, _i64, _i64, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _int]),
    "bta_pobtaf_batched": (_int, [_c_void_p, _int, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                                  _c_void_p, _pi64]),
    "bta_pobtaf_batched_ex": (_int, [_c_void_p, _int, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                                     _c_void_p, _c_void_p, _pi64, _int]),
    "bta_pobtas_batched": (_int, [_c_void_p, _int, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                                  _c_void_p, _c_void_p, _int]),
    "bta_pobtasi_batched": (_int, [_c_void_p, _int, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                                   _c_void_p, _c_void_p]),
    "bta_pobtasi_batched_ex": (_int, [_c_void_p, _int, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                                      _c_void_p, _c_void_p, _int]),
    "bta_block_inverses": (_int, [_c_void_p, _int, _c_void_p, _c_void_p, _c_void_p, _c_void_p]),
    "bta_pobtas_inv_batched": (_int, [_c_void_p, _int, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                                      _c_void_p, _c_void_p, _c_void_p, _int]),
    "bta_pobtasi_batched_v": (_int, [_c_void_p, _int, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                                     _c_void_p, _c_void_p, _c_void_p, _int]),
    "bta_gemm": (_int, [_c_void_p, _int, _i64, _i64, _i64, _dbl, _c_void_p, _i64, _int, _c_void_p, _i64, _int,
                        _dbl, _c_void_p, _i64, _int, _int]),
    "bta_pobtasi": (_int, [_c_void_p, _i64, _i64, _i64, _c_void_p, _c_void_p, _c_void_p, _c_void_p]),
    "bta_logdet": (_int, [_c_void_p, _i64, _i64, _i64, _c_void_p, _c_void_p, _int, _c_void_p, _pdbl]),
    "bta_get_status": (_int, [_c_void_p, _pi64]),
    "bta_reset_status": (_int, [_c_void_p]),
    "bta_launch_count": (ctypes.c_longlong, []),
    "bta_pobtaf_noalloc": (_int, [_i64, _i64, _i64, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _pi64, _c_void_p]),
    "bta_noalloc_scratch_bytes": (ctypes.c_size_t, []),
    "bta_noalloc_get_status": (_int, [_pi64, _c_void_p]),
    "bta_prof_enable": (_int, [_int]),
    "bta_prof_mask": (_int, [_int]),
    "bta_prof_read": (_int, [_pdbl, ctypes.POINTER(ctypes.c_longlong)]),
    "bta_panel_task_list": (_int, [_int, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _int, ctypes.POINTER(_int)]),
    "bta_panel_task_list_ex": (_int, [_int, _c_void_p, _c_void_p, _c_void_p, _int, _int, _c_void_p, _int,
                                      ctypes.POINTER(_int)]),
    "bta_panel_task_list_all": (_int, [_int, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _int, _int, _c_void_p, _int,
                                       ctypes.POINTER(_int)]),
    "bta_tune_report": (_int, [ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "bta_tune_pending": (_int, []),
    "bta_gather_coo": (_int, [_c_void_p, _i64, _i64, _i64, _c_void_p, _c_void_p, _i64, _int,
                              _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p]),
    "bta_scatter_coo": (_int, [_c_void_p, _i64, _i64, _i64, _c_void_p, _c_void_p, _c_void_p, _i64, _int,
                               _c_void_p, _c_void_p, _c_void_p, _c_void_p]),
    "bta_assemble_prior": (_int, [_c_void_p, _i64, _i64, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                                  _c_void_p]),
    "bta_add_entries": (_int, [_c_void_p, _i64, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                               ctypes.c_double, _c_void_p]),
    "bta_arrow_tip": (_int, [_c_void_p, _i64, _i64, _c_void_p, _c_void_p, ctypes.c_double, ctypes.c_double,
                             _c_void_p, _int, _c_void_p]),
    "bta_block_inner": (_int, [_c_void_p, _i64, _i64, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                               _c_void_p]),
    "bta_block_quad": (_int, [_c_void_p, _i64, _i64, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p]),
    "bta_gather_dot": (_int, [_c_void_p, _i64, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _int, _c_void_p]),
    "bta_assemble_prior_mv": (_int, [_c_void_p, _i64, _i64, _i64, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                                     _c_void_p, _c_void_p]),
    "bta_block_inner_mv": (_int, [_c_void_p, _i64, _i64, _i64, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                                  _c_void_p, _c_void_p]),
    "bta_block_quad_mv": (_int, [_c_void_p, _i64, _i64, _i64, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                                 _c_void_p]),
    "bta_kron_symv": (_int, [_c_void_p, _i64, _i64, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _dbl,
                             _dbl, _c_void_p]),
    "bta_poisson_terms": (_int, [_c_void_p, _i64, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                                 _int, _c_void_p]),
    "bta_block_bilinear": (_int, [_c_void_p, _i64, _i64, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                                  _c_void_p]),
    "bta_obs_quad": (_int, [_c_void_p, _i64, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _i64, _c_void_p, _c_void_p,
                            _c_void_p, _c_void_p]),
    "bta_csr_spmv": (_int, [_c_void_p, _i64, _c_void_p, _c_void_p, _c_void_p, _c_void_p, ctypes.c_double,
                            ctypes.c_double, _c_void_p]),
    "bta_symv": (_int, [_c_void_p, _i64, _i64, _i64, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                        _c_void_p]),
    "bta_dot": (_int, [_c_void_p, _i64, _c_void_p, _c_void_p, _c_void_p, _int, _c_void_p]),
    "bta_axpby": (_int, [_c_void_p, _i64, ctypes.c_double, _c_void_p, ctypes.c_double, _c_void_p]),
}

_lib = None
_lock = threading.Lock()


def load() -> ctypes.CDLL:
    """Load the CUDA library (does not touch the GPU)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python -m dalia_b200.build` (nvcc, sm_100a)")
            lib = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


class BTAError(RuntimeError):
    pass


def check(rc: int, what: str = "") -> None:
    if rc == BTA_OK:
        return
    msg = load().bta_error_string(rc).decode()
    if rc == BTA_ERR_NOT_SPD:
        raise np.linalg.LinAlgError(f"{what}: {msg}")
    if rc == BTA_ERR_INVALID:
        raise ValueError(f"{what}: {msg}")
    raise BTAError(f"{what}: {msg} (code {rc})")


def _require_cuda():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("dalia_b200 needs a CUDA device (B200, sm_100a); no CPU fallback exists")
    return torch


class Handle:
    """Owns a ``bta_handle_t`` bound to one device; follows torch's current stream."""

    def __init__(self, device=None):
        torch = _require_cuda()
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        with torch.cuda.device(self.device):
            torch.cuda.init()
            torch.empty(1, device=self.device)  # make the primary context current
            h = _c_void_p()
            check(load().bta_create(ctypes.byref(h)), "bta_create")
        self.h = h
        self._stream = None

    def bind_stream(self):
        import torch

        s = torch.cuda.current_stream(self.device).cuda_stream
        if s != self._stream:
            check(load().bta_set_stream(self.h, _c_void_p(s)), "bta_set_stream")
            self._stream = s
        return self.h

    def workspace_bytes(self) -> int:
        return int(load().bta_workspace_bytes(self.h))

    def __del__(self):
        try:
            if getattr(self, "h", None) is not None and _lib is not None:
                _lib.bta_destroy(self.h)
        except Exception:
            pass


_handles: dict = {}


def handle(device=None) -> Handle:
    torch = _require_cuda()
    dev = torch.cuda.current_device() if device is None else torch.device(device).index
    h = _handles.get(dev)
    if h is None:
        h = _handles[dev] = Handle(dev)
    return h


def stream_ptr(device=None) -> ctypes.c_void_p:
    import torch

    return _c_void_p(torch.cuda.current_stream(device).cuda_stream)


def ptr(t) -> ctypes.c_void_p:
    """Device pointer of a torch tensor (None -> NULL)."""
    if t is None:
        return _c_void_p(0)
    return _c_void_p(t.data_ptr())


def tune_report():
    """The autotuner's decisions so far, one line each (``bta_tune_report``)."""
    lib = load()
    n = ctypes.c_size_t(0)
    lib.bta_tune_report(None, 0, ctypes.byref(n))
    buf = ctypes.create_string_buffer(n.value + 1)
    check(lib.bta_tune_report(buf, n.value + 1, ctypes.byref(n)), "tune_report")
    return [ln for ln in buf.value.decode().splitlines() if ln]
