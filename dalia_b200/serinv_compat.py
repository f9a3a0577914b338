"""Serinv-compatible entry points backed by the CUDA library.

The reference imports ``from serinv.algs import pobtaf, pobtas, pobtasi, pobtf,
pobts, pobtsi`` (``src/dalia/solvers/structured_solver.py:12-15``) and calls
them in place on four FP64 arrays (call sites ``:83-93, :112-140, :176-186``).
These functions keep those names, argument meanings and in-place semantics.

Accepted arrays: torch CUDA tensors (used in place, no copies), objects with
``__cuda_array_interface__`` (e.g. CuPy, viewed through torch), and NumPy
host arrays (copied to the device and back, so the call is a drop-in for the
reference's NumPy path).  A non-positive-definite block raises
``numpy.linalg.LinAlgError`` (a ``ValueError``), like ``numpy.linalg.cholesky``.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


def _torch():
    import torch

    return torch


class _Arr:
    """A device view of one argument, with write-back for host arrays."""

    def __init__(self, x, name):
        torch = _torch()
        self.orig = x
        self.host = False
        if x is None:
            self.t = None
        elif isinstance(x, torch.Tensor):
            if not x.is_cuda:
                self.host = True
                self.t = x.to("cuda", dtype=torch.float64).contiguous()
            else:
                if x.dtype != torch.float64 or not x.is_contiguous():
                    raise ValueError(f"{name}: needs a contiguous float64 CUDA tensor")
                self.t = x
        elif isinstance(x, np.ndarray):
            if x.dtype != np.float64:
                raise ValueError(f"{name}: needs float64")
            self.host = True
            self.t = torch.from_numpy(np.ascontiguousarray(x)).to("cuda")
        elif hasattr(x, "__cuda_array_interface__"):
            t = torch.as_tensor(x, device="cuda")
            if t.dtype != torch.float64 or not t.is_contiguous():
                raise ValueError(f"{name}: needs a contiguous float64 device array")
            self.t = t
        else:
            raise TypeError(f"{name}: unsupported array type {type(x)}")

    def writeback(self):
        if not self.host:
            return
        torch = _torch()
        if isinstance(self.orig, np.ndarray):
            self.orig[...] = self.t.cpu().numpy().reshape(self.orig.shape)
        else:
            self.orig.copy_(self.t.reshape(self.orig.shape).to(self.orig.device))


def _shapes(D, L, Ab, T):
    n, b = int(D.shape[0]), int(D.shape[1])
    if D.shape != (n, b, b):
        raise ValueError("A_diagonal_blocks must be (n, b, b)")
    if n > 1 and (L is None or tuple(L.shape) != (n - 1, b, b)):
        raise ValueError("A_lower_diagonal_blocks must be (n-1, b, b)")
    a = 0
    if Ab is not None and T is not None:
        a = int(Ab.shape[1])
        if tuple(Ab.shape) != (n, a, b) or tuple(T.shape) != (a, a):
            raise ValueError("arrow blocks must be (n, a, b) and (a, a)")
    return n, b, a


def _call(fn, *args):
    return fn(*args)


def pobtaf(A_diagonal_blocks, A_lower_diagonal_blocks, A_arrow_bottom_blocks, A_arrow_tip_block,
           device_streaming: bool = False):
    """In-place BTA Cholesky (Serinv ``pobtaf``)."""
    arrs = [_Arr(x, nm) for x, nm in zip(
        (A_diagonal_blocks, A_lower_diagonal_blocks, A_arrow_bottom_blocks, A_arrow_tip_block),
        ("A_diagonal_blocks", "A_lower_diagonal_blocks", "A_arrow_bottom_blocks", "A_arrow_tip_block"))]
    D, L, Ab, T = (a.t for a in arrs)
    n, b, a = _shapes(D, L, Ab, T)
    h = _lib.handle(D.device)
    info = ctypes.c_int64(0)
    rc = _lib.load().bta_pobtaf(h.bind_stream(), n, b, a, _lib.ptr(D), _lib.ptr(L if n > 1 else None),
                                _lib.ptr(Ab if a else None), _lib.ptr(T if a else None), ctypes.byref(info))
    _lib.check(rc, f"pobtaf (leading minor {info.value} not positive definite)" if rc == 3 else "pobtaf")
    for x in arrs:
        x.writeback()


def pobtf(A_diagonal_blocks, A_lower_diagonal_blocks, device_streaming: bool = False):
    """In-place BT Cholesky (Serinv ``pobtf``)."""
    pobtaf(A_diagonal_blocks, A_lower_diagonal_blocks, None, None)


def pobtas(L_diagonal_blocks, L_lower_diagonal_blocks, L_arrow_bottom_blocks, L_arrow_tip_block, B,
           trans: str = "N", device_streaming: bool = False):
    """One triangular sweep in place on ``B`` (Serinv ``pobtas``);
    ``trans="N"`` solves ``L y = B``, ``"C"``/``"T"`` solves ``L^T x = B``."""
    if trans not in ("N", "C", "T"):
        raise ValueError(f"unknown trans {trans!r}")
    arrs = [_Arr(x, nm) for x, nm in zip(
        (L_diagonal_blocks, L_lower_diagonal_blocks, L_arrow_bottom_blocks, L_arrow_tip_block),
        ("L_diagonal_blocks", "L_lower_diagonal_blocks", "L_arrow_bottom_blocks", "L_arrow_tip_block"))]
    D, L, Ab, T = (x.t for x in arrs)
    n, b, a = _shapes(D, L, Ab, T)
    rb = _Arr(B, "B")
    Bt = rb.t
    N = n * b + a
    if Bt.shape[0] != N:
        raise ValueError(f"B must have {N} rows")
    cols = 1 if Bt.dim() == 1 else int(Bt.shape[1])
    h = _lib.handle(D.device)
    lib = _lib.load()
    tr = 0 if trans == "N" else 1
    if cols == 1:
        col = Bt.reshape(N)
        rc = lib.bta_pobtas(h.bind_stream(), n, b, a, _lib.ptr(D), _lib.ptr(L if n > 1 else None),
                            _lib.ptr(Ab if a else None), _lib.ptr(T if a else None), _lib.ptr(col), tr)
        _lib.check(rc, "pobtas")
    else:
        for j in range(cols):
            col = Bt[:, j].contiguous()
            rc = lib.bta_pobtas(h.bind_stream(), n, b, a, _lib.ptr(D), _lib.ptr(L if n > 1 else None),
                                _lib.ptr(Ab if a else None), _lib.ptr(T if a else None), _lib.ptr(col), tr)
            _lib.check(rc, "pobtas")
            Bt[:, j] = col
    rb.writeback()
    return B


def pobts(L_diagonal_blocks, L_lower_diagonal_blocks, B, trans: str = "N", device_streaming: bool = False):
    return pobtas(L_diagonal_blocks, L_lower_diagonal_blocks, None, None, B, trans)


def pobtasi(L_diagonal_blocks, L_lower_diagonal_blocks, L_arrow_bottom_blocks, L_arrow_tip_block,
            device_streaming: bool = False):
    """In-place selected inversion of the factor (Serinv ``pobtasi``)."""
    arrs = [_Arr(x, nm) for x, nm in zip(
        (L_diagonal_blocks, L_lower_diagonal_blocks, L_arrow_bottom_blocks, L_arrow_tip_block),
        ("L_diagonal_blocks", "L_lower_diagonal_blocks", "L_arrow_bottom_blocks", "L_arrow_tip_block"))]
    D, L, Ab, T = (x.t for x in arrs)
    n, b, a = _shapes(D, L, Ab, T)
    h = _lib.handle(D.device)
    rc = _lib.load().bta_pobtasi(h.bind_stream(), n, b, a, _lib.ptr(D), _lib.ptr(L if n > 1 else None),
                                 _lib.ptr(Ab if a else None), _lib.ptr(T if a else None))
    _lib.check(rc, "pobtasi")
    for x in arrs:
        x.writeback()


def pobtsi(L_diagonal_blocks, L_lower_diagonal_blocks, device_streaming: bool = False):
    pobtasi(L_diagonal_blocks, L_lower_diagonal_blocks, None, None)


def logdet(L_diagonal_blocks, L_arrow_tip_block=None, sparsity: str = "bta") -> float:
    """``2 sum log diag`` of the factor; the tip only for ``"bta"``."""
    D = _Arr(L_diagonal_blocks, "L_diagonal_blocks").t
    T = None if L_arrow_tip_block is None else _Arr(L_arrow_tip_block, "L_arrow_tip_block").t
    n, b = int(D.shape[0]), int(D.shape[1])
    a = 0 if T is None else int(T.shape[0])
    h = _lib.handle(D.device)
    out = ctypes.c_double(0.0)
    rc = _lib.load().bta_logdet(h.bind_stream(), n, b, a, _lib.ptr(D), _lib.ptr(T),
                                1 if (sparsity == "bta" and a) else 0, None, ctypes.byref(out))
    _lib.check(rc, "logdet")
    return float(out.value)
