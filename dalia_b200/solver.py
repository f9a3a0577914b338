"""``B200Solver``: DALIA's structured-solver interface on the CUDA library.

Mirrors ``SerinvSolver`` (``src/dalia/solvers/structured_solver.py:19-549``),
the implementation of DALIA's ``Solver`` ABC (``src/dalia/core/solver.py:9-63``):
same constructor arguments, same ``cholesky / solve / logdet /
selected_inversion / _structured_to_spmatrix / get_solver_memory`` methods,
same ``sparsity in {"bt", "bta"}`` semantics and the same errors.  The BTA
arrays live on the GPU for the solver's lifetime; sparse inputs are scattered
into them on the device (the structure is uploaded once and cached, like the
reference's GPU block-sort cache, ``:252-390``).

Differences, on purpose:
* ``cholesky(A)`` accepts a missing ``sparsity`` (default ``"bta"``); the
  reference's non-Gaussian path calls it that way (``src/dalia/core/dalia.py:1058``)
  and ``SerinvSolver`` would raise ``TypeError``.
"""

from __future__ import annotations

import time

import numpy as np
import scipy.sparse as sps

from . import _lib


def _check_sparsity(sparsity):
    if sparsity not in ("bt", "bta"):
        raise ValueError(f"Unknown sparsity pattern: {sparsity}. Use 'bt' or 'bta'.")


class B200Solver:
    """GPU BTA solver with the reference's ``Solver`` interface."""

    def __init__(self, config=None, diagonal_blocksize: int = None, n_diag_blocks: int = None,
                 arrowhead_blocksize: int = 0, device=None, **kwargs):
        import torch

        self.config = config
        self.diagonal_blocksize = int(diagonal_blocksize)
        self.n_diag_blocks = int(n_diag_blocks)
        self.arrowhead_blocksize = int(arrowhead_blocksize)
        self.h = _lib.handle(device)
        self.device = self.h.device
        n, b, a = self.n_diag_blocks, self.diagonal_blocksize, self.arrowhead_blocksize
        f64 = dict(dtype=torch.float64, device=self.device)
        self.A_diagonal_blocks = torch.empty((n, b, b), **f64)
        self.A_lower_diagonal_blocks = torch.empty((max(n - 1, 0), b, b), **f64)
        self.A_arrow_bottom_blocks = torch.empty((n, a, b), **f64) if a > 0 else None
        self.A_arrow_tip_block = torch.empty((a, a), **f64) if a > 0 else None
        self._coo_cache = {}
        self.total_bytes = 0
        self.t_cholesky = 0.0
        self.t_solve = 0.0

    # -- helpers -------------------------------------------------------------
    @property
    def _n(self):
        return self.n_diag_blocks

    def _dims(self, sparsity):
        a = self.arrowhead_blocksize if sparsity == "bta" else 0
        return self.n_diag_blocks, self.diagonal_blocksize, a

    def _ptrs(self, sparsity):
        P = _lib.ptr
        L = self.A_lower_diagonal_blocks if self.n_diag_blocks > 1 else None
        if sparsity == "bta" and self.arrowhead_blocksize > 0:
            return P(self.A_diagonal_blocks), P(L), P(self.A_arrow_bottom_blocks), P(self.A_arrow_tip_block)
        return P(self.A_diagonal_blocks), P(L), P(None), P(None)

    def _device_coo(self, A, lower_only=False):
        """Device copies of the COO structure of ``A`` (cached per pattern)."""
        import torch

        C = sps.coo_matrix(A)
        if lower_only:
            C = sps.tril(C).tocoo()
        key = (C.shape, C.nnz, lower_only, hash(C.row[: 64].tobytes()), hash(C.col[-64:].tobytes()))
        ent = self._coo_cache.get(key)
        if ent is None or not (np.array_equal(ent[2], C.row) and np.array_equal(ent[3], C.col)):
            r = torch.from_numpy(C.row.astype(np.int64)).to(self.device, non_blocking=False)
            c = torch.from_numpy(C.col.astype(np.int64)).to(self.device, non_blocking=False)
            ent = (r, c, C.row.copy(), C.col.copy())
            self._coo_cache[key] = ent
        return C, ent[0], ent[1]

    def _spmatrix_to_structured(self, A, sparsity):
        import torch

        _check_sparsity(sparsity)
        C, r, c = self._device_coo(A)
        v = torch.from_numpy(np.ascontiguousarray(C.data, dtype=np.float64)).to(self.device)
        n, b, a = self._dims(sparsity)
        D, L, Ab, T = self._ptrs("bta")
        rc = _lib.load().bta_scatter_coo(self.h.bind_stream(), n, b, self.arrowhead_blocksize, _lib.ptr(r),
                                         _lib.ptr(c), _lib.ptr(v), int(C.nnz), 1 if sparsity == "bt" else 0,
                                         D, L, Ab, T)
        _lib.check(rc, "scatter")

    # -- Solver interface ------------------------------------------------------
    def cholesky(self, A, sparsity: str = "bta") -> None:
        """Factor ``A`` (scipy sparse, or a ``(D, L, Ab, T)`` tuple of device
        tensors already in BTA layout) in place."""
        import torch

        _check_sparsity(sparsity)
        if isinstance(A, tuple):
            D, L, Ab, T = A
            self.A_diagonal_blocks.copy_(D)
            if self.n_diag_blocks > 1:
                self.A_lower_diagonal_blocks.copy_(L)
            if sparsity == "bta" and self.arrowhead_blocksize > 0:
                self.A_arrow_bottom_blocks.copy_(Ab)
                self.A_arrow_tip_block.copy_(T)
        else:
            self._spmatrix_to_structured(A, sparsity)
        tic = time.perf_counter()
        n, b, a = self._dims(sparsity)
        D, L, Ab, T = self._ptrs(sparsity)
        info = __import__("ctypes").c_int64(0)
        rc = _lib.load().bta_pobtaf(self.h.bind_stream(), n, b, a, D, L, Ab, T, __import__("ctypes").byref(info))
        if rc == _lib.BTA_ERR_NOT_SPD:
            raise np.linalg.LinAlgError(
                f"Matrix is not positive definite (leading minor of order {info.value})")
        _lib.check(rc, "cholesky")
        torch.cuda.current_stream(self.device).synchronize()
        self.t_cholesky += time.perf_counter() - tic

    def solve(self, rhs, sparsity: str = "bta"):
        """``Q^{-1} rhs`` in place (forward then backward sweep); returns rhs."""
        import torch

        _check_sparsity(sparsity)
        tic = time.perf_counter()
        n, b, a = self._dims(sparsity)
        host = isinstance(rhs, np.ndarray)
        x = torch.from_numpy(np.ascontiguousarray(rhs, dtype=np.float64)).to(self.device) if host else rhs
        if x.dim() != 1 or x.numel() != n * b + a:
            raise ValueError(f"rhs must be a vector of length {n * b + a}")
        D, L, Ab, T = self._ptrs(sparsity)
        lib = _lib.load()
        hd = self.h.bind_stream()
        _lib.check(lib.bta_pobtas(hd, n, b, a, D, L, Ab, T, _lib.ptr(x), 0), "solve")
        _lib.check(lib.bta_pobtas(hd, n, b, a, D, L, Ab, T, _lib.ptr(x), 1), "solve")
        if host:
            rhs[:] = x.cpu().numpy()
        else:
            torch.cuda.current_stream(self.device).synchronize()
        self.t_solve += time.perf_counter() - tic
        return rhs

    def logdet(self, sparsity: str = "bta") -> float:
        import ctypes

        _check_sparsity(sparsity)
        n, b, a = self._dims(sparsity)
        out = ctypes.c_double(0.0)
        T = self.A_arrow_tip_block if a > 0 else None
        rc = _lib.load().bta_logdet(self.h.bind_stream(), n, b, a, _lib.ptr(self.A_diagonal_blocks),
                                    _lib.ptr(T), 1 if a > 0 else 0, None, ctypes.byref(out))
        _lib.check(rc, "logdet")
        if np.isnan(out.value):
            raise ValueError("Logdet is NaN. Check the input matrix.")
        return float(out.value)

    def selected_inversion(self, sparsity: str = "bta") -> None:
        _check_sparsity(sparsity)
        n, b, a = self._dims(sparsity)
        D, L, Ab, T = self._ptrs(sparsity)
        _lib.check(_lib.load().bta_pobtasi(self.h.bind_stream(), n, b, a, D, L, Ab, T), "selected_inversion")

    def _structured_to_spmatrix(self, A, sparsity: str = "bta"):
        """Symmetric sparse matrix with the BTA values at ``A``'s lower-triangle
        pattern, symmetrised like the reference (``:476-538``)."""
        import torch

        _check_sparsity(sparsity)
        C, r, c = self._device_coo(sps.csc_matrix(A), lower_only=True)
        out = torch.empty(C.nnz, dtype=torch.float64, device=self.device)
        n, b, a = self._dims(sparsity)
        D, L, Ab, T = self._ptrs(sparsity)
        rc = _lib.load().bta_gather_coo(self.h.bind_stream(), n, b, a, _lib.ptr(r), _lib.ptr(c), int(C.nnz),
                                        1 if sparsity == "bt" else 0, D, L, Ab, T, _lib.ptr(out))
        _lib.check(rc, "gather")
        B = sps.coo_matrix((out.cpu().numpy(), (C.row, C.col)), shape=C.shape).tocsc()
        return B + sps.tril(B, k=-1).T

    def get_solver_memory(self) -> int:
        tot = self.A_diagonal_blocks.nbytes + self.A_lower_diagonal_blocks.nbytes
        if self.A_arrow_bottom_blocks is not None:
            tot += self.A_arrow_bottom_blocks.nbytes + self.A_arrow_tip_block.nbytes
        return int(tot + self.h.workspace_bytes())
