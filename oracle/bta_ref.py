"""CPU oracle: block-tridiagonal-arrowhead (BTA) Cholesky, solve and selected
inversion restated in NumPy/SciPy (LAPACK), FP64.

TEST INFRASTRUCTURE ONLY. This module is the checker for the CUDA library;
only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it.  The product path never calls it.

The reference (DALIA) delegates this arithmetic to the third-party package
Serinv (``serinv @ git+https://github.com/vincent-maillou/serinv``, unpinned,
``pyproject.toml:40``), which is absent here.  The functions below restate the
published block-Cholesky / Takahashi selected-inversion recurrences with the
call signatures DALIA uses at its call sites:

* ``pobtaf``  -- ``src/dalia/solvers/structured_solver.py:83-88``
* ``pobtf``   -- ``src/dalia/solvers/structured_solver.py:90-93``
* ``pobtas``  -- ``src/dalia/solvers/structured_solver.py:112-127`` (one sweep per call)
* ``pobts``   -- ``src/dalia/solvers/structured_solver.py:129-140``
* ``pobtasi`` -- ``src/dalia/solvers/structured_solver.py:176-181``
* ``pobtsi``  -- ``src/dalia/solvers/structured_solver.py:183-186``
* ``logdet``  -- ``src/dalia/solvers/structured_solver.py:151-166``

Storage (``structured_solver.py:37-60``): ``D[n,b,b]`` diagonal blocks,
``L[n-1,b,b]`` sub-diagonal blocks ``Q[(i+1)b:(i+2)b, ib:(i+1)b]``,
``Ab[n,a,b]`` arrow bottom ``Q[nb:, ib:(i+1)b]``, ``T[a,a]`` tip.  All
operations are in place.  After ``pobtaf`` the diagonal blocks hold the lower
Cholesky factors with zeros above the diagonal; after ``pobtasi`` every array
holds the corresponding block of ``Q^{-1}`` (diagonal blocks full symmetric).
"""

from __future__ import annotations

import numpy as np
import scipy.linalg as sla


def _chol(A: np.ndarray) -> np.ndarray:
    # numpy raises LinAlgError (a ValueError) on a non-SPD block
    return np.linalg.cholesky(A)


def _inv_lower(Lb: np.ndarray) -> np.ndarray:
    return sla.solve_triangular(Lb, np.eye(Lb.shape[0]), lower=True)


def pobtaf(D, L, Ab, T):
    """In-place BTA Cholesky: for i = 0..n-1,
    ``L_ii = chol(A_ii)``; ``L_{i+1,i} = A_{i+1,i} L_ii^-T``;
    ``A_{i+1,i+1} -= L_{i+1,i} L_{i+1,i}^T``; ``L_{a,i} = A_{a,i} L_ii^-T``;
    ``A_{a,i+1} -= L_{a,i} L_{i+1,i}^T``; ``A_aa -= L_{a,i} L_{a,i}^T``;
    finally ``L_aa = chol(A_aa)``."""
    n = D.shape[0]
    has_arrow = Ab is not None and T is not None and Ab.shape[1] > 0
    for i in range(n):
        D[i] = _chol(D[i])
        LinvT = _inv_lower(D[i]).T
        if i < n - 1:
            L[i] = L[i] @ LinvT
            D[i + 1] -= L[i] @ L[i].T
        if has_arrow:
            Ab[i] = Ab[i] @ LinvT
            if i < n - 1:
                Ab[i + 1] -= Ab[i] @ L[i].T
            T -= Ab[i] @ Ab[i].T
    if has_arrow:
        T[:] = _chol(T)


def pobtf(D, L):
    """In-place BT Cholesky (``pobtaf`` without arrowhead)."""
    pobtaf(D, L, None, None)


def pobtas(D, L, Ab, T, B, trans="N"):
    """One triangular sweep on ``B`` (length ``n*b + a``, or ``(n*b+a, k)``).

    ``trans="N"``: forward ``L y = B``:
    ``y_i = L_ii^-1 (B_i - L_{i,i-1} y_{i-1})``, ``y_a = L_aa^-1 (B_a - sum_i L_{a,i} y_i)``.
    ``trans="C"`` (or "T"): backward ``L^T x = B``:
    ``x_a = L_aa^-T B_a``, ``x_i = L_ii^-T (B_i - L_{i+1,i}^T x_{i+1} - L_{a,i}^T x_a)``.
    """
    n, b = D.shape[0], D.shape[1]
    has_arrow = Ab is not None and T is not None and Ab.shape[1] > 0
    a = Ab.shape[1] if has_arrow else 0
    vec = B.ndim == 1
    X = B.reshape(n * b + a, -1)
    blk = lambda i: slice(i * b, (i + 1) * b)
    if trans == "N":
        for i in range(n):
            if i > 0:
                X[blk(i)] -= L[i - 1] @ X[blk(i - 1)]
            X[blk(i)] = sla.solve_triangular(D[i], X[blk(i)], lower=True)
        if has_arrow:
            for i in range(n):
                X[n * b:] -= Ab[i] @ X[blk(i)]
            X[n * b:] = sla.solve_triangular(T, X[n * b:], lower=True)
    elif trans in ("C", "T"):
        if has_arrow:
            X[n * b:] = sla.solve_triangular(T, X[n * b:], lower=True, trans="T")
        for i in range(n - 1, -1, -1):
            if i < n - 1:
                X[blk(i)] -= L[i].T @ X[blk(i + 1)]
            if has_arrow:
                X[blk(i)] -= Ab[i].T @ X[n * b:]
            X[blk(i)] = sla.solve_triangular(D[i], X[blk(i)], lower=True, trans="T")
    else:
        raise ValueError(f"unknown trans {trans!r}")
    if vec:
        B[:] = X.reshape(-1)
    return B


def pobts(D, L, B, trans="N"):
    return pobtas(D, L, None, None, B, trans)


def pobtasi(D, L, Ab, T):
    """In-place selected inversion (Takahashi / Erisman-Tinney) of the factor:
    ``S_aa = L_aa^-T L_aa^-1``; for i = n-1..0 with ``G = L_{i+1,i} L_ii^-1``,
    ``G_a = L_{a,i} L_ii^-1``:
    ``S_{i+1,i} = -(S_{i+1,i+1} G + S_{a,i+1}^T G_a)``,
    ``S_{a,i} = -(S_{a,i+1} G + S_aa G_a)``,
    ``S_ii = L_ii^-T L_ii^-1 - G^T S_{i+1,i} - G_a^T S_{a,i}``."""
    n = D.shape[0]
    has_arrow = Ab is not None and T is not None and Ab.shape[1] > 0
    if has_arrow:
        Ti = _inv_lower(T)
        T[:] = Ti.T @ Ti
    for i in range(n - 1, -1, -1):
        Linv = _inv_lower(D[i])
        S = Linv.T @ Linv
        if i < n - 1:
            G = L[i] @ Linv
            if has_arrow:
                Ga = Ab[i] @ Linv
                S_lo = -(D[i + 1] @ G + Ab[i + 1].T @ Ga)
                S_ar = -(Ab[i + 1] @ G + T @ Ga)
            else:
                S_lo = -(D[i + 1] @ G)
            S -= G.T @ S_lo
            L[i] = S_lo
        elif has_arrow:
            Ga = Ab[i] @ Linv
            S_ar = -(T @ Ga)
        if has_arrow:
            S -= Ga.T @ S_ar
            Ab[i] = S_ar
        D[i] = 0.5 * (S + S.T)


def pobtsi(D, L):
    pobtasi(D, L, None, None)


def logdet(D, T=None, sparsity="bta"):
    """``2 (sum_i sum_k log L_ii[k,k] + sum_k log L_aa[k,k])``; the tip is
    dropped for ``"bt"`` (``structured_solver.py:151-166``)."""
    s = 0.0
    for i in range(D.shape[0]):
        s += np.sum(np.log(np.diagonal(D[i])))
    if sparsity == "bta" and T is not None and T.size:
        s += np.sum(np.log(np.diagonal(T)))
    if np.isnan(s):
        raise ValueError("Logdet is NaN. Check the input matrix.")
    return 2.0 * s


# ---------------------------------------------------------------------------
# dense <-> BTA helpers (test utilities)


def bta_to_dense(D, L, Ab, T, lower_only=False):
    n, b = D.shape[0], D.shape[1]
    a = 0 if Ab is None else Ab.shape[1]
    N = n * b + a
    M = np.zeros((N, N))
    for i in range(n):
        M[i * b:(i + 1) * b, i * b:(i + 1) * b] = D[i]
        if i < n - 1:
            M[(i + 1) * b:(i + 2) * b, i * b:(i + 1) * b] = L[i]
        if a:
            M[n * b:, i * b:(i + 1) * b] = Ab[i]
    if a:
        M[n * b:, n * b:] = T
    if lower_only:
        return np.tril(M)
    Ml = np.tril(M, -1)
    return np.tril(M) + Ml.T


def dense_to_bta(M, n, b, a):
    D = np.empty((n, b, b))
    L = np.empty((max(n - 1, 0), b, b))
    Ab = np.empty((n, a, b))
    T = np.empty((a, a))
    for i in range(n):
        D[i] = M[i * b:(i + 1) * b, i * b:(i + 1) * b]
        if i < n - 1:
            L[i] = M[(i + 1) * b:(i + 2) * b, i * b:(i + 1) * b]
        Ab[i] = M[n * b:, i * b:(i + 1) * b]
    T[:] = M[n * b:, n * b:]
    return D, L, Ab, T


def sparse_to_bta(Q, n, b, a):
    """Scatter a scipy sparse matrix into zeroed BTA blocks, like the CPU
    branch of ``SerinvSolver._spmatrix_to_structured``
    (``src/dalia/solvers/structured_solver.py:198-250``)."""
    import scipy.sparse as sps

    C = sps.coo_matrix(Q)
    D = np.zeros((n, b, b))
    L = np.zeros((max(n - 1, 0), b, b))
    Ab = np.zeros((n, a, b))
    T = np.zeros((a, a))
    r, c, v = C.row, C.col, C.data
    nb_ = n * b
    bi_r, bi_c = r // b, c // b
    m = (r < nb_) & (c < nb_) & (bi_r == bi_c)
    np.add.at(D, (bi_r[m], r[m] % b, c[m] % b), v[m])
    m = (r < nb_) & (c < nb_) & (bi_r == bi_c + 1)
    np.add.at(L, (bi_c[m], r[m] % b, c[m] % b), v[m])
    if a:
        m = (r >= nb_) & (c < nb_)
        np.add.at(Ab, (bi_c[m], r[m] - nb_, c[m] % b), v[m])
        m = (r >= nb_) & (c >= nb_)
        np.add.at(T, (r[m] - nb_, c[m] - nb_), v[m])
    return D, L, Ab, T


def random_bta(n, b, a, rng, diag_shift=None):
    """Random SPD BTA matrix (dense blocks), diagonally dominant."""
    D = rng.standard_normal((n, b, b)) * 0.1
    D = 0.5 * (D + D.transpose(0, 2, 1))
    L = rng.standard_normal((max(n - 1, 0), b, b)) * 0.1
    Ab = rng.standard_normal((n, a, b)) * 0.1
    T = rng.standard_normal((a, a)) * 0.1
    T = 0.5 * (T + T.T)
    shift = diag_shift if diag_shift is not None else 0.3 * (3 * b + a) ** 0.5 + 1.0
    for i in range(n):
        D[i] += shift * np.eye(b)
    T += (shift + 0.1 * n * b ** 0.5) * np.eye(a)
    return D, L, Ab, T
