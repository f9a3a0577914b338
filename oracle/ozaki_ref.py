"""CPU restatement of the 8-bit-slice GEMM's arithmetic (test infrastructure).

The library's reduced-precision block products (``BTA_PREC_I8SLICE``,
``dalia_b200/csrc/gemm_i8.cu``) follow the published Ozaki splitting; the
reference has no counterpart (its block products are FP64).  This module
restates that arithmetic step by step in NumPy so that the device result can
be checked bit for bit, not only against an FP64 product:

* one exponent e per row of op(A) (over all segments of a problem) and f per
  column of op(B): the frexp exponent of max |alpha x| (max < 2^e), or
  ``EXP_NONE`` for an all-zero row;
* U = trunc(|alpha x| 2^(49 - e)) < 2^49 cut into seven 7-bit digits
  d_p = (U >> 7 (6 - p)) & 127, signed like alpha x;
* per level d = p + q <= 6 the exact integer sums sum_k a_p b_q;
* hi = levels 0-3 and lo = levels 4-6 combined exactly (Horner, base 128),
  v = hi + lo 2^-21 (the only rounding), C = v 2^(e + f - 35), then
  C += beta C_old when beta != 0.

Only ``tests/`` may import it.
"""

from __future__ import annotations

import numpy as np

OZ_S = 7
EXP_NONE = -1100


def exponents(ops):
    """ops: list of (X rows x K, alpha) sharing rows; frexp exponent per row."""
    m = np.zeros(ops[0][0].shape[0])
    for X, alpha in ops:
        if X.shape[1]:
            m = np.maximum(m, abs(alpha) * np.max(np.abs(X), axis=1))
    e = np.frexp(m)[1].astype(np.int64)
    e[m == 0.0] = EXP_NONE
    return e


def digits(X, alpha, e):
    """Seven signed digit planes (int64) of alpha X with row exponents e."""
    sh = (7 * OZ_S - e).astype(np.int64)
    mag = np.abs(X * alpha)
    U = np.zeros(X.shape, dtype=np.int64)
    ok = e != EXP_NONE
    U[ok] = np.floor(np.ldexp(mag[ok], sh[ok, None].repeat(X.shape[1], axis=1).astype(np.int32))).astype(np.int64)
    neg = (X < 0.0) != (alpha < 0.0)
    planes = []
    for p in range(OZ_S):
        d = (U >> (7 * (OZ_S - 1 - p))) & 127
        planes.append(np.where(neg, -d, d))
    return planes


def gemm(segments, M, N, beta=0.0, C=None, lower=False, mirror=False):
    """C = beta C + sum_s alpha_s opA_s opB_s with the 8-bit-slice arithmetic.

    segments: list of (opA M x K, opB^T N x K, alpha).  Returns the new C
    (lower: only m >= n written; mirror: C[n][m] = C[m][n] for n < m)."""
    eA = exponents([(a, al) for a, _, al in segments])
    fB = exponents([(b, 1.0) for _, b, _ in segments])
    lev = [np.zeros((M, N), dtype=np.int64) for _ in range(OZ_S)]
    for a, b, al in segments:
        if a.shape[1] == 0:
            continue
        da, db = digits(a, al, eA), digits(b, 1.0, fB)
        for p in range(OZ_S):
            for q in range(OZ_S - p):
                # digit products <= 127^2 K: exact in float64 for K < 2^38
                lev[p + q] += np.rint(da[p].astype(np.float64) @ db[q].astype(np.float64).T).astype(np.int64)
    hi = ((lev[0] * 128 + lev[1]) * 128 + lev[2]) * 128 + lev[3]
    lo = (lev[4] * 128 + lev[5]) * 128 + lev[6]
    v = hi.astype(np.float64) + lo.astype(np.float64) * 2.0 ** -21
    x = np.ldexp(v, (eA[:, None] + fB[None, :] - 35).astype(np.int32))
    out = np.zeros((M, N)) if C is None else C.copy()
    if beta != 0.0:
        x = x + beta * out
    keep = np.tril(np.ones((M, N), dtype=bool)) if lower else np.ones((M, N), dtype=bool)
    out[keep] = x[keep]
    if mirror:
        il = np.tril_indices(M, -1)
        out[il[1], il[0]] = out[il]
    return out
