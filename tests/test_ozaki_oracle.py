"""The CPU restatement of the 8-bit-slice GEMM (``oracle/ozaki_ref.py``):
its accuracy against an FP64 product, the design claim the device path rests
on (~1e-14 relative to max|a_m| max|b_n| K with seven 7-bit digits), and the
digit reconstruction bound."""
import numpy as np
import pytest

from oracle import ozaki_ref


@pytest.mark.parametrize("M,N,K,decay", [(40, 30, 50, 0.0), (64, 64, 300, 0.0), (50, 70, 200, 8.0)])
def test_restatement_accuracy_against_fp64(M, N, K, decay):
    rng = np.random.default_rng(M + N + K)
    A = rng.standard_normal((M, K)) * np.exp(-decay * rng.random((M, K)))
    B = rng.standard_normal((N, K)) * np.exp(-decay * rng.random((N, K)))
    got = ozaki_ref.gemm([(A, B, -1.5)], M, N)
    ref = -1.5 * (A @ B.T)
    # one scale per row / column: the truncation is relative to the row and
    # column maxima (small entries of a row with a wide range keep fewer bits)
    bound = 1.5 * np.outer(np.max(np.abs(A), axis=1), np.max(np.abs(B), axis=1)) * K
    assert np.max(np.abs(got - ref) / bound) < 1e-14
    if decay == 0.0:
        assert np.max(np.abs(got - ref) / (1.5 * (np.abs(A) @ np.abs(B).T))) < 1e-13


def test_digits_reconstruct_within_truncation():
    rng = np.random.default_rng(3)
    X = rng.standard_normal((20, 33)) * 10.0 ** rng.integers(-6, 6, size=(20, 1))
    X[3] = 0.0
    e = ozaki_ref.exponents([(X, 0.5)])
    planes = ozaki_ref.digits(X, 0.5, e)
    assert all(np.all(np.abs(p) <= 127) for p in planes)
    rec = sum(p.astype(np.float64) * 2.0 ** (-7 * (i + 1)) for i, p in enumerate(planes))
    rec = np.ldexp(rec, np.where(e == ozaki_ref.EXP_NONE, 0, e)[:, None].repeat(33, axis=1).astype(np.int32))
    rowmax = np.max(np.abs(0.5 * X), axis=1, keepdims=True)
    ok = rowmax[:, 0] > 0
    # truncation below 2^-49 of the row's scale 2^e < 2 rowmax
    assert np.all(np.abs(rec[ok] - 0.5 * X[ok]) <= 2.0 ** -48 * rowmax[ok])
    assert np.all(rec[3] == 0.0)


def test_lower_mirror_and_beta():
    rng = np.random.default_rng(5)
    A = rng.standard_normal((30, 20))
    C = rng.standard_normal((30, 30))
    got = ozaki_ref.gemm([(A, A, 1.0)], 30, 30, beta=0.5, C=C, lower=True, mirror=True)
    ref = 0.5 * C + A @ A.T
    full = np.where(np.tril(np.ones((30, 30), bool)), ref, ref.T)
    assert np.max(np.abs(got - full)) < 1e-12 * np.max(np.abs(full))
