"""FP32-class (split TF32 x3, tcgen05 tensor cores) block products: the
grouped GEMM through the C ABI against NumPy, the selected inversion against
the FP64 oracle, and the adjoint gradient's accuracy check with its FP64
fallback.

Measured accuracy: the tensor cores accumulate in FP32 with truncating
alignment, so the error grows with K (~1e-6 relative at K ~ 300 on random
data, ~1e-5 for a selected inverse); the GEMM is held to 5e-6 and the
selected inverse to 3e-5 (norm-wise).  That is not enough for the adjoint
gradient's 1e-6 bar, so the default tolerance of the <S, Q> = N check
sends TF32x3 points back to FP64, whose results must then be reproduced
exactly.

The 8-bit-slice arithmetic (BTA_PREC_I8SLICE) accumulates exactly; its error
is the digit truncation, ~1e-9 relative per product (2e-8 after the selected
inversion's recurrence), so it is held to 1e-8 on the GEMM, 1e-7 on the
selected inverse and to the gradient bar of 1e-6."""
import ctypes

import numpy as np
import pytest

from golden_util import load, problem, rel
from oracle import bta_ref

pytestmark = pytest.mark.gpu

GEMM_CASES = [
    # M, N, K, a_trans, b_kn, lower_only, mirror, alpha, beta
    (128, 128, 32, 0, 0, 0, 0, 1.0, 0.0),
    (200, 130, 70, 0, 0, 0, 0, -1.0, 1.0),
    (257, 300, 129, 1, 0, 0, 0, 1.0, 0.0),
    (300, 257, 200, 0, 1, 0, 0, 1.0, 1.0),
    (190, 260, 333, 1, 1, 0, 0, -1.0, 0.0),
    (6, 300, 301, 0, 1, 0, 0, 1.0, 0.0),
    (300, 6, 300, 1, 0, 0, 0, 1.0, 0.0),
    (310, 310, 150, 1, 1, 1, 1, 1.0, 0.0),
    (200, 200, 90, 0, 1, 1, 1, -1.0, 0.5),
    (384, 384, 512, 0, 0, 1, 0, -1.0, 1.0),
    (100, 100, 0, 0, 0, 0, 0, 1.0, 0.5),
]


def _gemm(lib, h, prec, M, N, K, at, bkn, lower, mirror, alpha, beta, seed):
    import torch

    rng = np.random.default_rng(seed)
    A = rng.standard_normal((K, M) if at else (M, K))
    B = rng.standard_normal((K, N) if bkn else (N, K))
    C = rng.standard_normal((M, N))
    opA = A.T if at else A
    opB = B if bkn else B.T
    ref = beta * C + alpha * (opA @ opB)
    dA, dB, dC = (torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (A, B, C))
    from dalia_b200 import _lib

    rc = lib.bta_gemm(h.bind_stream(), prec, M, N, K, alpha, _lib.ptr(dA), A.shape[1], at, _lib.ptr(dB),
                      B.shape[1], bkn, beta, _lib.ptr(dC), N, lower, mirror)
    _lib.check(rc, "gemm")
    st = ctypes.c_int64(0)
    _lib.check(lib.bta_get_status(h.bind_stream(), ctypes.byref(st)), "status")
    got = dC.cpu().numpy()
    if lower:
        keep = np.tril(np.ones((M, N), dtype=bool))
        if mirror:
            keep = keep | keep.T
            ref = np.where(np.tril(np.ones((M, N), dtype=bool)), ref, ref.T)
        exp = np.where(keep, ref, C)
    else:
        exp = ref
    return got, exp


@pytest.mark.parametrize("case", GEMM_CASES)
def test_gemm_tf32x3_and_fp64_match_numpy(case):
    from dalia_b200 import _lib

    lib = _lib.load()
    h = _lib.handle()
    M, N, K, at, bkn, lower, mirror, alpha, beta = case
    got, exp = _gemm(lib, h, _lib.BTA_PREC_FP64, *case, seed=M + N + K)
    assert rel(got, exp) < 1e-13
    got, exp = _gemm(lib, h, _lib.BTA_PREC_TF32X3, *case, seed=M + N + K)
    assert rel(got, exp) < 5e-6


@pytest.mark.parametrize("n,b,a", [(3, 200, 6), (4, 129, 0), (2, 300, 70)])
def test_selinv_tf32x3_matches_oracle(n, b, a):
    import torch

    from dalia_b200 import _lib

    lib = _lib.load()
    h = _lib.handle()
    rng = np.random.default_rng(7 * n + b + a)
    D, L, Ab, T = bta_ref.random_bta(n, b, a, rng)
    ref = [x.copy() for x in (D, L, Ab, T)]
    bta_ref.pobtaf(*ref)
    bta_ref.pobtasi(*ref)
    d = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (D, L, Ab, T)]
    arr = lambda t: (ctypes.c_void_p * 1)(t.data_ptr() if t.numel() else None)
    i64 = lambda v: (ctypes.c_int64 * 1)(v)
    args = (h.bind_stream(), 1, i64(n), i64(b), i64(a), arr(d[0]), arr(d[1]), arr(d[2]), arr(d[3]))
    _lib.check(lib.bta_pobtaf_batched(*args, None), "pobtaf")
    _lib.check(lib.bta_pobtasi_batched_ex(*args, _lib.BTA_PREC_TF32X3), "pobtasi")
    st = ctypes.c_int64(0)
    _lib.check(lib.bta_get_status(h.bind_stream(), ctypes.byref(st)), "status")
    got = [t.cpu().numpy() for t in d]
    assert rel(got[0], ref[0]) < 3e-5
    if n > 1:
        assert rel(got[1], ref[1]) < 3e-5
    if a:
        assert rel(got[2], ref[2]) < 3e-5 and rel(got[3], ref[3]) < 3e-5


@pytest.mark.parametrize("name", ["gst_300x10", "pst_150x6"])
def test_tf32x3_adjoint_check_and_fallback(name):
    from dalia_b200.model import SpatioTemporalModel

    g = load(name)
    prob = problem(g)
    th = g["theta"]
    m64 = SpatioTemporalModel(prob)
    f64, g64 = m64.objective_adjoint(th)
    chk64 = m64.last_check[0]
    assert chk64["residual_c"] < 1e-11 and chk64["residual_p"] < 1e-11
    # no fallback: the check reports the reduced precision
    mm = SpatioTemporalModel(prob, selinv_precision="tf32x3", mixed_tolerance=1.0)
    fm, gm = mm.objective_adjoint(th)
    chk = mm.last_check[0]
    assert chk["precision"] == "tf32x3" and not chk["fallback"]
    assert abs(fm - f64) < 1e-12 * abs(f64)
    assert rel(gm, g64) < 1e-2
    assert max(chk["residual_c"], chk["residual_p"]) > 100 * max(chk64["residual_c"], chk64["residual_p"])
    # default tolerance: the point is recomputed in FP64
    md = SpatioTemporalModel(prob, selinv_precision="tf32x3")
    fd, gd = md.objective_adjoint(th)
    assert md.last_check[0]["fallback"] and md.last_check[0]["precision"] == "tf32x3"
    assert abs(fd - f64) < 1e-12 * abs(f64) and rel(gd, g64) < 1e-10


def test_mixed_fallback_recomputes_in_fp64():
    from dalia_b200.model import SpatioTemporalModel

    g = load("gst_ragged")
    prob = problem(g)
    th = g["theta"]
    f64, g64 = SpatioTemporalModel(prob).objective_adjoint(th)
    mm = SpatioTemporalModel(prob, selinv_precision="tf32x3", mixed_tolerance=0.0)
    fm, gm = mm.objective_adjoint(th)
    assert mm.last_check[0]["fallback"]
    assert abs(fm - f64) < 1e-12 * abs(f64)
    assert rel(gm, g64) < 1e-10


def test_failed_check_runs_the_next_evaluations_in_fp64():
    """After a fallback at the model's own precision, the next mixed_retry
    evaluations at that precision run in FP64 directly (marked demoted), then
    the reduced precision is tried again; an explicit precision is honoured."""
    from dalia_b200.model import SpatioTemporalModel

    g = load("gst_ragged")
    prob = problem(g)
    th = g["theta"]
    f64, g64 = SpatioTemporalModel(prob).objective_adjoint(th)
    mm = SpatioTemporalModel(prob, selinv_precision="i8slice", mixed_tolerance=0.0, mixed_retry=2)
    seen = []
    for _ in range(4):
        fm, gm = mm.objective_adjoint(th)
        c = mm.last_check[0]
        seen.append((c["precision"], c["fallback"], c.get("demoted", False)))
        assert abs(fm - f64) < 1e-12 * abs(f64)
        assert rel(gm, g64) < 1e-10
    assert seen == [("i8slice", True, False), ("fp64", False, True), ("fp64", False, True),
                    ("i8slice", True, False)]
    mm.objective_adjoint_batched([th], precision="i8slice")  # explicit: tried although demoted
    assert mm.last_check[0]["precision"] == "i8slice" and mm.last_check[0]["fallback"]
    mm.mixed_retry = 0
    mm.objective_adjoint(th)
    assert mm.last_check[0]["precision"] == "fp64"  # the two evaluations left from the fallback above
    mm.objective_adjoint(th)
    mm.objective_adjoint(th)
    assert mm.last_check[0]["precision"] == "i8slice"


@pytest.mark.parametrize("case", GEMM_CASES)
def test_gemm_i8slice_matches_numpy(case):
    from dalia_b200 import _lib

    lib = _lib.load()
    h = _lib.handle()
    M, N, K, at, bkn, lower, mirror, alpha, beta = case
    for rep in range(2):
        got, exp = _gemm(lib, h, _lib.BTA_PREC_I8SLICE, *case, seed=M + N + K + rep)
        assert rel(got, exp) < 1e-8


@pytest.mark.parametrize("n,b,a", [(3, 200, 6), (4, 129, 0), (2, 300, 70)])
def test_selinv_i8slice_matches_oracle(n, b, a):
    import torch

    from dalia_b200 import _lib

    lib = _lib.load()
    h = _lib.handle()
    rng = np.random.default_rng(7 * n + b + a)
    D, L, Ab, T = bta_ref.random_bta(n, b, a, rng)
    ref = [x.copy() for x in (D, L, Ab, T)]
    bta_ref.pobtaf(*ref)
    bta_ref.pobtasi(*ref)
    d = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (D, L, Ab, T)]
    arr = lambda t: (ctypes.c_void_p * 1)(t.data_ptr() if t.numel() else None)
    i64 = lambda v: (ctypes.c_int64 * 1)(v)
    args = (h.bind_stream(), 1, i64(n), i64(b), i64(a), arr(d[0]), arr(d[1]), arr(d[2]), arr(d[3]))
    _lib.check(lib.bta_pobtaf_batched(*args, None), "pobtaf")
    _lib.check(lib.bta_pobtasi_batched_ex(*args, _lib.BTA_PREC_I8SLICE), "pobtasi")
    st = ctypes.c_int64(0)
    _lib.check(lib.bta_get_status(h.bind_stream(), ctypes.byref(st)), "status")
    got = [t.cpu().numpy() for t in d]
    assert rel(got[0], ref[0]) < 1e-7
    if n > 1:
        assert rel(got[1], ref[1]) < 1e-7
    if a:
        assert rel(got[2], ref[2]) < 1e-7 and rel(got[3], ref[3]) < 1e-7


@pytest.mark.parametrize("name", ["gst_300x10", "pst_150x6"])
def test_i8slice_adjoint_meets_the_gradient_bar(name):
    from dalia_b200.model import SpatioTemporalModel

    g = load(name)
    prob = problem(g)
    th = g["theta"]
    f64, g64 = SpatioTemporalModel(prob).objective_adjoint(th)
    m = SpatioTemporalModel(prob, selinv_precision="i8slice")
    f, gr = m.objective_adjoint(th)
    chk = m.last_check[0]
    assert chk["precision"] == "i8slice" and not chk["fallback"]
    assert abs(f - f64) < 1e-12 * abs(f64)
    assert rel(gr, g64) < 1e-6


def test_i8slice_coregional_adjoint():
    from golden_util import coreg_problem

    from dalia_b200.coregional import CoregionalModel

    g = load("gst_coreg3_small")
    prob = coreg_problem(g)
    f64, g64 = CoregionalModel(prob).objective_adjoint(g["theta"])
    m = CoregionalModel(prob, selinv_precision="i8slice")
    f, gr = m.objective_adjoint(g["theta"])
    assert not m.last_check[0]["fallback"]
    assert abs(f - f64) < 1e-12 * max(1.0, abs(f64)) and rel(gr, g64) < 1e-6


@pytest.mark.parametrize("tile", [0, 1])
@pytest.mark.parametrize("case", GEMM_CASES)
def test_gemm_i8slice_bit_exact_against_restatement(case, tile, monkeypatch):
    """The device's 8-bit-slice product equals the step-by-step CPU restatement
    of its arithmetic (oracle/ozaki_ref.py) bit for bit: digits and level sums
    are integers, the level combination is exact, and the one rounding
    (hi + lo 2^-21) and the power-of-two scalings are the same.  Both output
    tile widths the autotuner chooses from (64; 32 with two accumulator sets)."""
    import torch

    from dalia_b200 import _lib
    from oracle import ozaki_ref

    monkeypatch.setenv("DALIA_B200_TUNE_FORCE", f"gemm_i8={tile}")

    lib = _lib.load()
    h = _lib.handle()
    M, N, K, at, bkn, lower, mirror, alpha, beta = case
    rng = np.random.default_rng(M + 7 * N + K)
    A = rng.standard_normal((K, M) if at else (M, K)) * np.exp(-4.0 * rng.random((K, M) if at else (M, K)))
    B = rng.standard_normal((K, N) if bkn else (N, K))
    C = rng.standard_normal((M, N))
    exp = ozaki_ref.gemm([(A.T if at else A, B.T if bkn else B, alpha)], M, N, beta, C, bool(lower), bool(mirror))
    dA, dB, dC = (torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (A, B, C))
    for _ in range(2):  # twice: the shared workspace and images carry nothing over
        dC.copy_(torch.from_numpy(C))
        _lib.check(lib.bta_gemm(h.bind_stream(), _lib.BTA_PREC_I8SLICE, M, N, K, alpha, _lib.ptr(dA), A.shape[1],
                                at, _lib.ptr(dB), B.shape[1], bkn, beta, _lib.ptr(dC), N, lower, mirror), "gemm")
        st = ctypes.c_int64(0)
        _lib.check(lib.bta_get_status(h.bind_stream(), ctypes.byref(st)), "status")
        got = dC.cpu().numpy()
        assert np.array_equal(got, exp), f"max diff {np.max(np.abs(got - exp))}"


@pytest.mark.parametrize("n,b,a", [(4, 200, 6), (3, 300, 70), (5, 129, 0)])
def test_factor_with_i8slice_schur_updates(n, b, a):
    """bta_pobtaf_batched_ex with the previous-column Schur updates in 8-bit
    slices: the factor, and the log-determinant from it, against the FP64
    oracle (the updates are exact to ~1e-14 of sum |L||L|)."""
    import torch

    from dalia_b200 import _lib

    lib = _lib.load()
    h = _lib.handle()
    D, L, Ab, T = bta_ref.random_bta(n, b, a, np.random.default_rng(n + b + a))
    ref = [x.copy() for x in (D, L, Ab, T)]
    bta_ref.pobtaf(*ref)
    d = [torch.from_numpy(x.copy()).cuda() for x in (D, L, Ab, T)]
    one = lambda v: (ctypes.c_int64 * 1)(v)  # noqa: E731
    ptr = lambda t: (ctypes.c_void_p * 1)(t.data_ptr() if t.numel() else None)  # noqa: E731
    info = ctypes.c_int64(-1)
    rc = lib.bta_pobtaf_batched_ex(h.bind_stream(), 1, one(n), one(b), one(a), *[ptr(t) for t in d],
                                   ctypes.byref(info), _lib.BTA_PREC_I8SLICE)
    assert rc == 0 and info.value == 0
    for g, r in zip(d, ref):
        if r.size:
            assert rel(g.cpu().numpy(), r) < 1e-11
    ld = bta_ref.logdet(ref[0], ref[3] if a else None, "bta" if a else "bt")
    ldg = bta_ref.logdet(d[0].cpu().numpy(), d[3].cpu().numpy() if a else None, "bta" if a else "bt")
    assert abs(ldg - ld) <= 1e-12 * abs(ld)


@pytest.mark.parametrize("name", ["gst_300x10", "gst_ragged"])
def test_adjoint_with_i8slice_factor_updates(name):
    """Both the factorisations' Schur updates and the selected inversion in
    8-bit slices: f (hence the log-determinants) within 1e-10 of the FP64
    path, the gradient within 1e-6."""
    from dalia_b200.model import SpatioTemporalModel

    g = load(name)
    m = SpatioTemporalModel(problem(g), selinv_precision="i8slice", factor_precision="i8slice")
    f64, g64 = m.objective_adjoint_batched([g["theta"]], precision="fp64")
    fm, gm = m.objective_adjoint_batched([g["theta"]])
    assert abs(fm[0] - f64[0]) <= 1e-10 * abs(f64[0])
    assert rel(gm[0], g64[0]) < 1e-6
    assert not m.last_check[0]["fallback"]


@pytest.mark.parametrize("M,K", [(300, 257), (1500, 1500)])
def test_gemm_i8slice_syrk_bit_exact(M, K):
    """C -= A A^T (lower, beta = 1) with the same array as both operands, the
    factorisation's Schur update: the negation moves to the epilogue and A's
    digits are cut once for both sides; the result equals the restatement bit
    for bit."""
    import torch

    from dalia_b200 import _lib
    from oracle import ozaki_ref

    lib = _lib.load()
    h = _lib.handle()
    rng = np.random.default_rng(M + K)
    A = rng.standard_normal((M, K)) * np.exp(-3.0 * rng.random((M, K)))
    C = rng.standard_normal((M, M))
    exp = ozaki_ref.gemm([(A, A, -1.0)], M, M, 1.0, C, True, False)
    dA, dC = (torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (A, C))
    _lib.check(lib.bta_gemm(h.bind_stream(), _lib.BTA_PREC_I8SLICE, M, M, K, -1.0, _lib.ptr(dA), K, 0,
                            _lib.ptr(dA), K, 0, 1.0, _lib.ptr(dC), M, 1, 0), "gemm")
    st = ctypes.c_int64(0)
    _lib.check(lib.bta_get_status(h.bind_stream(), ctypes.byref(st)), "status")
    got = dC.cpu().numpy()
    assert np.array_equal(got, exp), f"max diff {np.max(np.abs(got - exp))}"
