"""The online autotuner: every candidate launch configuration it chooses from
gives the same results (the factorisation's CTAs per SM, queue order and
lookahead, in both the FP64 and the split Schur-update forms; the persistent
sweep's CTAs per SM and row segments), and a factorisation of a new shape
records a decision after trying them."""
import ctypes

import numpy as np
import pytest

from golden_util import rel
from oracle import bta_ref

pytestmark = pytest.mark.gpu


def _factor(count, n, b, a, seed, precision=None):
    import torch

    from dalia_b200 import _lib

    lib = _lib.load()
    h = _lib.handle()
    mats = [bta_ref.random_bta(n, b, a, np.random.default_rng(seed + k)) for k in range(count)]
    dev = [[torch.from_numpy(x.copy()).cuda() for x in m] for m in mats]
    arr = lambda vals, t=ctypes.c_int64: (t * count)(*vals)  # noqa: E731
    ptrs = [(ctypes.c_void_p * count)(*[d[j].data_ptr() for d in dev]) for j in range(4)]
    info = ctypes.c_int64(-1)
    if precision is None:
        rc = lib.bta_pobtaf_batched(h.bind_stream(), count, arr([n] * count), arr([b] * count), arr([a] * count),
                                    *ptrs, ctypes.byref(info))
    else:
        rc = lib.bta_pobtaf_batched_ex(h.bind_stream(), count, arr([n] * count), arr([b] * count),
                                       arr([a] * count), *ptrs, ctypes.byref(info), precision)
    assert rc == 0 and info.value == 0
    return mats, dev


# FP64 launches with previous-column terms: 2 CTAs-per-SM x 2 orders x 3
# lookaheads; split-form launches (Schur updates as 8-bit-slice GEMMs): 2 x 2
@pytest.mark.parametrize("persist", ["1", "0"])
@pytest.mark.parametrize("cand", range(12))
def test_every_panel_candidate_factors_exactly(cand, persist, monkeypatch):
    # the whole factorisation in one launch ("panel_all") and column by column ("panel")
    monkeypatch.setenv("DALIA_B200_TUNE_FORCE", f"panel={cand},panel_all={cand}")
    monkeypatch.setenv("DALIA_B200_PANEL_PERSIST", persist)
    mats, dev = _factor(3, 6, 200, 5, 100 + cand)
    for m, d in zip(mats, dev):
        ref = [x.copy() for x in m]
        bta_ref.pobtaf(*ref)
        for g, r in zip(d, ref):
            assert rel(g.cpu().numpy(), r) < 1e-10


@pytest.mark.parametrize("cand", range(4))
def test_every_split_panel_candidate_factors(cand, monkeypatch):
    from dalia_b200 import _lib

    monkeypatch.setenv("DALIA_B200_TUNE_FORCE", f"panel={cand}")
    mats, dev = _factor(3, 6, 200, 5, 200 + cand, precision=_lib.BTA_PREC_I8SLICE)
    for m, d in zip(mats, dev):
        ref = [x.copy() for x in m]
        bta_ref.pobtaf(*ref)
        for g, r in zip(d, ref):
            assert rel(g.cpu().numpy(), r) < 1e-10


@pytest.mark.parametrize("cand", range(3))
def test_every_sweep_candidate_solves_exactly(cand, monkeypatch):
    import torch

    from dalia_b200 import serinv_compat as sc

    monkeypatch.setenv("DALIA_B200_TUNE_FORCE", f"sweep={cand}")
    n, b, a = 5, 300, 4
    D, L, Ab, T = bta_ref.random_bta(n, b, a, np.random.default_rng(9))
    M = bta_ref.bta_to_dense(D, L, Ab, T)
    d = [torch.from_numpy(x.copy()).cuda() for x in (D, L, Ab, T)]
    sc.pobtaf(*d)
    rhs = np.random.default_rng(10).standard_normal(n * b + a)
    x = torch.from_numpy(rhs.copy()).cuda()
    sc.pobtas(*d, x, "N")
    sc.pobtas(*d, x, "C")
    assert rel(x.cpu().numpy(), np.linalg.solve(M, rhs)) < 1e-10


def test_tuner_decides_and_reports(monkeypatch):
    """Launched column by column, a batched factorisation with many block
    columns of one new shape lets the tuner try the panel candidates on its
    block columns and record a decision; as one launch per factorisation,
    the candidates are tried on successive factorisations of one shape
    (12 candidates, 2 trials each).  Every factor stays exact."""
    from dalia_b200 import _lib

    monkeypatch.delenv("DALIA_B200_TUNE_FORCE", raising=False)
    monkeypatch.delenv("DALIA_B200_TUNE", raising=False)
    monkeypatch.setenv("DALIA_B200_PANEL_PERSIST", "0")
    # 29 launches with a previous-column term: 12 candidates x 2 trials, then the decision
    mats, dev = _factor(2, 30, 131, 3, 300)
    for m, d in zip(mats, dev):
        ref = [x.copy() for x in m]
        bta_ref.pobtaf(*ref)
        for g, r in zip(d, ref):
            assert rel(g.cpu().numpy(), r) < 1e-10
    lines = _lib.tune_report()
    assert any(ln.startswith("panel|") and "best=" in ln for ln in lines), lines
    monkeypatch.setenv("DALIA_B200_PANEL_PERSIST", "1")
    for it in range(25):
        mats, dev = _factor(2, 4, 133, 3, 400 + it)
        for m, d in zip(mats, dev):
            ref = [x.copy() for x in m]
            bta_ref.pobtaf(*ref)
            for g, r in zip(d, ref):
                assert rel(g.cpu().numpy(), r) < 1e-10
    lines = _lib.tune_report()
    assert any(ln.startswith("panel_all|") and "best=" in ln for ln in lines), lines
