"""Host logic of the coregional model (no GPU): the per-sub-block Kronecker
coefficients rebuild the oracle's permuted joint prior, and the latent
permutation equals the oracle's restatement of the reference's."""
import numpy as np
import pytest
import scipy.sparse as sps

from golden_util import coreg_problem, load, rel
from oracle import coreg_ref


def _host_model(prob):
    from dalia_b200.coregional import CoregionalModel
    from dalia_b200.model import _tridiag

    m = object.__new__(CoregionalModel)
    m.nv, m.nt, m.ns = prob.nv, prob.nt, prob.ns
    m.sigma_st = np.asarray(prob.sigma_st, dtype=np.float64)
    m.m_diag = [_tridiag(x, prob.nt)[0] for x in (prob.m0, prob.m1, prob.m2)]
    m.m_sub = [_tridiag(x, prob.nt)[1] for x in (prob.m0, prob.m1, prob.m2)]
    return m


@pytest.mark.parametrize("name", ["gst_coreg3_small", "gst_coreg2_ragged"])
def test_coefficients_rebuild_the_joint_prior(name):
    g = load(name)
    prob = coreg_problem(g)
    m = _host_model(prob)
    th = g["theta"]
    nv, ns, nt = prob.nv, prob.ns, prob.nt
    b = nv * ns
    cf = m.coef_blocks(th).reshape(2 * nt - 1, nv, nv, 4)
    Ks = [sps.csr_matrix(K).toarray() for K in (prob.c0, prob.g1, prob.g2, prob.g3)]
    Q = np.zeros((nt * b, nt * b))
    for blk in range(2 * nt - 1):
        t, tc = (blk, blk) if blk < nt else (blk - nt + 1, blk - nt)
        B = np.zeros((b, b))
        for v in range(nv):
            for w in range(nv):
                B[v * ns:(v + 1) * ns, w * ns:(w + 1) * ns] = sum(cf[blk, v, w, k] * Ks[k] for k in range(4))
        Q[t * b:(t + 1) * b, tc * b:(tc + 1) * b] = B
        if blk >= nt:
            Q[tc * b:(tc + 1) * b, t * b:(t + 1) * b] = B.T
    orc = coreg_ref.CoregionalOracle(prob)
    assert rel(Q, orc.q_re(th, dense=True)) < 1e-14
    # complex step through the coefficients: derivative of sigma_0
    thc = th.astype(np.complex128)
    thc[3 * nv] += 1e-30j
    d = np.imag(m.coef_blocks(thc)) / 1e-30
    h = 1e-6
    tp, tm = th.copy(), th.copy()
    tp[3 * nv] += h
    tm[3 * nv] -= h
    assert rel(d, (m.coef_blocks(tp) - m.coef_blocks(tm)) / (2 * h)) < 1e-8


def test_latent_permutation_matches_oracle():
    from dalia_b200.coregional import latent_permutation

    for nt, ns, nv, nb in ((4, 40, 3, 1), (3, 70, 2, 2)):
        assert np.array_equal(latent_permutation(nt, ns, nv, nb), coreg_ref.perm_latent(nt, ns, nv, nb))
