"""Element-wise check of the device assembly: the BTA blocks of Q_conditional
and Q_prior written by the assembly kernels against the sparse matrices the
reference itself built (``Model.construct_Q_prior`` / ``construct_Q_conditional``,
stored as COO in the golden fixtures by running DALIA)."""
import numpy as np
import pytest
import scipy.sparse as sps

from golden_util import coreg_problem, load, problem, rel
from oracle import bta_ref

pytestmark = pytest.mark.gpu

TOL = 1e-13


def _compare(dev, ref):
    dev = np.asarray(dev)
    assert rel(dev, ref) < TOL
    scale = max(float(np.max(np.abs(ref))), 1e-300)
    assert float(np.max(np.abs(dev - ref))) <= TOL * scale


def _check(m, g, Qc_ref, Qp_ref):
    n, b, a = m.nt, m.b, m.nb
    nst = n * b
    D, L, Ab, T = bta_ref.sparse_to_bta(Qc_ref.tocsc(), n, b, a)
    sl = m.slots[0]
    _compare(sl.Qc.D.cpu().numpy(), D)
    _compare(sl.Qc.L.cpu().numpy(), L)
    _compare(sl.Qc.Ab.cpu().numpy(), Ab)
    _compare(sl.Qc.T.cpu().numpy(), T)
    Dp, Lp, _, _ = bta_ref.sparse_to_bta(Qp_ref.tocsc()[:nst, :nst], n, b, 0)
    _compare(sl.Qp.D.cpu().numpy(), Dp)
    _compare(sl.Qp.L.cpu().numpy(), Lp)
    # the fixed-effect block of Q_prior is fe_prec I (the tip of Q_c carries it)
    np.testing.assert_allclose(Qp_ref.tocsc()[nst:, nst:].toarray(), m.fe_prec * np.eye(a), rtol=0, atol=0)


@pytest.mark.parametrize("name", ["gst_small", "gst_ragged", "gst_300x10", "pst_small", "pst_150x6"])
def test_univariate_assembly_matches_reference(name):
    """Against the reference's own matrices where the fixture stores them,
    else against the oracle's assembly (pinned to those matrices on the CPU
    to 1e-13)."""
    from dalia_b200.model import SpatioTemporalModel
    from oracle import model_ref

    g = load(name)
    prob = problem(g)
    m = SpatioTemporalModel(prob)
    th = np.asarray(g["theta"], dtype=np.float64)
    sl = m.slots[0]
    if m.gaussian:
        m._gauss_conditional(th, sl)
    else:
        # the fixture holds Q_conditional at eta = 0: D = e * exp(0)
        m.assemble_conditional(th, m.e, 1.0, sl)
    m.assemble_prior_bt(th, sl)
    N = m.N
    if "qc_data" in g:
        Qc = sps.coo_matrix((g["qc_data"], (g["qc_row"], g["qc_col"])), shape=(N, N))
        Qp = sps.coo_matrix((g["qp_data"], (g["qp_row"], g["qp_col"])), shape=(N, N))
    else:
        om = model_ref.OracleModel(prob)
        Qc = om.q_cond(th, np.zeros(len(prob.y)))
        Qp = om.q_prior(th)
    _check(m, g, Qc, Qp)


@pytest.mark.parametrize("name", ["gst_coreg3_small", "gst_coreg2_ragged"])
def test_coregional_assembly_matches_reference(name):
    """The reference's coregional matrices are stored in its permuted order
    (variates interleaved per time step, fixed effects last,
    ``coregional_model.py:750-853``), which is the device's BTA order."""
    from dalia_b200.coregional import CoregionalModel

    g = load(name)
    m = CoregionalModel(coreg_problem(g))
    th = np.asarray(g["theta"], dtype=np.float64)
    sl = m.slots[0]
    m._gauss_conditional(th, sl)
    m.assemble_prior_bt(th, sl)
    N = m.N
    Qc = sps.coo_matrix((g["qc_data"], (g["qc_row"], g["qc_col"])), shape=(N, N))
    Qp = sps.coo_matrix((g["qp_data"], (g["qp_row"], g["qp_col"])), shape=(N, N))
    _check(m, g, Qc, Qp)
