"""The coregional oracle against fixtures written by running the reference's
CoregionalModel (tests/golden/make_golden.py): assembly of Q_prior and
Q_conditional, f(theta), the FD gradient and the latent mean; and the dense
adjoint gradient against a fine FD of the oracle."""
import numpy as np
import pytest
import scipy.sparse as sps

from golden_util import coreg_problem, load, rel
from oracle import coreg_ref

CASES = ["gst_coreg3_small", "gst_coreg2_ragged"]


@pytest.mark.parametrize("name", CASES)
def test_assembly_matches_reference(name):
    g = load(name)
    orc = coreg_ref.CoregionalOracle(coreg_problem(g))
    th = g["theta"]
    N = orc.N
    Qp = sps.coo_matrix((g["qp_data"], (g["qp_row"], g["qp_col"])), shape=(N, N)).toarray()
    Qc = sps.coo_matrix((g["qc_data"], (g["qc_row"], g["qc_col"])), shape=(N, N)).toarray()
    assert rel(orc.q_prior(th).toarray(), Qp) < 1e-14
    assert rel(orc.q_cond(th).toarray(), Qc) < 1e-14


@pytest.mark.parametrize("name", CASES)
def test_objective_matches_reference_serinv_path(name):
    g = load(name)
    orc = coreg_ref.CoregionalOracle(coreg_problem(g))
    f, grad = orc.objective(g["theta"])
    assert abs(f - float(g["f_serinv"])) < 1e-10 * max(1.0, abs(float(g["f_serinv"])))
    assert rel(grad, g["grad_serinv"]) < 1e-9
    assert rel(orc.x, g["x_serinv"]) < 1e-10
    # Serinv path vs dense path: the prior log-determinant drops the nv*nb tip
    nv, nb = int(g["shape"][2]), int(g["shape"][3])
    assert abs((float(g["f_dense"]) - float(g["f_serinv"])) - (-0.5 * nv * nb * np.log(1e-3))) < 1e-8


@pytest.mark.parametrize("name", CASES)
def test_dense_adjoint_matches_fd(name):
    g = load(name)
    orc = coreg_ref.CoregionalOracle(coreg_problem(g))
    ga = coreg_ref.dense_adjoint_gradient(orc, g["theta"])
    assert rel(ga, g["grad_serinv"]) < 1e-5
    orc.eps = 1e-5
    _, gfd = orc.objective(g["theta"])
    assert rel(ga, gfd) < 1e-7
