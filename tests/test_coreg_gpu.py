"""Coregional model on the device against the reference (fixtures written
by running its CoregionalModel) and the dense oracle adjoint."""
import numpy as np
import pytest

from golden_util import coreg_problem, load, rel
from oracle import coreg_ref

pytestmark = pytest.mark.gpu

CASES = ["gst_coreg3_small", "gst_coreg2_ragged"]


@pytest.mark.parametrize("name", CASES)
def test_f_and_fd_gradient_match_reference(name):
    from dalia_b200.coregional import CoregionalModel

    g = load(name)
    m = CoregionalModel(coreg_problem(g))
    f = m.evaluate_f(g["theta"])
    assert abs(f - float(g["f_serinv"])) < 1e-10 * max(1.0, abs(float(g["f_serinv"])))
    assert rel(m.x.cpu().numpy(), g["x_serinv"]) < 1e-10
    f, grad = m.objective_fd(g["theta"])
    assert abs(f - float(g["f_serinv"])) < 1e-10 * max(1.0, abs(float(g["f_serinv"])))
    assert rel(grad, g["grad_serinv"]) < 1e-7


@pytest.mark.parametrize("name", CASES)
def test_adjoint_gradient(name):
    from dalia_b200.coregional import CoregionalModel

    g = load(name)
    prob = coreg_problem(g)
    m = CoregionalModel(prob)
    f, grad = m.objective_adjoint(g["theta"])
    assert abs(f - float(g["f_serinv"])) < 1e-10 * max(1.0, abs(float(g["f_serinv"])))
    ga = coreg_ref.dense_adjoint_gradient(coreg_ref.CoregionalOracle(prob), g["theta"])
    assert rel(grad, ga) < 1e-9
    assert rel(grad, g["grad_serinv"]) < 1e-5
    chk = m.last_check[0]
    assert chk["residual_c"] < 1e-11 and chk["residual_p"] < 1e-11


def test_batched_adjoint_matches_single_points():
    from dalia_b200.coregional import CoregionalModel

    g = load("gst_coreg3_small")
    m = CoregionalModel(coreg_problem(g))
    thetas = [g["theta"] + d for d in (0.0, 0.01, -0.02)]
    fs, gs = m.objective_adjoint_batched(thetas)
    for th, f, gr in zip(thetas, fs, gs):
        f1, g1 = m.objective_adjoint(th)
        assert abs(f - f1) < 1e-10 * max(1.0, abs(f1))
        assert rel(gr, g1) < 1e-10


def test_marginal_variances():
    from dalia_b200.coregional import CoregionalModel

    g = load("gst_coreg2_ragged")
    prob = coreg_problem(g)
    m = CoregionalModel(prob)
    orc = coreg_ref.CoregionalOracle(prob)
    S = np.linalg.inv(orc.q_cond(g["theta"]).toarray())
    mv = m.marginal_variances_latent(g["theta"]).cpu().numpy()
    assert rel(mv, np.diag(S)) < 1e-10
    Ad = orc.A.toarray()
    mo = m.marginal_variances_observations(g["theta"]).cpu().numpy()
    assert rel(mo, np.einsum("ij,jk,ik->i", Ad, S, Ad)) < 1e-10


@pytest.mark.parametrize("name", CASES)
def test_batched_fd_stencil_matches_sequential(name):
    from dalia_b200.coregional import CoregionalModel

    g = load(name)
    m = CoregionalModel(coreg_problem(g))
    f, grad = m.objective_fd_batched(g["theta"], max_points=8)
    assert abs(f - float(g["f_serinv"])) < 1e-10 * max(1.0, abs(float(g["f_serinv"])))
    assert rel(grad, g["grad_serinv"]) < 1e-7
    assert rel(m.x.cpu().numpy(), g["x_serinv"]) < 1e-10
