"""The device objective f(theta) and its gradients against the reference
(golden fixtures written by running DALIA) and the dense oracle adjoint."""
import numpy as np
import pytest

from golden_util import load, problem, rel
from oracle import model_ref

pytestmark = pytest.mark.gpu

GAUSS = ["gst_small", "gst_ragged", "gst_300x10"]
POIS = ["pst_small", "pst_150x6"]


@pytest.mark.parametrize("name", GAUSS)
def test_f_matches_reference_serinv_path(name):
    from dalia_b200.model import SpatioTemporalModel

    g = load(name)
    m = SpatioTemporalModel(problem(g))
    f = m.evaluate_f(g["theta"])
    assert abs(f - float(g["f_serinv"])) < 1e-10 * abs(float(g["f_serinv"]))
    # the latent mean (model.x in the reference)
    assert rel(m.x.cpu().numpy(), g["x_serinv"]) < 1e-10


@pytest.mark.parametrize("name", GAUSS)
def test_fd_gradient_matches_reference(name):
    from dalia_b200.model import SpatioTemporalModel

    g = load(name)
    m = SpatioTemporalModel(problem(g))
    f, grad = m.objective_fd(g["theta"])
    assert abs(f - float(g["f_serinv"])) < 1e-10 * abs(float(g["f_serinv"]))
    assert rel(grad, g["grad_serinv"]) < 1e-7


@pytest.mark.parametrize("name", GAUSS)
def test_adjoint_gradient(name):
    from dalia_b200.model import SpatioTemporalModel

    g = load(name)
    prob = problem(g)
    m = SpatioTemporalModel(prob)
    f, grad = m.objective_adjoint(g["theta"])
    assert abs(f - float(g["f_serinv"])) < 1e-10 * abs(float(g["f_serinv"]))
    # FD truncation error of the reference gradient (eps = 1e-3) bounds the gap
    assert rel(grad, g["grad_serinv"]) < 1e-5
    if prob.ns * prob.nt <= 400:
        ga = model_ref.dense_adjoint_gradient(model_ref.OracleModel(prob), g["theta"])
        assert rel(grad, ga) < 1e-9


def test_batched_adjoint_matches_single_points():
    from dalia_b200.model import SpatioTemporalModel

    g = load("gst_ragged")
    m = SpatioTemporalModel(problem(g))
    thetas = [g["theta"] + d for d in (0.0, 0.01, -0.02)]
    fs, gs = m.objective_adjoint_batched(thetas)
    for th, f, gr in zip(thetas, fs, gs):
        f1, g1 = m.objective_adjoint(th)
        assert abs(f - f1) < 1e-10 * abs(f1)
        assert rel(gr, g1) < 1e-10


@pytest.mark.parametrize("name", POIS)
def test_poisson_fd_objective_matches_reference(name):
    """Newton inner iteration on the device, the reference's FD stencil with
    warm starts carried from point to point (golden: DALIA's Serinv path)."""
    from dalia_b200.model import SpatioTemporalModel

    g = load(name)
    m = SpatioTemporalModel(problem(g))
    f, grad = m.objective_fd(g["theta"])
    assert abs(f - float(g["f_serinv"])) < 1e-10 * abs(float(g["f_serinv"]))
    assert rel(grad, g["grad_serinv"]) < 1e-7
    assert rel(m.x.cpu().numpy(), g["x_serinv"]) < 1e-9


@pytest.mark.parametrize("name", POIS)
def test_poisson_adjoint_gradient(name):
    from dalia_b200.model import SpatioTemporalModel

    g = load(name)
    prob = problem(g)
    m = SpatioTemporalModel(prob)
    f, grad = m.objective_adjoint(g["theta"])
    om = model_ref.OracleModel(prob)
    f_ref = model_ref.OracleModel(prob).evaluate_f(g["theta"])
    ga = model_ref.dense_adjoint_gradient_poisson(om, g["theta"])
    assert abs(f - f_ref) < 1e-10 * abs(f_ref)
    assert rel(grad, ga) < 1e-8
    # the reference's FD gradient carries its Newton-tolerance noise
    assert rel(grad, g["grad_serinv"]) < 1e-2


def test_poisson_batched_adjoint_matches_single_points():
    from dalia_b200.model import SpatioTemporalModel

    g = load("pst_150x6")
    prob = problem(g)
    m = SpatioTemporalModel(prob)
    m.objective_adjoint(g["theta"])
    x0 = m.x.clone()
    thetas = [g["theta"] + d for d in (0.0, 0.02, -0.03)]
    fs, gs = m.objective_adjoint_batched(thetas)
    m1 = SpatioTemporalModel(prob)
    for th, f, gr in zip(thetas, fs, gs):
        m1.x.copy_(x0)
        f1, g1 = m1.objective_adjoint(th)
        assert abs(f - f1) < 1e-10 * abs(f1)
        assert rel(gr, g1) < 1e-9


@pytest.mark.parametrize("name", ["gst_small", "pst_150x6"])
def test_marginal_variances(name):
    from dalia_b200.model import SpatioTemporalModel

    g = load(name)
    prob = problem(g)
    m = SpatioTemporalModel(prob)
    om = model_ref.OracleModel(prob)
    th = g["theta"]
    x = g["x_serinv"]
    Qc = om.q_cond(th, om.A @ x).toarray()
    S = np.linalg.inv(Qc)
    Ad = om.A.toarray()
    mv = m.marginal_variances_latent(th, x).cpu().numpy()
    assert rel(mv, np.diag(S)) < 1e-10
    if "marg_var_serinv" in g:
        assert rel(mv, g["marg_var_serinv"]) < 1e-10
    mo = m.marginal_variances_observations(th, x).cpu().numpy()
    assert rel(mo, np.einsum("ij,jk,ik->i", Ad, S, Ad)) < 1e-10


def test_batched_fd_stencil_matches_reference():
    from dalia_b200.model import SpatioTemporalModel

    g = load("gst_300x10")
    m = SpatioTemporalModel(problem(g))
    f, grad = m.objective_fd_batched(g["theta"])
    assert abs(f - float(g["f_serinv"])) < 1e-10 * abs(float(g["f_serinv"]))
    assert rel(grad, g["grad_serinv"]) < 1e-7
    assert rel(m.x.cpu().numpy(), g["x_serinv"]) < 1e-10
