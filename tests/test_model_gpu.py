"""The device objective f(theta) and its gradients against the reference
(golden fixtures written by running DALIA) and the dense oracle adjoint."""
import numpy as np
import pytest

from golden_util import load, problem, rel
from oracle import model_ref

pytestmark = pytest.mark.gpu

GAUSS = ["gst_small", "gst_ragged", "gst_300x10"]


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
