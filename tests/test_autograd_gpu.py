"""The objective as a torch.autograd function: forward = f(theta) (assembly,
factorisations, log-determinants, latent mean), backward = the adjoint
gradient (selected inversions and contraction kernels).  Checked against the
model's fused adjoint evaluation, the reference's FD gradient (golden
fixtures written by running DALIA) and torch's own finite differences of f."""
import numpy as np
import pytest

from golden_util import coreg_problem, load, problem, rel

pytestmark = pytest.mark.gpu


def _grad(model, theta, **kw):
    import torch

    from dalia_b200.autograd import objective

    th = torch.tensor(np.asarray(theta), dtype=torch.float64, requires_grad=True)
    f = objective(model, th, **kw)
    (g,) = torch.autograd.grad(f, th)
    return float(f.detach()), g.numpy()


@pytest.mark.parametrize("name", ["gst_small", "gst_300x10", "pst_small"])
def test_autograd_matches_adjoint_and_reference_fd(name):
    from dalia_b200.model import SpatioTemporalModel

    from oracle import model_ref

    gld = load(name)
    prob = problem(gld)
    m = SpatioTemporalModel(prob)
    f, g = _grad(m, gld["theta"])
    if not m.gaussian:
        m.slots[0].x.zero_()  # the Newton iteration starts where the autograd forward started
    f1, g1 = m.objective_adjoint(gld["theta"])
    assert abs(f - f1) <= 1e-12 * abs(f1)
    assert rel(g, g1) < 1e-12
    if m.gaussian:
        # the reference's central differences (eps = 1e-3) carry truncation error
        assert abs(f - float(gld["f_serinv"])) < 1e-10 * abs(float(gld["f_serinv"]))
        assert rel(g, gld["grad_serinv"]) < 1e-5
    else:
        # f from x = 0 as the oracle evaluates it; the reference's FD gradient
        # carries the noise of its warm-started Newton iterations
        f_ref = model_ref.OracleModel(prob).evaluate_f(gld["theta"])
        assert abs(f - f_ref) < 1e-10 * abs(f_ref)
        assert rel(g, gld["grad_serinv"]) < 1e-2


def test_autograd_coregional():
    from dalia_b200.coregional import CoregionalModel

    gld = load("gst_coreg3_small")
    m = CoregionalModel(coreg_problem(gld))
    f, g = _grad(m, gld["theta"])
    f1, g1 = m.objective_adjoint(gld["theta"])
    assert abs(f - f1) <= 1e-12 * abs(f1)
    assert rel(g, g1) < 1e-12
    assert rel(g, gld["grad_serinv"]) < 1e-5


def test_autograd_batched_points_with_weights():
    """theta of shape (K, d): f of shape (K,), and the backward of a weighted
    sum gives each point's gradient times its weight."""
    import torch

    from dalia_b200.autograd import objective
    from dalia_b200.model import SpatioTemporalModel

    gld = load("gst_ragged")
    m = SpatioTemporalModel(problem(gld))
    pts = np.stack([gld["theta"] + d for d in (0.0, 0.01, -0.02)])
    th = torch.tensor(pts, dtype=torch.float64, requires_grad=True)
    f = objective(m, th)
    assert f.shape == (3,)
    w = torch.tensor([1.0, -2.0, 0.5], dtype=torch.float64, device=f.device)
    (g,) = torch.autograd.grad((w * f).sum(), th)
    for j, p in enumerate(pts):
        f1, g1 = m.objective_adjoint(p)
        assert abs(float(f[j]) - f1) <= 1e-10 * abs(f1)
        assert rel(g[j].numpy(), float(w[j]) * g1) < 1e-10


def test_autograd_recomputes_an_overwritten_forward():
    """A second forward overwrites the device state of the first; the first
    one's backward recomputes its forward and still returns its gradient."""
    import torch

    from dalia_b200.autograd import objective
    from dalia_b200.model import SpatioTemporalModel

    gld = load("gst_small")
    m = SpatioTemporalModel(problem(gld))
    th1 = torch.tensor(gld["theta"], dtype=torch.float64, requires_grad=True)
    th2 = torch.tensor(gld["theta"] + 0.05, dtype=torch.float64, requires_grad=True)
    f1 = objective(m, th1)
    f2 = objective(m, th2)
    (g1,) = torch.autograd.grad(f1, th1)
    (g2,) = torch.autograd.grad(f2, th2)
    _, r1 = m.objective_adjoint(gld["theta"])
    _, r2 = m.objective_adjoint(gld["theta"] + 0.05)
    assert rel(g1.numpy(), r1) < 1e-12
    assert rel(g2.numpy(), r2) < 1e-12


def test_autograd_gradient_against_finite_differences_of_its_forward():
    """Fine central differences of the autograd forward itself (h = 1e-5)."""
    import torch

    from dalia_b200.autograd import objective
    from dalia_b200.model import SpatioTemporalModel

    gld = load("gst_small")
    m = SpatioTemporalModel(problem(gld))
    theta = np.asarray(gld["theta"], dtype=np.float64)
    _, g = _grad(m, theta)
    h = 1e-5
    fd = np.zeros_like(theta)
    with torch.no_grad():
        for k in range(theta.size):
            e = np.zeros_like(theta)
            e[k] = h
            fp = float(objective(m, torch.tensor(theta + e)))
            fm = float(objective(m, torch.tensor(theta - e)))
            fd[k] = (fp - fm) / (2 * h)
    assert rel(g, fd) < 1e-6


def test_autograd_mixed_precision_within_bar():
    """The 8-bit-slice selected inversion behind the backward: gradient
    within 1e-6 of the FP64 backward, f unchanged (the forward is FP64)."""
    from dalia_b200.model import SpatioTemporalModel

    gld = load("gst_300x10")
    m = SpatioTemporalModel(problem(gld))
    f64, g64 = _grad(m, gld["theta"], precision="fp64")
    fi8, gi8 = _grad(m, gld["theta"], precision="i8slice")
    assert abs(fi8 - f64) <= 1e-13 * abs(f64)
    assert rel(gi8, g64) < 1e-6
    assert not m.last_check[0]["fallback"]
