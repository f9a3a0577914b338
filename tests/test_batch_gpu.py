"""Batched evaluation: the whole finite-difference stencil of a 15-parameter
coregional model in one batch, and a mixed-size batch (bivariate and
univariate models, different block and arrowhead sizes) whose
factorisations, sweeps and selected inversions share their launches.  Every
batched result equals the result of the same point evaluated on its own."""
import numpy as np
import pytest

from golden_util import rel

pytestmark = pytest.mark.gpu

TOL = 1e-10


def test_coregional_stencil_of_31_points_in_one_batch():
    """Trivariate coregional model, d = 15: all 2d + 1 = 31 stencil points of
    the reference's central differences (``dalia.py:558-564``) are factorised
    in one batched launch sequence (62 matrices), with the same f values as
    point-by-point evaluation."""
    from dalia_b200 import synth
    from dalia_b200.coregional import CoregionalModel

    cfg = synth.COREG_CONFIGS["gst_coreg3_600x40"]
    prob = synth.make_coregional_problem(ns=150, nt=6, nv=3, nb=1, no=60, theta=cfg["theta"], seed=3)
    m = CoregionalModel(prob)
    theta = np.asarray(cfg["theta"], dtype=np.float64)
    d = theta.size
    assert d == 15
    f_b, g_b = m.objective_fd_batched(theta)
    assert len(m.slots) >= 2 * d + 1  # the whole stencil was resident at once
    f_s, g_s = m.objective_fd(theta)
    assert abs(f_b - f_s) <= TOL * abs(f_s)
    # compare the stencil's f values directly (the FD quotient divides by 2 eps)
    pts = [theta] + [theta + m.eps * e for e in np.eye(d)] + [theta - m.eps * e for e in np.eye(d)]
    fb = m.evaluate_f_batched(pts)
    for p, fv in zip(pts, fb):
        f1 = m.evaluate_f(p)
        assert abs(fv - f1) <= TOL * abs(f1)
    assert rel(g_b, g_s) < 1e-6


def test_mixed_size_batch_shares_launches():
    """8 bivariate points (blocks 2 ns) and 16 univariate points (blocks ns)
    in one grouped adjoint evaluation: 48 matrices of two block sizes and
    two arrowhead sizes per launch; f and gradients equal each model's own
    batched evaluation."""
    from dalia_b200 import synth
    from dalia_b200.coregional import CoregionalModel
    from dalia_b200.model import SpatioTemporalModel, adjoint_group

    c2 = synth.COREG_CONFIGS["gst_coreg2_600x40"]
    u1 = synth.CONFIGS["gst_600x40"]
    m2 = CoregionalModel(synth.make_coregional_problem(ns=120, nt=5, nv=2, nb=1, no=50, theta=c2["theta"], seed=5))
    m1 = SpatioTemporalModel(synth.make_problem(120, 5, 1, 50, u1["theta"], "gaussian", seed=6))
    assert (m2.b, m2.nb, m1.b, m1.nb) == (240, 2, 120, 1)
    th2 = [np.asarray(c2["theta"]) + 0.01 * j for j in range(8)]
    th1 = [np.asarray(u1["theta"]) - 0.01 * j for j in range(16)]
    for precision in ("fp64", "i8slice"):
        (f2, g2), (f1, g1) = adjoint_group([(m2, th2), (m1, th1)], precision=precision)
        r2f, r2g = m2.objective_adjoint_batched(th2, precision=precision)
        r1f, r1g = m1.objective_adjoint_batched(th1, precision=precision)
        for a, b in zip(f2 + f1, r2f + r1f):
            assert abs(a - b) <= TOL * abs(b)
        for a, b in zip(g2 + g1, r2g + r1g):
            assert rel(a, b) < TOL
