"""Outer L-BFGS-B driver (``dalia_b200.optimize.minimize``) on the CPU.

The driver's logic is pinned to the reference's ``DALIA.minimize`` run in the
build container (``tests/golden/min_<case>.npz``, made by
``make_golden.py --minimize``): driven by the oracle's objective (the
reference's f and central-difference gradient restated on the CPU), it must
reproduce the reference's accepted iterates and optimum.  The early-exit rules
are checked on small functions."""
import numpy as np
import pytest

from golden_util import load, problem
from oracle import model_ref
from dalia_b200.optimize import minimize


class OracleFD:
    """The oracle behind the interface ``minimize`` expects."""

    def __init__(self, prob):
        self.m = model_ref.OracleModel(prob)

    def objective_fd(self, theta):
        return self.m.objective(theta)

    @property
    def x(self):
        return self.m.x


@pytest.mark.parametrize("name", ["gst_small", "gst_ragged", "pst_small"])
def test_driver_reproduces_reference_minimize(name):
    g = load(name)
    ref = load(f"min_{name}")
    r = minimize(OracleFD(problem(g)), ref["theta0"], gradient="fd")
    assert r["exit"] == "scipy" and r["success"]
    assert len(r["f_values"]) == len(ref["f_values"])
    np.testing.assert_allclose(r["f_values"], ref["f_values"], rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(np.asarray(r["theta_values"]), ref["theta_values"], rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(r["theta"], ref["theta"], rtol=1e-6, atol=1e-6)
    assert abs(r["f"] - float(ref["f"])) < 1e-9 * max(1.0, abs(float(ref["f"])))
    np.testing.assert_allclose(r["grad_f"], ref["grad_f"], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(r["x"], ref["x"], rtol=1e-6, atol=1e-8)


class Quadratic:
    """f = |A theta - c|^2 / 2 with its exact gradient; x = last theta."""

    def __init__(self, d=4, seed=0):
        rng = np.random.default_rng(seed)
        self.A = rng.standard_normal((d + 2, d))
        self.c = rng.standard_normal(d + 2)
        self.x = None
        self.calls = 0

    def objective_adjoint(self, theta):
        self.calls += 1
        self.x = theta.copy()
        r = self.A @ theta - self.c
        return 0.5 * r @ r, self.A.T @ r


def test_f_reduction_exit_after_lag():
    m = Quadratic()
    r = minimize(m, np.full(4, 3.0), gtol=1e-14, f_reduction_lag=3, f_reduction_tol=1e30,
                 theta_reduction_tol=0.0)
    # the rule first applies at the fourth accepted iterate
    assert r["exit"] == "f_reduction" and len(r["f_values"]) == 4
    np.testing.assert_allclose(r["theta"], r["theta_values"][-1])
    assert r["f"] == r["f_values"][-1] and r["n_evaluations"] == m.calls


def test_theta_reduction_exit_after_lag():
    m = Quadratic(seed=1)
    r = minimize(m, np.full(4, -2.0), gtol=1e-14, f_reduction_tol=0.0, theta_reduction_lag=2,
                 theta_reduction_tol=1e30)
    assert r["exit"] == "theta_reduction" and len(r["f_values"]) == 3


def test_scipy_convergence_reaches_the_minimum():
    m = Quadratic(seed=2)
    r = minimize(m, np.zeros(4), gtol=1e-10, f_reduction_tol=0.0, theta_reduction_tol=0.0)
    assert r["exit"] == "scipy" and r["success"]
    best = np.linalg.lstsq(m.A, m.c, rcond=None)[0]
    np.testing.assert_allclose(r["theta"], best, atol=1e-6)
    # x is the model's state after its last evaluation
    np.testing.assert_allclose(r["x"], m.x)


def test_no_hyperparameters_evaluates_once():
    class Empty:
        x = np.arange(3.0)

        def objective_adjoint(self, theta):
            assert theta.size == 0
            return 1.5, np.zeros(0)

    r = minimize(Empty(), [])
    assert r["f"] == 1.5 and r["n_evaluations"] == 1 and r["theta"].size == 0


def test_rejects_unknown_gradient():
    with pytest.raises(ValueError):
        minimize(Quadratic(), np.zeros(4), gradient="bfgs")


class CoregOracleFD:
    def __init__(self, prob):
        from oracle.coreg_ref import CoregionalOracle

        self.m = CoregionalOracle(prob)

    def objective_fd(self, theta):
        return self.m.objective(theta)

    @property
    def x(self):
        return self.m.x


def test_driver_reproduces_reference_minimize_coregional_prefix():
    """The first three accepted iterates of the reference's run on the
    2-variate coregional problem (the whole run takes a minute on the CPU;
    the GPU test follows it to the end)."""
    from golden_util import coreg_problem

    g = load("gst_coreg2_ragged")
    ref = load("min_gst_coreg2_ragged")
    r = minimize(CoregOracleFD(coreg_problem(g)), ref["theta0"], gradient="fd", max_iter=3)
    assert len(r["f_values"]) == 3
    np.testing.assert_allclose(r["f_values"], ref["f_values"][:3], rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(np.asarray(r["theta_values"]), ref["theta_values"][:3], rtol=1e-6, atol=1e-6)
