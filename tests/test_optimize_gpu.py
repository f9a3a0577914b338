"""Outer L-BFGS-B driver on the device objectives against the reference's
``DALIA.minimize`` (``tests/golden/min_<case>.npz``).

With the reference's central-difference gradient (``gradient="fd"``) the
device objective must retrace the reference's accepted iterates (its f and FD
gradient agree with the reference's to ~1e-10 and ~1e-7).  With the exact
adjoint gradient the path differs slightly; the optimum must agree to the
accuracy L-BFGS-B stops at (gtol = 0.1 on the gradient)."""
import numpy as np
import pytest

from golden_util import load, problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["gst_small", "gst_ragged", "pst_small"])
def test_fd_driver_retraces_reference(name):
    from dalia_b200.model import SpatioTemporalModel
    from dalia_b200.optimize import minimize

    g, ref = load(name), load(f"min_{name}")
    r = minimize(SpatioTemporalModel(problem(g)), ref["theta0"], gradient="fd")
    assert r["exit"] == "scipy" and r["success"]
    assert len(r["f_values"]) == len(ref["f_values"])
    np.testing.assert_allclose(r["f_values"], ref["f_values"], rtol=1e-8, atol=1e-8)
    np.testing.assert_allclose(r["theta"], ref["theta"], rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(r["x"], ref["x"], rtol=1e-5, atol=1e-7)


@pytest.mark.parametrize("name", ["gst_small", "gst_ragged", "pst_small"])
def test_adjoint_driver_reaches_reference_optimum(name):
    from dalia_b200.model import SpatioTemporalModel
    from dalia_b200.optimize import minimize

    g, ref = load(name), load(f"min_{name}")
    model = SpatioTemporalModel(problem(g))
    r = minimize(model, ref["theta0"])
    f_ref = float(ref["f"])
    assert r["success"]
    assert abs(r["f"] - f_ref) < 1e-3 * max(1.0, abs(f_ref))
    assert np.linalg.norm(r["theta"] - ref["theta"]) < 0.1 * max(1.0, np.linalg.norm(ref["theta"]))
    # the adjoint gradient at the returned point is small, as L-BFGS-B's stop demands
    _, gr = model.objective_adjoint(r["theta"])
    assert np.max(np.abs(gr)) < 1.0


def test_fd_driver_retraces_reference_coregional():
    from golden_util import coreg_problem

    from dalia_b200.coregional import CoregionalModel
    from dalia_b200.optimize import minimize

    g, ref = load("gst_coreg2_ragged"), load("min_gst_coreg2_ragged")
    m = CoregionalModel(coreg_problem(g))
    r = minimize(m, ref["theta0"], gradient="fd")
    assert r["exit"] == "scipy" and r["success"]
    assert len(r["f_values"]) == len(ref["f_values"])
    np.testing.assert_allclose(r["f_values"], ref["f_values"], rtol=1e-8, atol=1e-8)
    np.testing.assert_allclose(r["theta"], ref["theta"], rtol=1e-5, atol=1e-5)
    # the adjoint driver reaches the same optimum
    ra = minimize(CoregionalModel(coreg_problem(g)), ref["theta0"])
    assert abs(ra["f"] - float(ref["f"])) < 1e-3 * max(1.0, abs(float(ref["f"])))
