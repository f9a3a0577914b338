"""The FD Hessian on the device against the reference's own
_evaluate_hessian_f (fixtures) for a Gaussian, a Poisson and a coregional
model."""
import os

import numpy as np
import pytest

from golden_util import GOLDEN, coreg_problem, load, problem, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["gst_small", "pst_small", "gst_coreg2_ragged"])
def test_hessian_matches_reference(name):
    from dalia_b200.coregional import CoregionalModel
    from dalia_b200.model import SpatioTemporalModel

    g = load(name)
    h = dict(np.load(os.path.join(GOLDEN, f"hess_{name}.npz")))
    if name.startswith("gst_coreg"):
        m = CoregionalModel(coreg_problem(g))
    else:
        m = SpatioTemporalModel(problem(g))
    H = m.hessian_fd(h["theta"], float(h["eps_hessian_f"]), max_points=8)
    assert rel(H, h["hess"]) < 1e-6
    if m.gaussian:
        # a Poisson Hessian depends on the Newton warm starts of the call, so
        # the covariance (a second Hessian) is checked on the Gaussian models
        C = m.covariance_theta(h["theta"], float(h["eps_hessian_f"]))
        assert rel(C @ h["hess"], np.eye(len(h["theta"]))) < 1e-5
