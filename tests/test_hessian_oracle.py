"""The FD Hessian of the objective (DALIA._evaluate_hessian_f, the
θ-covariance behind compute_covariance_hp) restated in the oracle, against
fixtures written by running the reference's own method."""
import os

import numpy as np
import pytest

from golden_util import GOLDEN, coreg_problem, load, problem, rel
from oracle import coreg_ref, model_ref


def _hess(name):
    return dict(np.load(os.path.join(GOLDEN, f"hess_{name}.npz")))


@pytest.mark.parametrize("name", ["gst_small", "pst_small", "gst_coreg2_ragged"])
def test_oracle_hessian_matches_reference(name):
    g, h = load(name), _hess(name)
    if name.startswith("gst_coreg"):
        om = coreg_ref.CoregionalOracle(coreg_problem(g))
    else:
        om = model_ref.OracleModel(problem(g))
    H = model_ref.hessian_fd(om.evaluate_f, h["theta"], float(h["eps_hessian_f"]))
    assert rel(H, h["hess"]) < 1e-7
    assert np.allclose(H, H.T)
