"""Pin the CPU oracle against outputs of the reference itself (DALIA, run in
this repository's build container by ``tests/golden/make_golden.py``)."""
import numpy as np
import pytest
import scipy.sparse as sps

from golden_util import load, problem, rel
from oracle import bta_ref, model_ref

GAUSS = ["gst_small", "gst_ragged"]
POIS = ["pst_small", "pst_150x6"]


@pytest.mark.parametrize("name", GAUSS)
def test_assembly_matches_reference(name):
    g = load(name)
    prob = problem(g)
    om = model_ref.OracleModel(prob)
    th = g["theta"]
    N = om.N
    Qp_ref = sps.coo_matrix((g["qp_data"], (g["qp_row"], g["qp_col"])), shape=(N, N)).toarray()
    Qc_ref = sps.coo_matrix((g["qc_data"], (g["qc_row"], g["qc_col"])), shape=(N, N)).toarray()
    assert rel(om.q_prior(th).toarray(), Qp_ref) < 1e-13
    assert rel(om.q_cond(th, np.zeros(len(prob.y))).toarray(), Qc_ref) < 1e-13


@pytest.mark.parametrize("name", GAUSS)
def test_bta_oracle_matches_dense_lapack(name):
    g = load(name)
    ns, nt, nb = (int(v) for v in g["shape"][:3])
    N = ns * nt + nb
    Qc = sps.coo_matrix((g["qc_data"], (g["qc_row"], g["qc_col"])), shape=(N, N))
    D, L, Ab, T = bta_ref.sparse_to_bta(Qc, nt, ns, nb)
    bta_ref.pobtaf(D, L, Ab, T)
    assert abs(bta_ref.logdet(D, T) - float(g["logdet_qc"])) < 1e-10 * abs(float(g["logdet_qc"]))
    x = g["rhs"].copy()
    bta_ref.pobtas(D, L, Ab, T, x, "N")
    bta_ref.pobtas(D, L, Ab, T, x, "C")
    assert rel(x, g["x_solve"]) < 1e-10
    bta_ref.pobtasi(D, L, Ab, T)
    for k, arr in (("sel_D", D), ("sel_L", L), ("sel_Ab", Ab), ("sel_T", T)):
        assert rel(arr, g[k]) < 1e-10, k


@pytest.mark.parametrize("name", GAUSS + POIS)
def test_objective_matches_reference_serinv_path(name):
    g = load(name)
    prob = problem(g)
    om = model_ref.OracleModel(prob)
    f, grad = om.objective(g["theta"])
    assert abs(f - float(g["f_serinv"])) < 1e-10 * max(1.0, abs(float(g["f_serinv"])))
    assert rel(grad, g["grad_serinv"]) < 1e-8
    assert rel(om.x, g["x_serinv"]) < 1e-10


@pytest.mark.parametrize("name", GAUSS + POIS)
def test_serinv_and_dense_paths_differ_by_tip_constant(name):
    """Reference quirk: the Serinv path's prior log-determinant drops the
    fixed-effect tip, so f differs from the dense path by -0.5 nb log(1e-3)."""
    g = load(name)
    nb = int(g["shape"][2])
    assert abs((float(g["f_dense"]) - float(g["f_serinv"])) - (-0.5 * nb * np.log(1e-3))) < 1e-8
    assert rel(g["grad_dense"], g["grad_serinv"]) < 1e-6


@pytest.mark.parametrize("name", GAUSS)
def test_marginal_variances_match_reference(name):
    g = load(name)
    prob = problem(g)
    om = model_ref.OracleModel(prob)
    mv = om.marginal_variances(g["theta"], g["x_dense"])
    assert rel(mv, g["marg_var_dense"]) < 1e-10
    assert rel(mv, g["marg_var_serinv"]) < 1e-10


def test_config0_scalars_match_reference():
    g = load("gst_300x10")
    prob = problem(g)
    om = model_ref.OracleModel(prob)
    f = om.evaluate_f(g["theta"])
    assert abs(f - float(g["f_serinv"])) < 1e-10 * abs(float(g["f_serinv"]))
    assert rel(om.x, g["x_dense"]) < 1e-9


@pytest.mark.parametrize("name", GAUSS)
def test_dense_adjoint_matches_reference_fd_gradient(name):
    """The adjoint formula (dense oracle) agrees with the reference's own FD
    gradient up to the FD truncation error (eps = 1e-3), and with a finer
    oracle FD to ~1e-8."""
    g = load(name)
    prob = problem(g)
    om = model_ref.OracleModel(prob)
    ga = model_ref.dense_adjoint_gradient(om, g["theta"])
    assert rel(ga, g["grad_serinv"]) < 1e-5
    om.eps = 1e-5
    _, gfd = om.objective(g["theta"])
    assert rel(ga, gfd) < 1e-7


@pytest.mark.parametrize("name", POIS)
def test_dense_poisson_adjoint_matches_fd_at_the_mode(name):
    """With a tight Newton tolerance (x* = the mode) the Poisson adjoint
    formula equals a fine central FD of the oracle objective."""
    g = load(name)
    prob = problem(g)
    th = g["theta"]
    om = model_ref.OracleModel(prob, eps_inner_iteration=1e-11)
    ga = model_ref.dense_adjoint_gradient_poisson(om, th)
    h = 1e-5
    fd = []
    for k in range(th.size):
        e = np.zeros(th.size)
        e[k] = h
        fd.append((om.evaluate_f(th + e) - om.evaluate_f(th - e)) / (2 * h))
    assert rel(ga, fd) < 1e-7
