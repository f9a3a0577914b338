"""Generate the golden fixtures in ``tests/golden/`` by running the reference
(DALIA, pure Python) in this container on seeded synthetic problems.

Usage (needs the reference checkout; it is not needed to *use* the fixtures)::

    ARRAY_MODULE=numpy python tests/golden/make_golden.py /path/to/DALIA [CASE ...]

For every case the reference's own classes are driven end to end:

* ``Model.construct_Q_prior`` / ``construct_Q_conditional`` -> the sparse
  precision matrices (COO triplets are stored);
* ``DenseSolver`` (exact LAPACK, ``src/dalia/solvers/dense_solver.py``):
  log-determinant, solution, full inverse restricted to the BTA pattern,
  marginal variances, ``f(theta)`` and the central-FD gradient via
  ``DALIA._objective_function``;
* ``SerinvSolver`` with ``serinv.algs`` provided by ``oracle.bta_ref`` (Serinv
  itself is not installable here): ``f(theta)`` and gradient.  For the Poisson
  case the solver's ``cholesky`` gets ``sparsity="bta"`` as default, because
  the reference calls it without that argument (``src/dalia/core/dalia.py:1058``).

The dense path pins the oracle; the Serinv path pins the oracle's restatement
of DALIA's driver logic (including the prior log-determinant quirk: ``"bt"``
drops the fixed-effect tip).
"""

from __future__ import annotations

import os
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


CASES = {
    # name: (ns, nt, nb, no, theta, likelihood, seed, store_selinv)
    "gst_small": (48, 4, 3, 40, (-1.0, 1.0, 0.0, 2.0), "gaussian", 1, True),
    "gst_ragged": (70, 3, 2, 50, (-0.5, 0.7, 0.2, 1.5), "gaussian", 2, True),
    "pst_small": (40, 4, 2, 60, (-1.2, 0.8, -0.3), "poisson", 3, False),
    "gst_300x10": (300, 10, 4, 200, (-1.0, 1.0, 0.0, 2.0), "gaussian", 0, False),
    "pst_150x6": (150, 6, 3, 120, (-1.0, 0.9, -0.2), "poisson", 4, False),
}


COREG_CASES = {
    # name: (ns, nt, nv, nb per variate, no, theta, seed)
    "gst_coreg3_small": (40, 4, 3, 1, 30, (-1.0, 1.0, 2.0, -0.8, 0.9, 1.8, -1.2, 1.1, 2.2,
                                           0.0, 0.2, -0.1, 0.5, -0.3, 0.4), 5),
    "gst_coreg2_ragged": (70, 3, 2, 2, 40, (-0.9, 0.8, 1.5, -1.1, 1.2, 2.1, 0.1, -0.2, 0.6), 6),
}


def checksums(prob):
    out = {}
    for nm in ("c0", "g1", "g2", "g3", "m0", "m1", "m2", "a_st"):
        d = getattr(prob, nm).tocsc().data
        out[nm] = np.array([d.sum(), (d * d).sum(), d.size], dtype=np.float64)
    out["a_fe"] = np.array([prob.a_fe.sum(), (prob.a_fe ** 2).sum(), prob.a_fe.size])
    out["y"] = np.array([prob.y.sum(), (prob.y ** 2).sum(), prob.y.size])
    return out


def _save_hessian(name, th, dal):
    """hess_<name>.npz: DALIA._evaluate_hessian_f at theta (Serinv path,
    default eps_hessian_f = 5e-3, points evaluated in the reference's order)."""
    h = dal._evaluate_hessian_f(th.copy())
    np.savez_compressed(os.path.join(HERE, f"hess_{name}.npz"), theta=th, hess=np.asarray(h),
                        eps_hessian_f=np.array(dal.eps_hessian_f))
    print(f"hess_{name}: diag={np.diag(np.asarray(h))}", flush=True)


def _save_minimize(name, th, dal):
    """min_<name>.npz: DALIA.minimize from theta (Serinv path, the reference's
    default BFGSConfig and early-exit settings, FD gradient)."""
    r = dal.minimize()
    out = {"theta0": th, "theta": np.asarray(r["theta"], dtype=np.float64), "f": np.array(r["f"]),
           "f_values": np.asarray(r["f_values"], dtype=np.float64),
           "theta_values": np.asarray(r["theta_values"], dtype=np.float64),
           "grad_f": np.asarray(r["grad_f"], dtype=np.float64), "x": np.asarray(r["x"], dtype=np.float64)}
    np.savez_compressed(os.path.join(HERE, f"min_{name}.npz"), **out)
    print(f"min_{name}: theta*={out['theta']} f*={float(out['f']):.10f} iterations={len(out['f_values'])}",
          flush=True)


def main(ref_root: str, only=None, hessian=False, minimize=False) -> None:
    os.environ.setdefault("ARRAY_MODULE", "numpy")
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(ref_root, "src"))

    from oracle import bta_ref

    fake = types.ModuleType("serinv")
    algs = types.ModuleType("serinv.algs")
    for nm in ("pobtaf", "pobtas", "pobtasi", "pobtf", "pobts", "pobtsi"):
        setattr(algs, nm, getattr(bta_ref, nm))
    fake.algs = algs
    sys.modules["serinv"] = fake
    sys.modules["serinv.algs"] = algs

    from dalia.configs import dalia_config, likelihood_config, submodels_config
    from dalia.core.dalia import DALIA
    from dalia.core.model import Model
    from dalia.solvers.structured_solver import SerinvSolver
    from dalia.submodels import RegressionSubModel, SpatioTemporalSubModel

    from dalia_b200 import synth

    _orig_chol = SerinvSolver.cholesky

    def _chol_default(self, A, sparsity="bta"):
        return _orig_chol(self, A, sparsity)

    SerinvSolver.cholesky = _chol_default

    for name, (ns, nt, nb, no, theta, lik, seed, store_selinv) in CASES.items():
        if only and name not in only:
            continue
        prob = synth.make_problem(ns, nt, nb, no, theta, lik, seed=seed)
        tmp = tempfile.mkdtemp(prefix=f"golden_{name}_")
        synth.save_dalia_layout(prob, tmp)

        def build(solver_type):
            st = SpatioTemporalSubModel(config=submodels_config.parse_config({
                "type": "spatio_temporal",
                "input_dir": f"{tmp}/inputs_spatio_temporal",
                "spatial_domain_dimension": 2,
                "r_s": theta[0], "r_t": theta[1], "sigma_st": theta[2],
                "manifold": "plane",
                "ph_s": {"type": "penalized_complexity", "alpha": 0.01, "u": 0.5},
                "ph_t": {"type": "penalized_complexity", "alpha": 0.01, "u": 5},
                "ph_st": {"type": "penalized_complexity", "alpha": 0.01, "u": 3},
            }))
            rg = RegressionSubModel(config=submodels_config.parse_config({
                "type": "regression",
                "input_dir": f"{tmp}/inputs_regression",
                "n_fixed_effects": nb,
                "fixed_effects_prior_precision": 0.001,
            }))
            if lik == "gaussian":
                ld = {"type": "gaussian", "prec_o": theta[3],
                      "prior_hyperparameters": {"type": "penalized_complexity", "alpha": 0.01, "u": 4}}
            else:
                ld = {"type": "poisson", "input_dir": tmp}
            model = Model(submodels=[rg, st], likelihood_config=likelihood_config.parse_config(ld))
            dal = DALIA(model=model, config=dalia_config.parse_config({
                "solver": {"type": solver_type},
                "inner_iteration_max_iter": 50,
                "eps_inner_iteration": 1e-3,
                "eps_gradient_f": 1e-3,
                "simulation_dir": tmp,
            }))
            dal.iter = 0
            return model, dal

        out = {"theta": np.asarray(theta, dtype=np.float64),
               "shape": np.array([ns, nt, nb, no, seed]),
               "likelihood": np.array(lik)}
        for k, v in checksums(prob).items():
            out[f"chk_{k}"] = v

        th = np.asarray(theta, dtype=np.float64)
        if hessian:
            _save_hessian(name, th, build("serinv")[1])
            continue
        if minimize:
            _save_minimize(name, th, build("serinv")[1])
            continue

        # --- dense solver: exact reference numbers
        model, dal = build("dense")
        model.theta[:] = th
        Qp = model.construct_Q_prior().tocoo()
        eta0 = np.zeros_like(model.y)
        Qc = model.construct_Q_conditional(eta0).tocoo()
        if lik == "gaussian" and store_selinv:
            out["qp_row"], out["qp_col"], out["qp_data"] = Qp.row, Qp.col, Qp.data
            out["qc_row"], out["qc_col"], out["qc_data"] = Qc.row, Qc.col, Qc.data
        if lik == "gaussian":
            dal.solver.cholesky(Qc)
            out["logdet_qc"] = np.array(dal.solver.logdet())
            rhs = model.construct_information_vector(eta0, np.zeros_like(model.x))
            out["rhs"] = rhs.copy()
            out["x_solve"] = dal.solver.solve(rhs.copy()).copy()
            if store_selinv:
                Sinv = dal.solver.selected_inversion()
                D, L, Ab, T = bta_ref.dense_to_bta(np.asarray(Sinv), nt, ns, nb)
                out["sel_D"], out["sel_L"], out["sel_Ab"], out["sel_T"] = D, L, Ab, T
        f_d, g_d = dal._objective_function(th.copy())
        out["f_dense"] = np.array(f_d)
        out["grad_dense"] = np.asarray(g_d)
        out["x_dense"] = model.x.copy()
        if lik == "gaussian":
            out["marg_var_dense"] = dal.get_marginal_variances_latent_parameters(
                th.copy(), model.x.copy())

        # --- Serinv solver path (serinv.algs = BTA oracle)
        model, dal = build("serinv")
        f_s, g_s = dal._objective_function(th.copy())
        out["f_serinv"] = np.array(f_s)
        out["grad_serinv"] = np.asarray(g_s)
        out["x_serinv"] = model.x.copy()
        if lik == "gaussian":
            out["marg_var_serinv"] = dal.get_marginal_variances_latent_parameters(
                th.copy(), model.x.copy())

        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(f"{name}: f_dense={f_d:.10f} f_serinv={f_s:.10f} "
              f"diff={f_d - f_s:.6f} grad_serinv={np.asarray(g_s)}", flush=True)


def coreg_checksums(prob):
    out = {}
    for nm in ("c0", "g1", "g2", "g3", "m0", "m1", "m2"):
        d = getattr(prob, nm).tocsc().data
        out[nm] = np.array([d.sum(), (d * d).sum(), d.size], dtype=np.float64)
    for v in range(prob.nv):
        d = prob.a_st[v].tocsc().data
        out[f"a_st{v}"] = np.array([d.sum(), (d * d).sum(), d.size])
        out[f"a_fe{v}"] = np.array([prob.a_fe[v].sum(), (prob.a_fe[v] ** 2).sum(), prob.a_fe[v].size])
        out[f"y{v}"] = np.array([prob.y[v].sum(), (prob.y[v] ** 2).sum(), prob.y[v].size])
    return out


def main_coregional(ref_root: str, only=None, hessian=False, minimize=False) -> None:
    """Coregional fixtures: the reference's ``CoregionalModel`` built from one
    ``Model`` per variate (Gaussian priors as in its coregional examples),
    driven through ``DALIA._objective_function`` with the dense and the
    Serinv solvers."""
    os.environ.setdefault("ARRAY_MODULE", "numpy")
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(ref_root, "src"))
    from oracle import bta_ref

    fake = types.ModuleType("serinv")
    algs = types.ModuleType("serinv.algs")
    for nm in ("pobtaf", "pobtas", "pobtasi", "pobtf", "pobts", "pobtsi"):
        setattr(algs, nm, getattr(bta_ref, nm))
    fake.algs = algs
    sys.modules["serinv"] = fake
    sys.modules["serinv.algs"] = algs

    from dalia.configs import dalia_config, likelihood_config, models_config, submodels_config
    from dalia.core.dalia import DALIA
    from dalia.core.model import Model
    from dalia.models import CoregionalModel
    from dalia.submodels import RegressionSubModel, SpatioTemporalSubModel

    from dalia_b200 import synth

    g = lambda mean: {"type": "gaussian", "mean": float(mean), "precision": 0.5}
    for name, (ns, nt, nv, nb, no, theta, seed) in COREG_CASES.items():
        if only and name not in only:
            continue
        prob = synth.make_coregional_problem(ns, nt, nv, nb, no, theta, seed=seed)
        th = np.asarray(theta, dtype=np.float64)
        tmp = tempfile.mkdtemp(prefix=f"golden_{name}_")
        synth.save_coregional_layout(prob, tmp)

        def build(solver_type):
            models = []
            for v in range(nv):
                mdir = f"{tmp}/model_{v + 1}"
                st = SpatioTemporalSubModel(config=submodels_config.parse_config({
                    "type": "spatio_temporal", "input_dir": f"{mdir}/inputs_spatio_temporal",
                    "spatial_domain_dimension": 2, "r_s": th[3 * v], "r_t": th[3 * v + 1], "sigma_st": 0.0,
                    "manifold": "plane", "ph_s": g(th[3 * v]), "ph_t": g(th[3 * v + 1]), "ph_st": g(0.0)}))
                rg = RegressionSubModel(config=submodels_config.parse_config({
                    "type": "regression", "input_dir": f"{mdir}/inputs_regression", "n_fixed_effects": nb,
                    "fixed_effects_prior_precision": 0.001}))
                lk = likelihood_config.parse_config({
                    "type": "gaussian", "prec_o": th[3 * v + 2], "prior_hyperparameters": g(th[3 * v + 2])})
                models.append(Model(submodels=[st, rg], likelihood_config=lk))
            cfg = {"type": "coregional", "n_models": nv,
                   "sigmas": [float(x) for x in th[3 * nv:4 * nv]],
                   "lambdas": [float(x) for x in th[4 * nv:]],
                   "ph_sigmas": [g(x) for x in th[3 * nv:4 * nv]],
                   "ph_lambdas": [g(0.0) for _ in th[4 * nv:]]}
            model = CoregionalModel(models=models, coregional_model_config=models_config.parse_config(cfg))
            dal = DALIA(model=model, config=dalia_config.parse_config({
                "solver": {"type": solver_type}, "inner_iteration_max_iter": 50,
                "eps_inner_iteration": 1e-3, "eps_gradient_f": 1e-3, "simulation_dir": tmp}))
            dal.iter = 0
            return model, dal

        if hessian:
            _save_hessian(name, th, build("serinv")[1])
            continue
        if minimize:
            _save_minimize(name, th, build("serinv")[1])
            continue
        out = {"theta": th, "shape": np.array([ns, nt, nv, nb, no, seed])}
        for k, v in coreg_checksums(prob).items():
            out[f"chk_{k}"] = v
        model, dal = build("dense")
        model.theta[:] = th
        Qp = model.construct_Q_prior().tocoo()
        Qc = model.construct_Q_conditional(np.zeros_like(model.y)).tocoo()
        out["qp_row"], out["qp_col"], out["qp_data"] = Qp.row, Qp.col, Qp.data
        out["qc_row"], out["qc_col"], out["qc_data"] = Qc.row, Qc.col, Qc.data
        f_d, g_d = dal._objective_function(th.copy())
        out["f_dense"], out["grad_dense"], out["x_dense"] = np.array(f_d), np.asarray(g_d), model.x.copy()
        model, dal = build("serinv")
        f_s, g_s = dal._objective_function(th.copy())
        out["f_serinv"], out["grad_serinv"], out["x_serinv"] = np.array(f_s), np.asarray(g_s), model.x.copy()
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(f"{name}: f_dense={f_d:.10f} f_serinv={f_s:.10f} diff={f_d - f_s:.6f}", flush=True)


if __name__ == "__main__":
    # usage: make_golden.py [REF_ROOT [--hessian | --minimize] [CASE ...]]
    #   --hessian writes hess_<CASE>.npz (the reference's FD Hessian) instead,
    #   --minimize writes min_<CASE>.npz (the reference's DALIA.minimize)
    _root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DALIA_REF")
    if not _root or not os.path.isdir(os.path.join(_root, "src", "dalia")):
        sys.exit("usage: make_golden.py REF_ROOT [--hessian | --minimize] [CASE ...]  (or set DALIA_REF): "
                 "REF_ROOT is a DALIA checkout containing src/dalia")
    _hess = "--hessian" in sys.argv[2:]
    _min = "--minimize" in sys.argv[2:]
    _only = [a for a in sys.argv[2:] if a not in ("--hessian", "--minimize")]
    if _min:
        if any(c in CASES for c in _only):
            main(_root, [c for c in _only if c in CASES], minimize=True)
        if any(c in COREG_CASES for c in _only):
            main_coregional(_root, [c for c in _only if c in COREG_CASES], minimize=True)
        sys.exit(0)
    if not _only or any(c in CASES for c in _only):
        main(_root, [c for c in _only if c in CASES], hessian=_hess)
    if not _only or any(c in COREG_CASES for c in _only):
        main_coregional(_root, [c for c in _only if c in COREG_CASES], hessian=_hess)
