"""Outer optimisation over theta: the reference's ``DALIA.minimize``
(``src/dalia/core/dalia.py:330-518``) on the device objectives.

scipy's L-BFGS-B minimises f(theta) = -log pi(theta | y) with its gradient,
options as the reference's ``BFGSConfig`` (``src/dalia/configs/dalia_config.py:18-31``;
``ftol`` fixed at 1e-22 as the reference passes it), and the reference's
callback: every accepted iterate's theta and f are recorded, and the run
stops early once f changed by less than ``f_reduction_tol`` over the last
``f_reduction_lag`` accepted iterates, or theta moved by less than
``theta_reduction_tol`` (2-norm) over the last ``theta_reduction_lag``
(``dalia.py:364-455``; defaults from ``DaliaConfig``, ``dalia_config.py:39-47``).

The gradient is the exact adjoint one (``gradient="adjoint"``, the default)
or the reference's central differences (``gradient="fd"``,
``model.objective_fd``), with which the iterates follow the reference's.
"""

from __future__ import annotations

import numpy as np

__all__ = ["minimize"]


class _EarlyExit(Exception):
    pass


def _host(x):
    if x is None:
        return None
    if hasattr(x, "detach"):
        return x.detach().cpu().numpy().copy()
    return np.array(x, copy=True)


def minimize(model, theta0, gradient: str = "adjoint", max_iter: int = 100, maxcor: int = 10, maxls: int = 20,
             gtol: float = 1e-1, disp: bool = False, f_reduction_lag: int = 3, f_reduction_tol: float = 1e-4,
             theta_reduction_lag: int = 3, theta_reduction_tol: float = 1e-4) -> dict:
    """Mode of pi(theta | y) from theta0.

    ``model`` provides ``objective_adjoint(theta)`` and/or
    ``objective_fd(theta)`` returning ``(f, grad)``, and ``x``, the latent
    mean / mode of its last evaluation.  Returns the reference's result
    dictionary: ``theta``, ``x`` (of the last evaluation), ``f``, ``grad_f``
    (last gradient evaluated), ``f_values`` and ``theta_values`` (accepted
    iterates), plus ``exit`` ("scipy", "f_reduction", "theta_reduction"),
    ``success``, ``message`` and ``n_evaluations``.  ``disp`` is accepted like
    the reference's config field; scipy's own iteration printout is not
    requested (current scipy no longer takes that option).
    """
    from scipy import optimize

    if gradient not in ("adjoint", "fd"):
        raise ValueError(f"gradient must be 'adjoint' or 'fd', not {gradient!r}")
    objective = model.objective_adjoint if gradient == "adjoint" else model.objective_fd
    theta0 = np.asarray(theta0, dtype=np.float64).copy()
    state = {"grad": None, "n": 0}

    if theta0.size == 0:
        # no hyperparameters: one evaluation (the reference runs its inner iteration)
        f, g = objective(theta0)
        return {"theta": theta0, "x": _host(getattr(model, "x", None)), "f": float(f), "grad_f": np.asarray(g),
                "f_values": [], "theta_values": [], "exit": "none", "success": True,
                "message": "no hyperparameters", "n_evaluations": 1}

    def fun(theta):
        f, g = objective(np.asarray(theta, dtype=np.float64).copy())
        state["grad"] = np.asarray(g, dtype=np.float64).copy()
        state["n"] += 1
        return float(f), state["grad"]

    f_values, theta_values = [], []
    result = {}

    def callback(intermediate_result):
        theta_i = np.asarray(intermediate_result.x, dtype=np.float64).copy()
        fun_i = float(intermediate_result.fun)
        theta_values.append(theta_i)
        f_values.append(fun_i)
        it = len(f_values)
        if it > f_reduction_lag and abs(f_values[-f_reduction_lag] - fun_i) < f_reduction_tol:
            result.update(exit="f_reduction", theta=theta_i, f=fun_i)
            raise _EarlyExit()
        if it > theta_reduction_lag and np.linalg.norm(theta_values[-theta_reduction_lag] - theta_i) < \
                theta_reduction_tol:
            result.update(exit="theta_reduction", theta=theta_i, f=fun_i)
            raise _EarlyExit()

    try:
        res = optimize.minimize(fun=fun, x0=theta0, method="L-BFGS-B", jac=True, callback=callback,
                                options={"maxiter": max_iter, "maxcor": maxcor, "maxls": maxls, "gtol": gtol,
                                         "ftol": 1e-22})
        result.update(exit="scipy", theta=np.asarray(res.x, dtype=np.float64), f=float(res.fun),
                      success=bool(res.success), message=str(res.message))
    except _EarlyExit:
        result.update(success=True, message=f"converged: {result['exit']}")
    result.update(x=_host(getattr(model, "x", None)), grad_f=state["grad"], f_values=f_values,
                  theta_values=theta_values, n_evaluations=state["n"])
    return result
