"""CPU oracle: the reference's spatio-temporal INLA objective restated with
SciPy sparse matrices and the BTA oracle in ``oracle.bta_ref``.

TEST INFRASTRUCTURE ONLY (see ``oracle/bta_ref.py``).

Restated reference behaviour, with citations:

* theta -> (gamma_s, gamma_t, gamma_st), plane manifold:
  ``src/dalia/submodels/spatio_temporal.py:151-197``
* ``Q_st = e^{2 g_st} [m0 (x) q3 + e^{g_t} m1 (x) q2 + e^{2 g_t} m2 (x) q1]``:
  ``spatio_temporal.py:114-149``; regression tip ``prec * I``:
  ``src/dalia/submodels/regression.py:27-35``; concatenation with the
  spatio-temporal block first: ``src/dalia/core/model.py:49-53,306-382``
* ``Q_c = Q_prior - A^T D A``: ``model.py:384-423``; Gaussian
  ``D = -e^{theta_y} I`` (``src/dalia/likelihoods/gaussian.py:98-131``),
  Poisson ``D = -diag(e exp(eta))`` (``src/dalia/likelihoods/poisson.py:55-63``)
* information vector ``-Q_prior x + A^T grad``: ``model.py:425-449``
* Gaussian f: ``src/dalia/core/dalia.py:631-698`` with
  ``_evaluate_conditional_latent_parameters`` (``:1110-1168``) and
  ``_evaluate_prior_latent_parameters`` (``:1074-1108``)
* non-Gaussian f + Newton inner iteration: ``dalia.py:699-729,1023-1072``
* central finite-difference gradient, reverse evaluation order:
  ``dalia.py:513-601``
* penalised-complexity priors:
  ``src/dalia/prior_hyperparameters/penalized_complexity.py:28-82``

The Serinv solver path is followed: the prior log-determinant is taken from a
BT factorisation of the spatio-temporal block only, so the fixed-effect tip is
excluded (``structured_solver.py:156-161`` with ``sparsity="bt"``).  The
reference's non-Gaussian path calls ``solver.cholesky(A=Q)`` without the
``sparsity`` argument (``dalia.py:1058``); here it is "bta".
"""

from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sps
import scipy.special as ssp

from . import bta_ref

# alpha_s = 2, alpha_t = 1, alpha_e = 1 (spatio_temporal.py:157-166)
_ALPHA_S, _ALPHA_T, _ALPHA_E = 2, 1, 1
_ALPHA = _ALPHA_E + _ALPHA_S * (_ALPHA_T - 0.5)
_NU_S = _ALPHA - 1
_NU_T = _ALPHA_T - 0.5
_C1 = (
    ssp.gamma(_NU_T) * ssp.gamma(_NU_S)
    / (ssp.gamma(_ALPHA_T) * ssp.gamma(_ALPHA) * pow(4 * math.pi, 1.5))
)

# PC priors as in the reference's gst examples (examples/gst_small/run.py:33-60)
DEFAULT_PRIORS = {
    "r_s": (0.01, 0.5),
    "r_t": (0.01, 5.0),
    "sigma_st": (0.01, 3.0),
    "prec_o": (0.01, 4.0),
}


def theta_to_gamma(r_s, r_t, sigma_st):
    g_s = 0.5 * math.log(8 * _NU_S) - r_s
    g_t = r_t - 0.5 * math.log(8 * _NU_T) + _ALPHA_S * g_s
    g_st = 0.5 * math.log(_C1) - 0.5 * g_t - _NU_S * g_s - sigma_st
    return g_s, g_t, g_st


def pc_log_prior(kind, theta, alpha, u):
    if kind == "r_s":
        lam = -math.log(alpha) * pow(u, 1.0)  # spatial_dim = 2 -> u^(d/2)
        return math.log(lam) - lam * math.exp(-theta) - theta
    if kind == "r_t":
        lam = -math.log(alpha) * pow(u, 0.5)
        return math.log(lam) - lam * math.exp(-0.5 * theta) + math.log(0.5) - 0.5 * theta
    if kind in ("sigma_st", "sigma_e", "prec_o"):
        lam = -math.log(alpha) / u
        return math.log(lam) - lam * math.exp(theta) + theta
    raise ValueError(kind)


class OracleModel:
    """Univariate spatio-temporal model (DEMF(1,2,1) + fixed effects)."""

    def __init__(self, prob, priors=None, fe_prec=1e-3, eps_gradient_f=1e-3,
                 eps_inner_iteration=1e-3, inner_iteration_max_iter=50):
        self.p = prob
        self.priors = dict(DEFAULT_PRIORS if priors is None else priors)
        self.fe_prec = fe_prec
        self.ns, self.nt, self.nb = prob.ns, prob.nt, prob.nb
        self.N = prob.ns * prob.nt + prob.nb
        self.A = prob.a.tocsr()
        self.AT = self.A.T.tocsr()
        self.y = prob.y
        self.gaussian = prob.likelihood == "gaussian"
        self.e = prob.e if prob.e is not None else np.ones(len(prob.y))
        self.eps = eps_gradient_f
        self.eps_inner = eps_inner_iteration
        self.max_inner = inner_iteration_max_iter
        self.x = np.zeros(self.N)
        self.theta_keys = ["r_s", "r_t", "sigma_st"] + (["prec_o"] if self.gaussian else [])

    # -- assembly ---------------------------------------------------------
    def q_st(self, theta):
        p = self.p
        g_s, g_t, g_st = theta_to_gamma(theta[0], theta[1], theta[2])
        es, et, est = math.exp(g_s), math.exp(g_t), math.exp(g_st)
        q1 = es ** 2 * p.c0 + p.g1
        q2 = es ** 4 * p.c0 + 2 * es ** 2 * p.g1 + p.g2
        q3 = es ** 6 * p.c0 + 3 * es ** 4 * p.g1 + 3 * es ** 2 * p.g2 + p.g3
        return sps.csc_matrix(
            est ** 2 * (sps.kron(p.m0, q3) + et * sps.kron(p.m1, q2) + et ** 2 * sps.kron(p.m2, q1))
        )

    def q_prior(self, theta):
        return sps.block_diag(
            [self.q_st(theta), self.fe_prec * sps.eye(self.nb)], format="csc"
        )

    def d_diag(self, theta, eta):
        """Diagonal of ``-Hessian`` of the log-likelihood in eta."""
        if self.gaussian:
            return np.full(len(self.y), math.exp(theta[-1]))
        return self.e * np.exp(eta)

    def q_cond(self, theta, eta):
        Qp = self.q_prior(theta)
        return (Qp + self.AT @ sps.diags(self.d_diag(theta, eta)) @ self.A).tocsc()

    def grad_lik(self, theta, eta):
        if self.gaussian:
            return -math.exp(theta[-1]) * (eta - self.y)
        return self.y - self.e * np.exp(eta)

    def lik(self, theta, eta):
        if self.gaussian:
            r = eta - self.y
            return 0.5 * theta[-1] * len(self.y) - 0.5 * math.exp(theta[-1]) * (r @ r)
        return float(eta @ self.y - np.sum(self.e * np.exp(eta)))

    def log_prior_theta(self, theta):
        s = 0.0
        for k, key in enumerate(self.theta_keys):
            al, u = self.priors[key]
            s += pc_log_prior(key, theta[k], al, u)
        return s

    # -- solver (Serinv semantics through the BTA oracle) ------------------
    def _factor_bta(self, Q):
        D, L, Ab, T = bta_ref.sparse_to_bta(Q, self.nt, self.ns, self.nb)
        bta_ref.pobtaf(D, L, Ab, T)
        return D, L, Ab, T

    def _logdet_prior_bt(self, theta):
        D, L, _, _ = bta_ref.sparse_to_bta(self.q_st(theta), self.nt, self.ns, 0)
        bta_ref.pobtf(D, L)
        return bta_ref.logdet(D, None, sparsity="bt")

    def _solve(self, fac, rhs):
        D, L, Ab, T = fac
        x = rhs.copy()
        bta_ref.pobtas(D, L, Ab, T, x, "N")
        bta_ref.pobtas(D, L, Ab, T, x, "C")
        return x

    # -- objective ------------------------------------------------------------
    def evaluate_f(self, theta):
        theta = np.asarray(theta, dtype=np.float64)
        if self.gaussian:
            eta = np.zeros(len(self.y))
            Qc = self.q_cond(theta, eta)
            fac = self._factor_bta(Qc)
            rhs = -self.q_prior(theta) @ np.zeros(self.N) + self.AT @ self.grad_lik(theta, eta)
            mu = self._solve(fac, rhs)
            self.x[:] = mu
            cond = 0.5 * bta_ref.logdet(fac[0], fac[3], "bta") - 0.5 * mu @ (Qc @ mu)
            f = cond - (
                self.log_prior_theta(theta) + self.lik(theta, eta)
                + 0.5 * self._logdet_prior_bt(theta)
            )
        else:
            Qc, xs, eta = self.inner_iteration(theta)
            self.x[:] = xs
            fac = self._factor_bta(Qc)
            cond = 0.5 * bta_ref.logdet(fac[0], fac[3], "bta")
            Qp = self.q_prior(theta)
            prior_x = 0.5 * self._logdet_prior_bt(theta) - 0.5 * xs @ (Qp @ xs)
            f = -(self.log_prior_theta(theta) + self.lik(theta, eta) + prior_x - cond)
        if np.isnan(f):
            raise ValueError("f(theta) is NaN")
        return float(f)

    def inner_iteration(self, theta):
        Qp = self.q_prior(theta)
        x_star = self.x.copy()
        x_update = np.zeros(self.N)
        norm = 1.0
        counter = 0
        while norm >= self.eps_inner:
            if counter > self.max_inner:
                raise ValueError(f"Inner iteration did not converge after {counter} iterations.")
            x_star += x_update
            eta = self.A @ x_star
            Qc = self.q_cond(theta, eta)
            fac = self._factor_bta(Qc)
            rhs = -Qp @ x_star + self.AT @ self.grad_lik(theta, eta)
            x_update = self._solve(fac, rhs)
            norm = np.linalg.norm(x_update)
            counter += 1
        return Qc, x_star, eta

    def objective(self, theta):
        """(f(theta), central-FD gradient) with the reference's ordering."""
        theta = np.asarray(theta, dtype=np.float64)
        d = len(theta)
        nf = 2 * d + 1
        tm = np.repeat(theta.reshape(-1, 1), nf, axis=1)
        tm[:, 1:1 + d] += self.eps * np.eye(d)
        tm[:, d + 1:nf] -= self.eps * np.eye(d)
        fv = np.zeros(nf)
        for k in range(nf - 1, -1, -1):
            fv[k] = self.evaluate_f(tm[:, k])
        grad = (fv[1:1 + d] - fv[d + 1:nf]) / (2 * self.eps)
        return fv[0], grad

    def marginal_variances(self, theta, x_star=None):
        """``diag(Q_c^{-1})`` via the BTA selected inverse
        (``dalia.py:912-962``)."""
        x_star = self.x if x_star is None else x_star
        Qc = self.q_cond(np.asarray(theta, dtype=np.float64), self.A @ x_star)
        D, L, Ab, T = self._factor_bta(Qc)
        bta_ref.pobtasi(D, L, Ab, T)
        return np.concatenate([np.concatenate([np.diagonal(D[i]) for i in range(self.nt)]),
                               np.diagonal(T)])


# ---------------------------------------------------------------------------
# Dense adjoint gradient (test oracle for the GPU adjoint).  For a Gaussian
# likelihood, with S_c = Q_c^{-1}, S_p = Q_st^{-1}, mu = Q_c^{-1} b:
#   df/dth_k = 1/2 tr(S_c dQ_c) - 1/2 tr(S_p dQ_st) + 1/2 mu^T dQ_c mu - mu^T db
#              - d log p(theta) - d lik(eta=0),
# with dQ obtained by the complex-step method on the restated assembly.

def _cstep(fun, theta, k, h=1e-30):
    th = np.asarray(theta, dtype=np.complex128).copy()
    th[k] += 1j * h
    return np.imag(fun(th)) / h


def _q_st_complex(model, theta):
    p = model.p
    g_s = 0.5 * math.log(8 * _NU_S) - theta[0]
    g_t = theta[1] - 0.5 * math.log(8 * _NU_T) + _ALPHA_S * g_s
    g_st = 0.5 * math.log(_C1) - 0.5 * g_t - _NU_S * g_s - theta[2]
    es, et, est = np.exp(g_s), np.exp(g_t), np.exp(g_st)
    q1 = es ** 2 * p.c0 + p.g1
    q2 = es ** 4 * p.c0 + 2 * es ** 2 * p.g1 + p.g2
    q3 = es ** 6 * p.c0 + 3 * es ** 4 * p.g1 + 3 * es ** 2 * p.g2 + p.g3
    return (est ** 2 * (sps.kron(p.m0, q3) + et * sps.kron(p.m1, q2) + et ** 2 * sps.kron(p.m2, q1))).toarray()


def _log_prior_complex(model, theta):
    s = 0.0
    for k, key in enumerate(model.theta_keys):
        al, u = model.priors[key]
        if key == "r_s":
            lam = -math.log(al) * u
            s = s + math.log(lam) - lam * np.exp(-theta[k]) - theta[k]
        elif key == "r_t":
            lam = -math.log(al) * math.sqrt(u)
            s = s + math.log(lam) - lam * np.exp(-0.5 * theta[k]) + math.log(0.5) - 0.5 * theta[k]
        else:
            lam = -math.log(al) / u
            s = s + math.log(lam) - lam * np.exp(theta[k]) + theta[k]
    return s


def dense_adjoint_gradient(model: OracleModel, theta):
    theta = np.asarray(theta, dtype=np.float64)
    assert model.gaussian
    nst = model.ns * model.nt
    tau = math.exp(theta[-1])
    Qc = model.q_cond(theta, np.zeros(len(model.y))).toarray()
    Qst = model.q_st(theta).toarray()
    Sc = np.linalg.inv(Qc)
    Sp = np.linalg.inv(Qst)
    Ad = model.A.toarray()
    b = tau * (Ad.T @ model.y)
    mu = Sc @ b
    grad = np.zeros(theta.size)
    for k in range(3):
        dQ = _cstep(lambda th: _q_st_complex(model, th), theta, k)
        dQc = np.zeros_like(Qc)
        dQc[:nst, :nst] = dQ
        grad[k] = (0.5 * np.sum(Sc * dQc) - 0.5 * np.sum(Sp * dQ) + 0.5 * mu @ dQc @ mu
                   - _cstep(lambda th: _log_prior_complex(model, th), theta, k))
    dQc = tau * (Ad.T @ Ad)
    dlik = 0.5 * len(model.y) - 0.5 * tau * (model.y @ model.y)
    grad[-1] = (0.5 * np.sum(Sc * dQc) + 0.5 * mu @ dQc @ mu - mu @ b - dlik
                - _cstep(lambda th: _log_prior_complex(model, th), theta, theta.size - 1))
    return grad


def dense_adjoint_gradient_poisson(model: OracleModel, theta):
    """Dense restatement of the GPU Poisson adjoint gradient: the Newton
    iteration of ``OracleModel.inner_iteration`` (warm started from
    ``model.x``) gives x*, eta = A x* and Q_c; dx is the final Newton update
    (not applied, as in the reference), S_c = Q_c^{-1}, S_p = Q_st^{-1},
    d = e exp(eta), z = S_c A^T (d * diag(A S_c A^T)):
      df/dth_k = 1/2 x*^T dQ x* + 1/2 tr(S_c dQ) - 1/2 tr(S_p dQ_st)
                 + (dx - z/2)^T dQ x* - d log p(theta)."""
    theta = np.asarray(theta, dtype=np.float64)
    assert not model.gaussian
    nst = model.ns * model.nt
    Qc_sp, xs, eta = model.inner_iteration(theta)
    model.x[:] = xs
    Qc = Qc_sp.toarray()
    Qp = model.q_prior(theta).toarray()
    Ad = model.A.toarray()
    rhs = -Qp @ xs + Ad.T @ model.grad_lik(theta, eta)
    dx = np.linalg.solve(Qc, rhs)
    Sc = np.linalg.inv(Qc)
    Sp = np.linalg.inv(model.q_st(theta).toarray())
    d = model.e * np.exp(eta)
    h = d * np.einsum("ij,jk,ik->i", Ad, Sc, Ad)
    z = Sc @ (Ad.T @ h)
    u = dx - 0.5 * z
    grad = np.zeros(theta.size)
    for k in range(theta.size):
        dQ = _cstep(lambda th: _q_st_complex(model, th), theta, k)
        dQc = np.zeros_like(Qc)
        dQc[:nst, :nst] = dQ
        grad[k] = (0.5 * xs @ dQc @ xs + 0.5 * np.sum(Sc * dQc) - 0.5 * np.sum(Sp * dQ) + u @ dQc @ xs
                   - _cstep(lambda th: _log_prior_complex(model, th), theta, k))
    return grad


def hessian_points(theta, eps):
    """The evaluation points of DALIA._evaluate_hessian_f in its order
    (``src/dalia/core/dalia.py:767-851``): theta, then for k = i*d + j:
    i == j -> theta +- eps e_i; i < j -> theta +eps_i +eps_j, +eps_i -eps_j,
    -eps_i +eps_j, -eps_i -eps_j.  Returns (points, combine) where
    combine(f_values) -> the Hessian (``:858-899``)."""
    theta = np.asarray(theta, dtype=np.float64)
    d = theta.size
    E = eps * np.eye(d)
    pts, keys = [theta.copy()], [("c",)]
    for k in range(d * d):
        i, j = divmod(k, d)
        if i == j:
            pts += [theta + E[i], theta - E[i]]
            keys += [("ii+", i), ("ii-", i)]
        elif i < j:
            for si, sj, tag in ((1, 1, 0), (1, -1, 1), (-1, 1, 2), (-1, -1, 3)):
                pts.append(theta + si * E[i] + sj * E[j])
                keys.append(("ij", i, j, tag))

    def combine(fv):
        f0 = fv[0]
        fii = np.zeros((2, d))
        fij = np.zeros((4, d, d))
        for key, f in zip(keys, fv):
            if key[0] == "ii+":
                fii[0, key[1]] = f
            elif key[0] == "ii-":
                fii[1, key[1]] = f
            elif key[0] == "ij":
                fij[key[3], key[1], key[2]] = f
        H = np.zeros((d, d))
        for i in range(d):
            H[i, i] = (fii[0, i] - 2 * f0 + fii[1, i]) / eps ** 2
            for j in range(i + 1, d):
                H[i, j] = H[j, i] = (fij[0, i, j] - fij[1, i, j] - fij[2, i, j] + fij[3, i, j]) / (4 * eps * eps)
        return H

    return pts, combine


def hessian_fd(evaluate_f, theta, eps=5e-3):
    """FD Hessian with f evaluated point by point in the reference's order."""
    pts, combine = hessian_points(theta, eps)
    return combine([evaluate_f(p) for p in pts])
