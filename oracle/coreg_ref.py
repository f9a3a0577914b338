"""CPU oracle: the reference's coregional (multivariate) spatio-temporal model
restated with SciPy sparse matrices and the BTA oracle.

TEST INFRASTRUCTURE ONLY (see ``oracle/bta_ref.py``): imported by the tests,
``__graft_entry__.smoke()`` and the benchmark's CPU baseline, never by the
product path.

Restated reference behaviour, with citations (``src/dalia/models/coregional_model.py``):

* theta: per variate the submodel and likelihood hyperparameters with the
  ``sigma_*`` keys removed (r_s, r_t, prec_o), then ``sigma_0..``, then
  ``lambda_i_j`` (``:104-147``; ``src/dalia/configs/models_config.py:62-71``);
  the submodels keep their configured sigma_st (``spatio_temporal.py:114-121``)
* q_vw from Qu_k / sigma_k^2 and the lambdas, including the reference's own
  lambda index pattern (``:314-440``)
* the spatio-temporal block permuted to per-time-step interleaving of the
  variates (``:770-797``), fixed effects last in variate order, and the
  design matrix block-diagonal over variates with its columns permuted the
  same way (``:217-251, 799-853``)
* Q_conditional = Q_prior + A^T D A with D = tau_v on variate v's rows
  (``:553-620``); Gaussian priors ``-0.5 precision (theta - mean)^2``
  (``src/dalia/prior_hyperparameters/gaussian.py:26-29``)
* f(theta) and its central-difference gradient follow the univariate oracle
  (``oracle/model_ref.py``), Serinv path (prior log-determinant without the tip).
"""

from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sps

from . import bta_ref
from .model_ref import _ALPHA_S, _C1, _NU_S, _NU_T, pc_log_prior


def default_priors(prob):
    """Gaussian priors as in the reference's coregional examples
    (``examples/gst_coreg3_small/run.py``): mean = the generating value,
    precision 0.5; lambdas centred at 0."""
    pri = {}
    for k, key in enumerate(prob.theta_keys):
        mean = 0.0 if key.startswith("lambda") else float(prob.theta[k])
        pri[key] = ("gaussian", mean, 0.5)
    return pri


def log_prior(priors, keys, theta):
    s = 0.0
    for k, key in enumerate(keys):
        spec = priors[key]
        if spec[0] == "gaussian":
            s = s - 0.5 * spec[2] * (theta[k] - spec[1]) ** 2
        else:
            kind = key.rsplit("_", 1)[0]
            s = s + pc_log_prior(kind, theta[k], spec[1], spec[2])
    return s


def _q_st(prob, r_s, r_t, sigma_st):
    g_s = 0.5 * math.log(8 * _NU_S) - r_s
    g_t = r_t - 0.5 * math.log(8 * _NU_T) + _ALPHA_S * g_s
    g_st = 0.5 * math.log(_C1) - 0.5 * g_t - _NU_S * g_s - sigma_st
    es, et, est = np.exp(g_s), np.exp(g_t), np.exp(g_st)
    q1 = es ** 2 * prob.c0 + prob.g1
    q2 = es ** 4 * prob.c0 + 2 * es ** 2 * prob.g1 + prob.g2
    q3 = es ** 6 * prob.c0 + 3 * es ** 4 * prob.g1 + 3 * es ** 2 * prob.g2 + prob.g3
    return est ** 2 * (sps.kron(prob.m0, q3) + et * sps.kron(prob.m1, q2) + et ** 2 * sps.kron(prob.m2, q1))


def mixing_blocks(nv, theta):
    """[(v, w, [(k, weight)])]: q_vw = sum_k weight * Qu_k, the reference's
    formulas (``coregional_model.py:314-440``); complex-safe."""
    s = [np.exp(theta[3 * nv + v]) for v in range(nv)]
    if nv == 2:
        l01 = theta[3 * nv + 2]
        return {(0, 0): [(0, 1 / s[0] ** 2), (1, l01 ** 2 / s[1] ** 2)],
                (1, 0): [(1, -l01 / s[1] ** 2)],
                (1, 1): [(1, 1 / s[1] ** 2)]}
    l01, l02, l12 = theta[3 * nv + 3], theta[3 * nv + 4], theta[3 * nv + 5]
    return {(0, 0): [(0, 1 / s[0] ** 2), (1, l01 ** 2 / s[1] ** 2), (2, l12 ** 2 / s[2] ** 2)],
            (1, 0): [(1, -l01 / s[1] ** 2), (2, l02 * l12 / s[2] ** 2)],
            (2, 0): [(2, -l12 / s[2] ** 2)],
            (1, 1): [(1, 1 / s[1] ** 2), (2, l02 ** 2 / s[2] ** 2)],
            (2, 1): [(2, -l02 / s[2] ** 2)],
            (2, 2): [(2, 1 / s[2] ** 2)]}


def perm_st(nt, ns, nv):
    """New position -> model-major index of the spatio-temporal unknowns."""
    idx = np.arange(nt * ns).reshape(nt, ns)
    return np.hstack([idx + v * nt * ns for v in range(nv)]).ravel()


def perm_latent(nt, ns, nv, nb):
    """New position -> index in the model-major latent vector
    [v0: st, fe; v1: st, fe; ...]."""
    idx = np.arange(nt * ns).reshape(nt, ns)
    st = np.hstack([idx + v * (nt * ns + nb) for v in range(nv)]).ravel()
    fe = np.concatenate([v * (nt * ns + nb) + nt * ns + np.arange(nb) for v in range(nv)])
    return np.concatenate([st, fe]).astype(np.int64)


class CoregionalOracle:
    def __init__(self, prob, priors=None, fe_prec=1e-3, eps_gradient_f=1e-3):
        self.p = prob
        self.nv, self.ns, self.nt, self.nbv = prob.nv, prob.ns, prob.nt, prob.nb
        self.b = self.nv * self.ns
        self.a = self.nv * self.nbv
        self.N = self.nt * self.b + self.a
        self.keys = prob.theta_keys
        self.priors = default_priors(prob) if priors is None else priors
        self.fe_prec = fe_prec
        self.eps = eps_gradient_f
        blocks = [sps.hstack([prob.a_st[v], sps.csc_matrix(prob.a_fe[v])], format="csc") for v in range(self.nv)]
        A_mm = sps.block_diag(blocks, format="csc")
        self.A = A_mm[:, perm_latent(self.nt, self.ns, self.nv, self.nbv)].tocsr()
        self.AT = self.A.T.tocsr()
        self.y = np.concatenate(prob.y)
        self.nobs = [len(y) for y in prob.y]
        self.obs_var = np.repeat(np.arange(self.nv), self.nobs)
        self.x = np.zeros(self.N)
        self.pst = perm_st(self.nt, self.ns, self.nv)

    def q_re(self, theta, dense=False):
        """Permuted multivariate spatio-temporal prior (nt*nv*ns square)."""
        nv = self.nv
        Qu = [_q_st(self.p, theta[3 * v], theta[3 * v + 1], self.p.sigma_st[v]) for v in range(nv)]
        mix = mixing_blocks(nv, theta)
        rows = []
        for v in range(nv):
            row = []
            for w in range(nv):
                key = (v, w) if v >= w else (w, v)
                q = sum(wt * Qu[k] for k, wt in mix[key])
                row.append(q if v >= w else q.T)
            rows.append(row)
        Q = sps.bmat(rows, format="csc")
        Q = Q[self.pst, :][:, self.pst]
        return Q.toarray() if dense else Q.tocsc()

    def q_prior(self, theta):
        return sps.block_diag([self.q_re(theta), self.fe_prec * sps.eye(self.a)], format="csc")

    def taus(self, theta):
        return np.array([math.exp(theta[3 * v + 2]) for v in range(self.nv)])

    def q_cond(self, theta):
        d = self.taus(theta)[self.obs_var]
        return (self.q_prior(theta) + self.AT @ sps.diags(d) @ self.A).tocsc()

    def lik0(self, theta):
        s = 0.0
        for v, y in enumerate(self.p.y):
            s += 0.5 * theta[3 * v + 2] * len(y) - 0.5 * math.exp(theta[3 * v + 2]) * float(y @ y)
        return s

    def evaluate_f(self, theta):
        theta = np.asarray(theta, dtype=np.float64)
        Qc = self.q_cond(theta)
        D, L, Ab, T = bta_ref.sparse_to_bta(Qc, self.nt, self.b, self.a)
        bta_ref.pobtaf(D, L, Ab, T)
        rhs = self.AT @ (self.taus(theta)[self.obs_var] * self.y)
        mu = rhs.copy()
        bta_ref.pobtas(D, L, Ab, T, mu, "N")
        bta_ref.pobtas(D, L, Ab, T, mu, "C")
        self.x[:] = mu
        cond = 0.5 * bta_ref.logdet(D, T, "bta") - 0.5 * mu @ (Qc @ mu)
        Dp, Lp, _, _ = bta_ref.sparse_to_bta(self.q_re(theta), self.nt, self.b, 0)
        bta_ref.pobtf(Dp, Lp)
        ld_p = bta_ref.logdet(Dp, None, "bt")
        f = cond - (log_prior(self.priors, self.keys, theta) + self.lik0(theta) + 0.5 * ld_p)
        return float(f)

    def objective(self, theta):
        theta = np.asarray(theta, dtype=np.float64)
        d = theta.size
        nf = 2 * d + 1
        tm = np.repeat(theta.reshape(-1, 1), nf, axis=1)
        tm[:, 1:1 + d] += self.eps * np.eye(d)
        tm[:, d + 1:nf] -= self.eps * np.eye(d)
        fv = np.zeros(nf)
        for k in range(nf - 1, -1, -1):
            fv[k] = self.evaluate_f(tm[:, k])
        return fv[0], (fv[1:1 + d] - fv[d + 1:nf]) / (2 * self.eps)


def dense_adjoint_gradient(orc: CoregionalOracle, theta):
    """Dense adjoint gradient of the coregional Gaussian objective:
    prior hyperparameters through dQ_re (complex step on the dense prior),
    tau_v through 1/2 tau_v tr(S_c A_v^T A_v) + 1/2 tau_v |A_v mu|^2
    - tau_v (A_v mu)^T y_v - d lik0."""
    theta = np.asarray(theta, dtype=np.float64)
    nst = orc.nt * orc.b
    Qc = orc.q_cond(theta).toarray()
    Sc = np.linalg.inv(Qc)
    Sp = np.linalg.inv(orc.q_re(theta, dense=True))
    Ad = orc.A.toarray()
    tau_obs = orc.taus(theta)[orc.obs_var]
    mu = Sc @ (Ad.T @ (tau_obs * orc.y))
    eta = Ad @ mu
    grad = np.zeros(theta.size)
    h = 1e-30
    for k in range(theta.size):
        if k < 3 * orc.nv and k % 3 == 2:
            v = k // 3
            rows = orc.obs_var == v
            tau = math.exp(theta[k])
            Av = Ad[rows]
            grad[k] = (0.5 * tau * np.sum(Sc * (Av.T @ Av)) + 0.5 * tau * eta[rows] @ eta[rows]
                       - tau * eta[rows] @ orc.y[rows]
                       - (0.5 * rows.sum() - 0.5 * tau * orc.y[rows] @ orc.y[rows]))
        else:
            th = theta.astype(np.complex128)
            th[k] += 1j * h
            dQ = np.imag(orc.q_re(th, dense=True)) / h
            grad[k] = 0.5 * np.sum(Sc[:nst, :nst] * dQ) - 0.5 * np.sum(Sp * dQ) + 0.5 * mu[:nst] @ dQ @ mu[:nst]
        th = theta.astype(np.complex128)
        th[k] += 1j * h
        grad[k] -= float(np.imag(log_prior(orc.priors, orc.keys, th)) / h)
    return grad
