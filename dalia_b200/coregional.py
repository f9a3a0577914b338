"""Coregional (multivariate) spatio-temporal model on one GPU.

Host mirror of the reference's ``CoregionalModel``
(``src/dalia/models/coregional_model.py``) for 2 or 3 Gaussian variates that
share one mesh: variate k carries a DEMF(1,2,1) field Qu_k(r_s_k, r_t_k) (its
submodel's configured sigma_st, not a hyperparameter, ``spatio_temporal.py:
114-121``), nb fixed effects and a Gaussian likelihood with precision
exp(prec_o_k).  The joint prior of the fields is M^T diag(Qu_k / sigma_k^2) M
with the reference's lower-triangular mixing (``coregional_model.py:314-440``),
interleaved per time step so that a BTA block is (nv ns) x (nv ns)
(``:770-797``); the fixed effects of all variates form the arrowhead in
variate order (``:799-853``).

Every block of the joint prior is, per sub-block (v, w), a combination of
the four spatial matrices (c0, g1, g2, g3), so assembly, the adjoint's trace
terms and its quadratic forms reuse the univariate kernels' multivariate
entry points (``bta_assemble_prior_mv``, ``bta_block_inner_mv``,
``bta_block_quad_mv``); the coefficients of a sub-block are
sum_k weight_k(v, w) * (field k's coefficients), complex-safe so that the
gradient's derivatives come from the complex-step method like the
univariate model's.
"""

from __future__ import annotations

import dataclasses
import math

import numpy as np
import scipy.sparse as sps

from .model import SpatioTemporalModel, pc_log_prior


def mixing_weights(nv, theta):
    """{(v, w): [(k, weight)]} with v >= w: sub-block (v, w) of the joint
    prior is sum_k weight * Qu_k.  theta holds sigma_k (log scale) at
    3 nv + k and the lambdas after them, in the reference's key order
    lambda_0_1, lambda_0_2, lambda_1_2 and its index pattern
    (``coregional_model.py:314-330, 356-400``).  Complex-safe."""
    s2 = [np.exp(2 * theta[3 * nv + k]) for k in range(nv)]
    if nv == 2:
        l01 = theta[3 * nv + 2]
        return {(0, 0): [(0, 1 / s2[0]), (1, l01 * l01 / s2[1])],
                (1, 0): [(1, -l01 / s2[1])],
                (1, 1): [(1, 1 / s2[1])]}
    if nv == 3:
        l01, l02, l12 = theta[3 * nv + 3], theta[3 * nv + 4], theta[3 * nv + 5]
        return {(0, 0): [(0, 1 / s2[0]), (1, l01 * l01 / s2[1]), (2, l12 * l12 / s2[2])],
                (1, 0): [(1, -l01 / s2[1]), (2, l02 * l12 / s2[2])],
                (2, 0): [(2, -l12 / s2[2])],
                (1, 1): [(1, 1 / s2[1]), (2, l02 * l02 / s2[2])],
                (2, 1): [(2, -l02 / s2[2])],
                (2, 2): [(2, 1 / s2[2])]}
    raise ValueError("nv must be 2 or 3")


def latent_permutation(nt, ns, nv, nb):
    """Position in the interleaved latent vector -> index in the variate-major
    vector [v0: field (nt ns), fixed effects (nb); v1: ...]
    (``coregional_model.py:799-853``)."""
    idx = np.arange(nt * ns).reshape(nt, ns)
    st = np.hstack([idx + v * (nt * ns + nb) for v in range(nv)]).ravel()
    fe = np.concatenate([v * (nt * ns + nb) + nt * ns + np.arange(nb) for v in range(nv)])
    return np.concatenate([st, fe]).astype(np.int64)


@dataclasses.dataclass
class _JointProblem:
    """The joint problem in the univariate model's input form."""

    ns: int
    nt: int
    nb: int
    nv: int
    c0: sps.csc_matrix
    g1: sps.csc_matrix
    g2: sps.csc_matrix
    g3: sps.csc_matrix
    m0: sps.csc_matrix
    m1: sps.csc_matrix
    m2: sps.csc_matrix
    a: sps.csc_matrix
    y: np.ndarray
    var_ranges: list
    tau_idx: list
    likelihood: str = "gaussian"
    e: np.ndarray | None = None


def default_priors(prob):
    """Gaussian priors as in the reference's coregional examples: mean = the
    given theta, precision 0.5; lambdas centred at 0."""
    return {key: ("gaussian", 0.0 if key.startswith("lambda") else float(prob.theta[k]), 0.5)
            for k, key in enumerate(prob.theta_keys)}


class CoregionalModel(SpatioTemporalModel):
    """nv = 2 or 3 Gaussian spatio-temporal variates on one mesh.

    priors: {key: ("gaussian", mean, precision) | ("penalized_complexity",
    alpha, u)} for every key of ``prob.theta_keys``."""

    def __init__(self, prob, priors=None, fe_prec=1e-3, eps_gradient_f=1e-3, device=None,
                 selinv_precision="fp64", mixed_tolerance=1e-8, factor_precision="fp64", mixed_retry=16):
        nv, ns, nt, nb = int(prob.nv), int(prob.ns), int(prob.nt), int(prob.nb)
        blocks = [sps.hstack([prob.a_st[v], sps.csc_matrix(prob.a_fe[v])], format="csc") for v in range(nv)]
        A = sps.block_diag(blocks, format="csc")[:, latent_permutation(nt, ns, nv, nb)].tocsc()
        bounds = np.cumsum([0] + [len(y) for y in prob.y])
        joint = _JointProblem(ns=ns, nt=nt, nb=nv * nb, nv=nv, c0=prob.c0, g1=prob.g1, g2=prob.g2, g3=prob.g3,
                              m0=prob.m0, m1=prob.m1, m2=prob.m2, a=A,
                              y=np.concatenate([np.asarray(y, dtype=np.float64) for y in prob.y]),
                              var_ranges=[(int(bounds[v]), int(bounds[v + 1])) for v in range(nv)],
                              tau_idx=[3 * v + 2 for v in range(nv)])
        self.coreg = prob
        self.sigma_st = np.asarray(prob.sigma_st, dtype=np.float64)
        super().__init__(joint, priors={}, fe_prec=fe_prec, eps_gradient_f=eps_gradient_f, device=device,
                         selinv_precision=selinv_precision, mixed_tolerance=mixed_tolerance,
                         factor_precision=factor_precision, mixed_retry=mixed_retry)
        self.theta_keys = list(prob.theta_keys)
        self.priors = default_priors(prob) if priors is None else dict(priors)
        missing = [k for k in self.theta_keys if k not in self.priors]
        if missing:
            raise ValueError(f"no prior for {missing}")

    def coef_blocks(self, theta):
        """(2n-1) x (nv nv 4): coefficients of (c0, g1, g2, g3) of sub-block
        (v, w) of every lower BTA block.  Complex-safe."""
        nv = self.nv
        fields = [self._coef_field(theta[3 * k], theta[3 * k + 1], self.sigma_st[k]) for k in range(nv)]
        cplx = any(np.iscomplexobj(f) for f in fields)
        out = np.zeros((2 * self.nt - 1, nv, nv, 4), dtype=np.complex128 if cplx else np.float64)
        for (v, w), terms in mixing_weights(nv, theta).items():
            c = sum(wt * fields[k] for k, wt in terms)
            out[:, v, w] = c
            out[:, w, v] = c
        return out.reshape(2 * self.nt - 1, nv * nv * 4)

    def log_prior_theta(self, theta):
        """Sum of the hyperparameter priors (``coregional_model.py:666-676``):
        Gaussian ``-0.5 precision (theta - mean)^2``
        (``src/dalia/prior_hyperparameters/gaussian.py:26-29``) or penalised
        complexity.  Complex-safe."""
        s = 0.0
        for k, key in enumerate(self.theta_keys):
            spec = self.priors[key]
            if spec[0] == "gaussian":
                s = s - 0.5 * spec[2] * (theta[k] - spec[1]) ** 2
            else:
                kind = key.rsplit("_", 1)[0]
                s = s + pc_log_prior("sigma_st" if kind == "sigma" else kind, theta[k], spec[1], spec[2])
        return s
