"""Seeded synthetic spatio-temporal INLA problems.

The reference's example datasets (``examples/gst_*``, ``examples/pst_small``)
are not available, so every workload here is generated from a seed with the
shapes and value distributions of the reference's examples:

* spatial mesh: ``ns`` nodes on a jittered ``ceil(sqrt(ns))^2`` grid in the unit
  square, Delaunay-triangulated; P1 finite elements give the lumped mass ``c0``
  (diagonal), the stiffness ``g1`` and ``g2 = g1 c0^-1 g1``, ``g3 = g1 c0^-1 g2``
  (both explicitly symmetrised, because the reference asserts
  ``|M - M^T| < 1e-10`` in ``src/dalia/submodels/spatio_temporal.py:91-112``);
* time: ``nt`` steps at unit spacing with the 1D FEM matrices ``m0`` (lumped
  mass), ``m1`` (boundary term, stored already multiplied by 2 so that the
  reference's ``kron(m1, q2)`` (``spatio_temporal.py:140-147``) equals the
  DEMF(1,2,1) term ``2 gamma_t M1 (x) q2``) and ``m2`` (1D stiffness);
* observations: ``no`` points per time step, uniform in ``[0.05, 0.95]^2``;
  ``A`` = barycentric interpolation (3 nnz per row) in the time-major latent
  ordering ``t*ns + s`` plus ``nb`` dense N(0,1) covariate columns appended last
  (the fixed effects form the arrowhead, ``src/dalia/core/model.py:49-53,541-560``);
* responses: Gaussian ``y = A x + eps / sqrt(tau_y)`` or Poisson
  ``y ~ Poisson(exp(A x))`` for a smooth random latent field ``x``.
"""

from __future__ import annotations

import dataclasses
import math

import numpy as np
import scipy.sparse as sps
from scipy.spatial import Delaunay


@dataclasses.dataclass
class SpatioTemporalProblem:
    """One synthetic spatio-temporal problem in the reference's data layout."""

    ns: int
    nt: int
    nb: int
    no: int
    c0: sps.csc_matrix
    g1: sps.csc_matrix
    g2: sps.csc_matrix
    g3: sps.csc_matrix
    m0: sps.csc_matrix
    m1: sps.csc_matrix
    m2: sps.csc_matrix
    a_st: sps.csc_matrix  # (no*nt) x (ns*nt) barycentric part
    a_fe: np.ndarray  # (no*nt) x nb dense covariates
    y: np.ndarray
    theta: np.ndarray  # (r_s, r_t, sigma_st[, prec_o])
    likelihood: str  # "gaussian" | "poisson"
    e: np.ndarray | None = None  # Poisson exposure (ones)
    # geometry of the observations (needed by the on-device assembly)
    obs_nodes: np.ndarray | None = None  # (no*nt, 3) spatial node ids
    obs_weights: np.ndarray | None = None  # (no*nt, 3) barycentric weights

    @property
    def n_latent(self) -> int:
        return self.ns * self.nt + self.nb

    @property
    def a(self) -> sps.csc_matrix:
        """Full design matrix ``[A_st | X]`` in the reference's latent order."""
        return sps.hstack([self.a_st, sps.csc_matrix(self.a_fe)], format="csc")


def _mesh(ns: int, rng: np.random.Generator):
    # k x k jittered grid spanning the unit square (boundary nodes stay on the
    # boundary so the mesh covers the observation window); the ns - k^2
    # remaining nodes are placed uniformly in the interior.
    k = int(math.floor(math.sqrt(ns)))
    g = np.linspace(0.0, 1.0, k)
    xx, yy = np.meshgrid(g, g, indexing="xy")
    pts = np.stack([xx.ravel(), yy.ravel()], axis=1)
    jit = 0.3 / k
    interior = (pts[:, 0] > 0) & (pts[:, 0] < 1) & (pts[:, 1] > 0) & (pts[:, 1] < 1)
    pts[interior] += rng.uniform(-jit, jit, size=(int(interior.sum()), 2))
    extra = ns - k * k
    if extra > 0:
        pts = np.concatenate([pts, rng.uniform(0.02, 0.98, size=(extra, 2))])
    tri = Delaunay(pts)
    return pts, tri


def _fem(pts: np.ndarray, simplices: np.ndarray):
    ns = pts.shape[0]
    p0 = pts[simplices[:, 0]]
    p1 = pts[simplices[:, 1]]
    p2 = pts[simplices[:, 2]]
    # signed area -> absolute
    area = 0.5 * np.abs(
        (p1[:, 0] - p0[:, 0]) * (p2[:, 1] - p0[:, 1])
        - (p2[:, 0] - p0[:, 0]) * (p1[:, 1] - p0[:, 1])
    )
    keep = area > 1e-14
    simplices, area = simplices[keep], area[keep]
    p = [pts[simplices[:, i]] for i in range(3)]
    # edge opposite vertex i
    e = [p[(i + 2) % 3] - p[(i + 1) % 3] for i in range(3)]
    rows, cols, vals = [], [], []
    for i in range(3):
        for j in range(3):
            rows.append(simplices[:, i])
            cols.append(simplices[:, j])
            vals.append((e[i] * e[j]).sum(axis=1) / (4.0 * area))
    g1 = sps.coo_matrix(
        (np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
        shape=(ns, ns),
    ).tocsc()
    g1 = 0.5 * (g1 + g1.T)
    c0d = np.zeros(ns)
    for i in range(3):
        np.add.at(c0d, simplices[:, i], area / 3.0)
    c0 = sps.diags(c0d).tocsc()
    c0inv = sps.diags(1.0 / c0d).tocsc()
    g2 = g1 @ c0inv @ g1
    g2 = (0.5 * (g2 + g2.T)).tocsc()
    g3 = g1 @ c0inv @ g2
    g3 = (0.5 * (g3 + g3.T)).tocsc()
    for m in (g1, g2, g3):
        m.sort_indices()
    return c0, g1, g2, g3


def _time_fem(nt: int):
    if nt < 2:
        raise ValueError("nt must be >= 2 for the 1D temporal FEM matrices")
    d0 = np.ones(nt)
    d0[0] = d0[-1] = 0.5
    m0 = sps.diags(d0).tocsc()
    d1 = np.zeros(nt)
    d1[0] = d1[-1] = 1.0  # 2 * diag(1/2, 0, ..., 0, 1/2)
    m1 = sps.diags(d1).tocsc()
    d2 = 2.0 * np.ones(nt)
    d2[0] = d2[-1] = 1.0
    off = -np.ones(nt - 1)
    m2 = sps.diags([off, d2, off], [-1, 0, 1]).tocsc()
    return m0, m1, m2


def _barycentric(tri: Delaunay, pts_obs: np.ndarray):
    simp = tri.find_simplex(pts_obs)
    if np.any(simp < 0):
        raise RuntimeError("observation outside the mesh")
    T = tri.transform[simp]
    bary2 = np.einsum("nij,nj->ni", T[:, :2, :], pts_obs - T[:, 2, :])
    w = np.concatenate([bary2, 1.0 - bary2.sum(axis=1, keepdims=True)], axis=1)
    nodes = tri.simplices[simp]
    return nodes, w


def make_problem(
    ns: int,
    nt: int,
    nb: int,
    no: int,
    theta,
    likelihood: str = "gaussian",
    seed: int = 0,
    log_intensity_scale: float = 1.0,
) -> SpatioTemporalProblem:
    """Generate one seeded synthetic problem (see the module docstring).
    ``log_intensity_scale`` multiplies the linear predictor of Poisson
    responses (lower counts keep the reference's undamped Newton iteration,
    started from x = 0, from overshooting on large meshes)."""
    rng = np.random.default_rng(seed)
    pts, tri = _mesh(ns, rng)
    c0, g1, g2, g3 = _fem(pts, tri.simplices)
    m0, m1, m2 = _time_fem(nt)

    nobs = no * nt
    obs_xy = rng.uniform(0.05, 0.95, size=(nobs, 2))
    nodes, w = _barycentric(tri, obs_xy)
    t_of = np.repeat(np.arange(nt), no)
    rows = np.repeat(np.arange(nobs), 3)
    cols = (t_of[:, None] * ns + nodes).ravel()
    a_st = sps.coo_matrix((w.ravel(), (rows, cols)), shape=(nobs, ns * nt)).tocsc()
    a_st.sum_duplicates()
    a_fe = rng.standard_normal((nobs, nb))

    # smooth latent field: random Fourier modes in space, AR(1) in time
    n_modes = 6
    kx = rng.uniform(0.5, 3.0, size=n_modes) * np.pi
    ky = rng.uniform(0.5, 3.0, size=n_modes) * np.pi
    ph = rng.uniform(0, 2 * np.pi, size=n_modes)
    basis = np.cos(kx[None, :] * pts[:, :1] + ky[None, :] * pts[:, 1:2] + ph[None, :])
    coef = np.zeros((nt, n_modes))
    coef[0] = rng.standard_normal(n_modes)
    for t in range(1, nt):
        coef[t] = 0.9 * coef[t - 1] + math.sqrt(1 - 0.81) * rng.standard_normal(n_modes)
    x_st = (coef @ basis.T).ravel() * 0.5
    beta = rng.standard_normal(nb) * 0.3
    eta = a_st @ x_st + a_fe @ beta

    theta = np.asarray(theta, dtype=np.float64)
    e = None
    if likelihood == "gaussian":
        tau = math.exp(theta[-1])
        y = eta + rng.standard_normal(nobs) / math.sqrt(tau)
    elif likelihood == "poisson":
        y = rng.poisson(np.exp(log_intensity_scale * eta)).astype(np.float64)
        e = np.ones(nobs)
    else:
        raise ValueError(f"unknown likelihood {likelihood}")

    return SpatioTemporalProblem(
        ns=ns, nt=nt, nb=nb, no=no,
        c0=c0, g1=g1, g2=g2, g3=g3, m0=m0, m1=m1, m2=m2,
        a_st=a_st, a_fe=a_fe, y=y, theta=theta, likelihood=likelihood, e=e,
        obs_nodes=nodes.astype(np.int64), obs_weights=w,
    )


@dataclasses.dataclass
class CoregionalProblem:
    """nv spatio-temporal variates on one mesh (the reference's
    ``CoregionalModel``, ``src/dalia/models/coregional_model.py``), each with
    its own observations, nb fixed effects and Gaussian likelihood.

    theta follows the reference's order: per variate (r_s, r_t, prec_o),
    then sigma_0..sigma_{nv-1}, then lambda_i_j for i < j."""

    ns: int
    nt: int
    nv: int
    nb: int  # fixed effects per variate
    c0: sps.csc_matrix
    g1: sps.csc_matrix
    g2: sps.csc_matrix
    g3: sps.csc_matrix
    m0: sps.csc_matrix
    m1: sps.csc_matrix
    m2: sps.csc_matrix
    a_st: list  # per variate (no_v*nt) x (ns*nt)
    a_fe: list  # per variate (no_v*nt) x nb
    y: list
    theta: np.ndarray
    sigma_st: np.ndarray  # fixed per-variate sigma_st of the submodels (not a hyperparameter)

    @property
    def theta_keys(self):
        keys = []
        for v in range(self.nv):
            keys += [f"r_s_{v}", f"r_t_{v}", f"prec_o_{v}"]
        keys += [f"sigma_{v}" for v in range(self.nv)]
        keys += [f"lambda_{i}_{j}" for i in range(self.nv) for j in range(i + 1, self.nv)]
        return keys


def make_coregional_problem(ns, nt, nv, nb, no, theta, seed=0):
    """Seeded synthetic coregional problem: one mesh and temporal FEM shared
    by the variates, no observations per time step and variate, responses
    y_v = A_v x_v + X_v beta_v + noise with x = mixtures of smooth fields."""
    if nv not in (2, 3):
        raise ValueError("nv must be 2 or 3")
    rng = np.random.default_rng(seed)
    pts, tri = _mesh(ns, rng)
    c0, g1, g2, g3 = _fem(pts, tri.simplices)
    m0, m1, m2 = _time_fem(nt)
    theta = np.asarray(theta, dtype=np.float64)
    a_st, a_fe, ys = [], [], []
    # smooth fields u_k, mixed lower-triangularly into the variates
    n_modes = 6
    fields = []
    for _ in range(nv):
        kx = rng.uniform(0.5, 3.0, size=n_modes) * np.pi
        ky = rng.uniform(0.5, 3.0, size=n_modes) * np.pi
        ph = rng.uniform(0, 2 * np.pi, size=n_modes)
        basis = np.cos(kx[None, :] * pts[:, :1] + ky[None, :] * pts[:, 1:2] + ph[None, :])
        coef = np.zeros((nt, n_modes))
        coef[0] = rng.standard_normal(n_modes)
        for t in range(1, nt):
            coef[t] = 0.9 * coef[t - 1] + math.sqrt(1 - 0.81) * rng.standard_normal(n_modes)
        fields.append((coef @ basis.T).ravel() * 0.5)
    for v in range(nv):
        x_v = sum((0.5 ** (v - k)) * fields[k] for k in range(v + 1))
        nobs = no * nt
        obs_xy = rng.uniform(0.05, 0.95, size=(nobs, 2))
        nodes, w = _barycentric(tri, obs_xy)
        t_of = np.repeat(np.arange(nt), no)
        rows = np.repeat(np.arange(nobs), 3)
        cols = (t_of[:, None] * ns + nodes).ravel()
        A = sps.coo_matrix((w.ravel(), (rows, cols)), shape=(nobs, ns * nt)).tocsc()
        A.sum_duplicates()
        X = rng.standard_normal((nobs, nb))
        beta = rng.standard_normal(nb) * 0.3
        tau = math.exp(theta[3 * v + 2])
        ys.append(A @ x_v + X @ beta + rng.standard_normal(nobs) / math.sqrt(tau))
        a_st.append(A)
        a_fe.append(X)
    return CoregionalProblem(ns=ns, nt=nt, nv=nv, nb=nb, c0=c0, g1=g1, g2=g2, g3=g3, m0=m0, m1=m1, m2=m2,
                             a_st=a_st, a_fe=a_fe, y=ys, theta=theta, sigma_st=np.zeros(nv))


def save_coregional_layout(prob: CoregionalProblem, root) -> None:
    """One reference model directory per variate (``model_<v+1>/inputs_*``,
    the layout of the reference's coregional examples) plus y per variate."""
    import os

    for v in range(prob.nv):
        st = os.path.join(root, f"model_{v + 1}", "inputs_spatio_temporal")
        rg = os.path.join(root, f"model_{v + 1}", "inputs_regression")
        os.makedirs(st, exist_ok=True)
        os.makedirs(rg, exist_ok=True)
        for nm in ("c0", "g1", "g2", "g3", "m0", "m1", "m2"):
            sps.save_npz(os.path.join(st, f"{nm}.npz"), getattr(prob, nm).tocsc())
        sps.save_npz(os.path.join(st, "a.npz"), prob.a_st[v].tocsc())
        sps.save_npz(os.path.join(rg, "a.npz"), sps.csc_matrix(prob.a_fe[v]))
        np.save(os.path.join(root, f"model_{v + 1}", "y.npy"), prob.y[v])


# Workloads with the reference examples' shapes (seed 0 each).
CONFIGS = {
    "gst_300x10": dict(ns=300, nt=10, nb=4, no=200, theta=(-1.0, 1.0, 0.0, 2.0), likelihood="gaussian"),
    "gst_1500x100": dict(ns=1500, nt=100, nb=6, no=600, theta=(-1.0, 1.0, 0.0, 2.0), likelihood="gaussian"),
    # same model on 20 time steps: a mid-size case (BTA factor 0.7 GB) for profiling
    "gst_1500x20": dict(ns=1500, nt=20, nb=6, no=600, theta=(-1.0, 1.0, 0.0, 2.0), likelihood="gaussian"),
    "pst_2500x60": dict(ns=2500, nt=60, nb=6, no=800, theta=(-1.2, 0.8, -0.3), likelihood="poisson",
                        log_intensity_scale=0.4),
    "gst_4000x250": dict(ns=4000, nt=250, nb=6, no=1500, theta=(-1.0, 1.0, 0.0, 2.0), likelihood="gaussian"),
    # the univariate members of the mixed-size batch (blocks 600 x 600, one fixed effect)
    "gst_600x40": dict(ns=600, nt=40, nb=1, no=200, theta=(-1.0, 1.0, 0.0, 2.0), likelihood="gaussian"),
}


# Coregional workloads: theta = per variate (r_s, r_t, prec_o), sigmas, lambdas.
COREG_CONFIGS = {
    "gst_coreg3_600x40": dict(ns=600, nt=40, nv=3, nb=1, no=200,
                              theta=(-1.0, 1.0, 2.0, -0.8, 0.9, 1.8, -1.2, 1.1, 2.2,
                                     0.0, 0.2, -0.1, 0.5, -0.3, 0.4)),
    "gst_coreg2_600x40": dict(ns=600, nt=40, nv=2, nb=1, no=200,
                              theta=(-1.0, 1.0, 2.0, -0.8, 0.9, 1.8, 0.0, 0.2, 0.5)),
}


# A batch of instances of uneven block sizes evaluated in shared launches:
# (workload, theta points) per member -- 8 bivariate (blocks 1200 x 1200) and
# 16 univariate (600 x 600) points on the same mesh size.
MIXED_BATCHES = {
    "mixed_8x1200_16x600": [("gst_coreg2_600x40", 8), ("gst_600x40", 16)],
}


def make_config(name: str, seed: int = 0):
    if name in COREG_CONFIGS:
        return make_coregional_problem(seed=seed, **COREG_CONFIGS[name])
    return make_problem(seed=seed, **CONFIGS[name])


def save_dalia_layout(prob: SpatioTemporalProblem, root) -> None:
    """Write ``prob`` in the reference's on-disk layout
    (``src/dalia/submodels/spatio_temporal.py:26-35``,
    ``src/dalia/core/submodel.py:23-41``, ``src/dalia/core/model.py:239-250``)."""
    import os

    st = os.path.join(root, "inputs_spatio_temporal")
    rg = os.path.join(root, "inputs_regression")
    os.makedirs(st, exist_ok=True)
    os.makedirs(rg, exist_ok=True)
    for nm in ("c0", "g1", "g2", "g3", "m0", "m1", "m2"):
        sps.save_npz(os.path.join(st, f"{nm}.npz"), getattr(prob, nm).tocsc())
    sps.save_npz(os.path.join(st, "a.npz"), prob.a_st.tocsc())
    sps.save_npz(os.path.join(rg, "a.npz"), sps.csc_matrix(prob.a_fe))
    np.save(os.path.join(root, "y.npy"), prob.y)
    if prob.e is not None:
        np.save(os.path.join(root, "e.npy"), prob.e)
