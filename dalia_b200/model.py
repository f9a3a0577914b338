"""Spatio-temporal INLA model evaluated on the GPU: theta -> BTA precision
matrices -> f(theta) and its gradient.

Host mirror of the reference's model classes for this path:

* ``SpatioTemporalSubModel.construct_Q_prior`` and ``_interpretable2compute``
  (``src/dalia/submodels/spatio_temporal.py:114-197``), plane manifold;
* ``RegressionSubModel`` (``src/dalia/submodels/regression.py:27-35``);
* ``Model.construct_Q_prior / construct_Q_conditional /
  construct_information_vector`` (``src/dalia/core/model.py:306-449``);
* ``GaussianLikelihood`` / ``PoissonLikelihood``
  (``src/dalia/likelihoods/gaussian.py:19-131``, ``poisson.py:31-63``);
* penalised-complexity priors
  (``src/dalia/prior_hyperparameters/penalized_complexity.py:28-82``);
* ``DALIA._evaluate_f`` and ``_objective_function``
  (``src/dalia/core/dalia.py:513-745``), Serinv solver semantics (the prior
  log-determinant comes from the BT factorisation of the spatio-temporal block,
  so the fixed-effect tip is excluded, ``structured_solver.py:151-166``).

Everything per theta runs on the device through the C ABI
(``include/dalia_bta.h``, ``include/dalia_assemble.h``); the host only forms
O(nt) scalar coefficients and reads back a few scalars.  Derivatives of the
scalar coefficients use the complex-step method (all coefficient functions
are complex-analytic), so they carry no truncation error.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np
import scipy.sparse as sps
import scipy.special as ssp

from . import _lib

# alpha_s = 2, alpha_t = 1, alpha_e = 1 (spatio_temporal.py:157-166)
_ALPHA_S, _ALPHA_T, _ALPHA_E = 2, 1, 1
_ALPHA = _ALPHA_E + _ALPHA_S * (_ALPHA_T - 0.5)
_NU_S = _ALPHA - 1
_NU_T = _ALPHA_T - 0.5
_LOG_C1 = math.log(
    ssp.gamma(_NU_T) * ssp.gamma(_NU_S)
    / (ssp.gamma(_ALPHA_T) * ssp.gamma(_ALPHA) * pow(4 * math.pi, 1.5)))

DEFAULT_PRIORS = {
    "r_s": (0.01, 0.5),
    "r_t": (0.01, 5.0),
    "sigma_st": (0.01, 3.0),
    "prec_o": (0.01, 4.0),
}

_CSTEP = 1e-30  # complex-step size


def theta_to_gamma(r_s, r_t, sigma_st):
    """(r_s, r_t, sigma_st) -> (gamma_s, gamma_t, gamma_st), plane manifold
    (``spatio_temporal.py:168-193``); complex-safe."""
    g_s = 0.5 * math.log(8 * _NU_S) - r_s
    g_t = r_t - 0.5 * math.log(8 * _NU_T) + _ALPHA_S * g_s
    g_st = 0.5 * _LOG_C1 - 0.5 * g_t - _NU_S * g_s - sigma_st
    return g_s, g_t, g_st


def pc_log_prior(kind, theta, alpha, u):
    """Penalised-complexity log-priors (``penalized_complexity.py:55-82``);
    complex-safe."""
    if kind == "r_s":
        lam = -math.log(alpha) * u  # spatial dimension 2: u^(d/2) = u
        return math.log(lam) - lam * np.exp(-theta) - theta
    if kind == "r_t":
        lam = -math.log(alpha) * math.sqrt(u)
        return math.log(lam) - lam * np.exp(-0.5 * theta) + math.log(0.5) - 0.5 * theta
    if kind in ("sigma_st", "sigma_e", "prec_o"):
        lam = -math.log(alpha) / u
        return math.log(lam) - lam * np.exp(theta) + theta
    raise ValueError(kind)


def _tridiag(m, nt):
    m = sps.csr_matrix(m).toarray()
    if m.shape != (nt, nt) or np.any(np.triu(m, 2)) or np.any(np.tril(m, -2)):
        raise ValueError("temporal FEM matrices must be tridiagonal (nt x nt)")
    return np.diagonal(m).copy(), np.diagonal(m, -1).copy()


def _pairs_per_row(A):
    """All (first, second) nnz position pairs that share a row of CSR A."""
    counts = np.diff(A.indptr)
    row_of_p = np.repeat(np.arange(A.shape[0]), counts)
    k_p = counts[row_of_p]
    first = np.repeat(np.arange(A.nnz), k_p)
    start = np.repeat(np.cumsum(k_p) - k_p, k_p)
    j = np.arange(first.size) - start
    second = A.indptr[row_of_p[first]] + j
    return first, second, row_of_p


def factor_flops(n, b, a):
    """Algorithmic flops of one BTA factorisation (pobtaf): per block column
    POTRF b^3/3, TRSM of the block below b^3 and of the arrow a b^2, the
    previous column's Schur update b^3 (SYRK, lower half), 2 a b^2 (arrow)
    and a^2 b (tip); plus the tip POTRF a^3/3."""
    f = n * (b ** 3 / 3 + a * b ** 2 + a * a * b) + (n - 1) * (b ** 3 + b ** 3 + 2 * a * b ** 2)
    return f + a ** 3 / 3


def selinv_gemm_flops(n, b, a):
    """Flops of the GEMMs of one selected inversion (pobtasi), per block
    column: G = L Linv (b^3), S_{i+1,i} = -S G (2 b^3), S_ii (b^3/3 + b^3),
    and the arrow terms."""
    return (n - 1) * (4 * b ** 3 + 6 * a * b ** 2) + n * (b ** 3 / 3 + 4 * a * b ** 2 + 4 * a * a * b)


_PRECISIONS = {"fp64": _lib.BTA_PREC_FP64, "tf32x3": _lib.BTA_PREC_TF32X3, "i8slice": _lib.BTA_PREC_I8SLICE}

# Smallest block size at which the factorisation's Schur updates as 8-bit-slice
# GEMMs beat the FP64 updates inside the panel kernel (measured on B200: faster
# at b = 1500 and 1800, slower for a batch of b = 1200 and 600 blocks).
AUTO_I8_FACTOR_MIN_BLOCK = 1500


def _factor_arith(requested, models, precision):
    """Arithmetic of the Schur updates of a forward evaluation: FP64 whenever
    the selected inversion is FP64 (a fully FP64 evaluation, e.g. the
    fallback), else the model's choice, "auto" resolved by block size."""
    if precision == "fp64" or requested == "fp64":
        return "fp64"
    if requested == "auto":
        return "i8slice" if min(m.b for m in models) >= AUTO_I8_FACTOR_MIN_BLOCK else "fp64"
    return requested


class BTAMatrix:
    """One BTA matrix in a single device allocation with D, L, Ab, T views."""

    def __init__(self, n, b, a, device):
        import torch

        self.n, self.b, self.a = n, b, a
        nD, nL, nA, nT = n * b * b, max(n - 1, 0) * b * b, n * a * b, a * a
        self.offL, self.offA, self.offT = nD, nD + nL, nD + nL + nA
        self.buf = torch.zeros(nD + nL + nA + nT, dtype=torch.float64, device=device)
        self.D = self.buf[:nD].view(n, b, b)
        self.L = self.buf[nD:nD + nL].view(max(n - 1, 0), b, b)
        self.Ab = self.buf[nD + nL:nD + nL + nA].view(n, a, b)
        self.T = self.buf[nD + nL + nA:].view(a, a)

    def ptrs(self):
        P = _lib.ptr
        L = self.L if self.n > 1 else None
        if self.a > 0:
            return P(self.D), P(L), P(self.Ab), P(self.T)
        return P(self.D), P(L), P(None), P(None)


class _Slot:
    """Device state of one theta point: the two BTA matrices, vectors and
    read-back scalars (one per point of a batched evaluation)."""

    def __init__(self, n, b, a, N, nobs, device, Qc=None, Qp=None, nv=1):
        import torch

        f64 = dict(dtype=torch.float64, device=device)
        self.Qc = Qc if Qc is not None else BTAMatrix(n, b, a, device)
        self.Qp = Qp if Qp is not None else BTAMatrix(n, b, 0, device)
        self.rhs = torch.zeros(N, **f64)
        self.x = torch.zeros(N, **f64)  # latent mean / mode, like the reference's model.x
        self.eta = torch.zeros(nobs, **f64)
        self.scal = torch.zeros(16, **f64)
        nb4 = (2 * n - 1) * 4 * nv * nv  # [block][v][w][K]
        self.vscal = torch.zeros(3 * nv, **f64)  # per variate: tr(S A_v^T A_v), |A_v mu|^2, (A_v mu)^T y_v
        self.inner_c = torch.zeros(nb4, **f64)
        self.inner_p = torch.zeros(nb4, **f64)
        self.quad_st = torch.zeros(nb4, **f64)
        self.bil = torch.zeros(nb4, **f64)
        # Newton inner iteration state (non-Gaussian likelihoods)
        self.upd = torch.zeros(N, **f64)  # last Newton update
        self.qpx = torch.zeros(N, **f64)  # Q_prior x
        self.z = torch.zeros(N, **f64)
        self.dvec = torch.zeros(nobs, **f64)  # e exp(eta)
        self.gvec = torch.zeros(nobs, **f64)  # y - e exp(eta)
        self.hvec = torch.zeros(nobs, **f64)
        self.Sc = None  # copy of Q_c's factor, selected-inverted (allocated on first use)
        self.Vc = None  # inverses of the diagonal factor blocks of Q_c (allocated on first use)
        # one pinned host buffer per assembly so that queued copies never race
        self.coef_host = [torch.zeros(nb4, dtype=torch.float64).pin_memory() for _ in range(2)]
        self.coef_dev = [torch.zeros(nb4, **f64) for _ in range(2)]


class SpatioTemporalModel:
    """DEMF(1,2,1) spatio-temporal field + fixed effects, Gaussian or Poisson
    likelihood, evaluated on one GPU."""

    def __init__(self, prob, priors=None, fe_prec=1e-3, eps_gradient_f=1e-3, eps_inner_iteration=1e-3,
                 inner_iteration_max_iter=50, device=None, selinv_precision="fp64", mixed_tolerance=1e-8,
                 factor_precision="fp64", mixed_retry=16):
        """selinv_precision: arithmetic of the selected inversions behind the
        adjoint gradient: "fp64", "tf32x3" (FP32-class block products on the
        tcgen05 tensor cores) or "i8slice" (8-bit digit products accumulated
        exactly in INT32 on the tensor cores, ~1e-10 relative).
        factor_precision: arithmetic of the factorisations' previous-column
        Schur updates in a reduced-precision adjoint evaluation ("fp64",
        "i8slice", or "auto": 8-bit slices when every block of the batch is at
        least AUTO_I8_FACTOR_MIN_BLOCK wide, where they measured faster than the
        FP64 updates fused into the panel kernel; the diagonal-block POTRF,
        the triangular solves, the log-determinants and the sweeps stay FP64,
        and the plain f / FD paths always factor in FP64).  Every adjoint
        evaluation checks its selected
        inverses through the identity <S, Q> = dim(Q) over the BTA pattern; a
        reduced-precision point whose relative residual exceeds
        mixed_tolerance is recomputed entirely in FP64.  After such a
        recomputation in an evaluation at the model's own precision, the next
        mixed_retry evaluations at the model's precision run in FP64 directly
        (the check failing again would cost the reduced-precision pass each
        time); then the reduced precision is tried again.  An explicit
        ``precision=`` argument is always honoured.  The residuals of the last
        evaluation are in ``last_check`` (``demoted`` marks points run in FP64
        by this rule)."""
        import torch

        if selinv_precision not in _PRECISIONS:
            raise ValueError(f"selinv_precision must be one of {sorted(_PRECISIONS)}")
        if factor_precision not in ("fp64", "i8slice", "auto"):
            raise ValueError("factor_precision must be 'fp64', 'i8slice' or 'auto'")
        self.selinv_precision = selinv_precision
        self.factor_precision = factor_precision
        self.mixed_tol = float(mixed_tolerance)
        self.mixed_retry = int(mixed_retry)
        self._demote_left = 0
        self.last_check = []

        self.h = _lib.handle(device)
        self.device = self.h.device
        self.lib = _lib.load()
        dev = self.device
        self.ns, self.nt, self.nb = int(prob.ns), int(prob.nt), int(prob.nb)
        # nv variates interleaved per time step (1: univariate): block size nv ns
        self.nv = int(getattr(prob, "nv", 1))
        self.b = self.nv * self.ns
        n, b, a, ns = self.nt, self.b, self.nb, self.ns
        self.N = n * b + a
        self.gaussian = prob.likelihood == "gaussian"
        if self.nv > 1 and not self.gaussian:
            raise NotImplementedError("multivariate models: Gaussian likelihoods only")
        self.priors = dict(DEFAULT_PRIORS if priors is None else priors)
        self.theta_keys = ["r_s", "r_t", "sigma_st"] + (["prec_o"] if self.gaussian else [])
        self.fe_prec = float(fe_prec)
        self.eps = float(eps_gradient_f)
        self.eps_inner = float(eps_inner_iteration)
        self.max_inner = int(inner_iteration_max_iter)

        # --- union pattern of c0, g1, g2, g3 with four values per entry
        U = (abs(prob.c0) + abs(prob.g1) + abs(prob.g2) + abs(prob.g3)).tocsr()
        U.sort_indices()
        rows = np.repeat(np.arange(ns), np.diff(U.indptr))
        cols = U.indices
        vals4 = np.stack([np.asarray(sps.csr_matrix(K)[rows, cols]).ravel()
                          for K in (prob.c0, prob.g1, prob.g2, prob.g3)], axis=1)
        i32 = dict(dtype=torch.int32, device=dev)
        f64 = dict(dtype=torch.float64, device=dev)
        i64 = dict(dtype=torch.int64, device=dev)
        self.u_rowptr = torch.tensor(U.indptr, **i32)
        self.u_col = torch.tensor(cols, **i32)
        self.u_vals4 = torch.tensor(np.ascontiguousarray(vals4), **f64)
        self.m_diag = [_tridiag(m, n)[0] for m in (prob.m0, prob.m1, prob.m2)]
        self.m_sub = [_tridiag(m, n)[1] for m in (prob.m0, prob.m1, prob.m2)]

        # --- design matrix, responses
        A = prob.a.tocsr()
        A.sort_indices()
        self.A_host = A
        self.nobs = A.shape[0]
        self.y_host = np.asarray(prob.y, dtype=np.float64)
        self.e_host = np.ones(self.nobs) if prob.e is None else np.asarray(prob.e, dtype=np.float64)
        self.A_rowptr = torch.tensor(A.indptr.astype(np.int64), **i64)
        self.A_col = torch.tensor(A.indices.astype(np.int32), **i32)
        self.A_val = torch.tensor(A.data, **f64)
        AT = A.T.tocsr()
        AT.sort_indices()
        self.AT_rowptr = torch.tensor(AT.indptr.astype(np.int64), **i64)
        self.AT_col = torch.tensor(AT.indices.astype(np.int32), **i32)
        self.AT_val = torch.tensor(AT.data, **f64)
        self.y = torch.tensor(self.y_host, **f64)
        self.e = torch.tensor(self.e_host, **f64)
        X = A[:, n * b:].toarray() if a > 0 else np.zeros((self.nobs, 0))
        self.X = torch.tensor(np.ascontiguousarray(X), **f64)
        # observation ranges of the variates, and the theta index of each
        # variate's Gaussian precision
        self.var_ranges = list(getattr(prob, "var_ranges", [(0, self.nobs)]))
        self.tau_idx = list(getattr(prob, "tau_idx", [len(self.theta_keys) - 1] if self.gaussian else []))
        self.XtX_var = [X[lo:hi].T @ X[lo:hi] for lo, hi in self.var_ranges]
        self.yty_var = [float(self.y_host[lo:hi] @ self.y_host[lo:hi]) for lo, hi in self.var_ranges]
        self.nobs_var = [hi - lo for lo, hi in self.var_ranges]
        Aty = []
        for lo, hi in self.var_ranges:
            yv = np.zeros(self.nobs)
            yv[lo:hi] = self.y_host[lo:hi]
            Aty.append(torch.tensor(A.T @ yv, **f64))
        self.Aty_var = Aty

        # --- A^T D A entry lists on the BTA pattern (tip handled separately)
        self.Qc = BTAMatrix(n, b, a, dev)
        self.Qp = BTAMatrix(n, b, 0, dev)
        self._dev = dev
        first, second, row_of_p = _pairs_per_row(A)
        # 64-bit positions: a BTA array of 250 blocks of 4000 x 4000 has 4e9 entries
        c1, c2 = A.indices[first].astype(np.int64), A.indices[second].astype(np.int64)
        fac = A.data[first] * A.data[second]
        obs = row_of_p[first]
        nbt = n * b
        bi, bj = c1 // b, c2 // b
        inD = (c1 < nbt) & (c2 < nbt) & (bi == bj)
        inL = (c1 < nbt) & (c2 < nbt) & (bi == bj + 1)
        inA = (c1 >= nbt) & (c2 < nbt)
        bad = (c1 < nbt) & (c2 < nbt) & (np.abs(bi - bj) > 1)
        if np.any(bad):
            raise ValueError("design matrix couples latent blocks more than one time step apart")
        dst = np.full(c1.shape, -1, dtype=np.int64)
        dst[inD] = (bi[inD] * b + c1[inD] % b) * b + c2[inD] % b
        dst[inL] = self.Qc.offL + (bj[inL] * b + c1[inL] % b) * b + c2[inL] % b
        dst[inA] = self.Qc.offA + ((c2[inA] // b) * a + (c1[inA] - nbt)) * b + c2[inA] % b
        keep = dst >= 0
        dst, obs, fac = dst[keep], obs[keep], fac[keep]
        kindmult = np.where(inD[keep], 1.0, 2.0)
        # the same pairs grouped by observation (weights doubled for L and Ab
        # entries): a_i^T S a_i per row of A, i.e. diag(A S A^T)
        o_order = np.argsort(obs, kind="stable")
        self.obs_off = torch.tensor(np.searchsorted(obs[o_order], np.arange(self.nobs + 1)).astype(np.int64), **i64)
        self.obs_dst = torch.tensor(dst[o_order], **i64)
        self.obs_w = torch.tensor((fac * kindmult)[o_order], **f64)
        order = np.argsort(dst, kind="stable")
        dst, obs, fac, kindmult = dst[order], obs[order], fac[order], kindmult[order]
        ud, start = np.unique(dst, return_index=True)
        off = np.append(start, dst.size).astype(np.int64)
        self.ent_dst = torch.tensor(ud, **i64)
        self.ent_off = torch.tensor(off, **i64)
        self.ent_obs = torch.tensor(obs.astype(np.int32), **i32)
        self.ent_fac = torch.tensor(fac, **f64)
        self.nent = int(ud.size)
        # trace weights of A_v^T A_v on the stored entries, per variate (lower
        # blocks count twice)
        self.ata_w_var = []
        for lo, hi in self.var_ranges:
            fv = np.where((obs >= lo) & (obs < hi), fac, 0.0)
            sumfac = np.add.reduceat(fv, start) if fv.size else np.zeros(0)
            self.ata_w_var.append(torch.tensor(sumfac * kindmult[start], **f64))

        # --- scratch
        self.nparts = 148
        self.part = torch.zeros(4096, **f64)
        self.dvec = torch.zeros(self.nobs, **f64)
        self.ones_obs = torch.ones(self.nobs, **f64)
        self.slots = [self._new_slot(self.Qc, self.Qp)]
        # algorithmic flops of the factorisations / selected-inversion GEMMs
        # issued so far, and Newton steps taken (non-Gaussian likelihoods)
        # (factor_schur: the part of "factor" applied by GEMMs outside the panel
        # kernel when the Schur updates run in reduced precision)
        self.work = {"factor": 0.0, "factor_schur": 0.0, "selinv_gemm": 0.0, "newton_steps": 0}

    def _new_slot(self, Qc=None, Qp=None):
        return _Slot(self.nt, self.b, self.nb, self.N, self.nobs, self._dev, Qc, Qp, self.nv)

    def slot(self, j):
        while len(self.slots) <= j:
            self.slots.append(self._new_slot())
        return self.slots[j]

    # slot 0 carries the state of single-point evaluations (model.x, ...)
    x = property(lambda self: self.slots[0].x)
    rhs = property(lambda self: self.slots[0].rhs)
    eta = property(lambda self: self.slots[0].eta)
    scal = property(lambda self: self.slots[0].scal)

    # ------------------------------------------------------------------ host
    def coef_blocks(self, theta):
        """Coefficients of (c0, g1, g2, g3) for every lower BTA block of Q_st;
        rows 0..n-1 diagonal blocks, rows n..2n-2 sub-diagonal blocks.
        Complex-safe."""
        return self._coef_field(theta[0], theta[1], theta[2])

    def _coef_field(self, r_s, r_t, sigma_st):
        """Kronecker coefficients of one DEMF(1,2,1) field, (2n-1) x 4."""
        g_s, g_t, g_st = theta_to_gamma(r_s, r_t, sigma_st)
        k2 = np.exp(2 * g_s)
        E = np.exp(2 * g_st)
        u = np.exp(g_t)
        m0 = np.concatenate([self.m_diag[0], self.m_sub[0]])
        m1 = np.concatenate([self.m_diag[1], self.m_sub[1]])
        m2 = np.concatenate([self.m_diag[2], self.m_sub[2]])
        # q1 = k2 c0 + g1; q2 = k2^2 c0 + 2 k2 g1 + g2; q3 = k2^3 c0 + 3 k2^2 g1 + 3 k2 g2 + g3
        c_c0 = E * (m0 * k2 ** 3 + u * m1 * k2 ** 2 + u * u * m2 * k2)
        c_g1 = E * (3 * m0 * k2 ** 2 + 2 * u * m1 * k2 + u * u * m2)
        c_g2 = E * (3 * m0 * k2 + u * m1)
        c_g3 = E * m0
        return np.stack([c_c0, c_g1, c_g2, c_g3], axis=1)

    def log_prior_theta(self, theta):
        s = 0.0
        for k, key in enumerate(self.theta_keys):
            al, u = self.priors[key]
            s = s + pc_log_prior(key, theta[k], al, u)
        return s

    def lik0(self, theta):
        """Gaussian log-likelihood at eta = 0 (``gaussian.py:55-62``), summed
        over the variates."""
        s = 0.0
        for k, nv_obs, yty in zip(self.tau_idx, self.nobs_var, self.yty_var):
            s = s + 0.5 * theta[k] * nv_obs - 0.5 * np.exp(theta[k]) * yty
        return s

    def _gauss_conditional(self, theta, sl):
        """Q_c of a Gaussian likelihood: one precision scales A^T A, several
        (one per variate) fill sl.dvec observation range by range."""
        if len(self.tau_idx) == 1:
            self.assemble_conditional(theta, None, math.exp(theta[self.tau_idx[0]]), sl)
            return
        s = self._stream()
        for k, (lo, hi) in zip(self.tau_idx, self.var_ranges):
            self._check(self.lib.bta_axpby(s, hi - lo, math.exp(theta[k]), _lib.ptr(self.ones_obs[lo:hi]), 0.0,
                                           _lib.ptr(sl.dvec[lo:hi])), "axpby")
        self.assemble_conditional(theta, sl.dvec, 1.0, sl)

    def _gauss_rhs(self, theta, sl):
        """Information vector at x = 0, eta = 0: sum_v tau_v A_v^T y_v."""
        s = self._stream()
        for j, k in enumerate(self.tau_idx):
            self._check(self.lib.bta_axpby(s, self.N, math.exp(theta[k]), _lib.ptr(self.Aty_var[j]),
                                           1.0 if j else 0.0, _lib.ptr(sl.rhs)), "axpby")

    # ---------------------------------------------------------------- device
    def _stream(self):
        return _lib.stream_ptr(self.device)

    def _check(self, rc, what):
        _lib.check(rc, what)

    def _assemble_prior(self, theta, M: BTAMatrix, sl, which):
        c = np.asarray(self.coef_blocks(theta), dtype=np.float64).ravel()
        sl.coef_host[which].numpy()[:] = c
        sl.coef_dev[which].copy_(sl.coef_host[which], non_blocking=True)
        D, L, _, _ = M.ptrs()
        self._check(self.lib.bta_assemble_prior_mv(self._stream(), M.n, self.ns, self.nv, _lib.ptr(sl.coef_dev[which]),
                                                   _lib.ptr(self.u_rowptr), _lib.ptr(self.u_col),
                                                   _lib.ptr(self.u_vals4), D, L), "assemble_prior")

    def assemble_conditional(self, theta, d=None, dscale=1.0, sl=None):
        """Q_c = Q_prior + A^T diag(dscale * d) A in BTA storage (``model.py:384-423``);
        d None means the Gaussian constant diagonal."""
        sl = self.slots[0] if sl is None else sl
        Q = sl.Qc
        self._assemble_prior(theta, Q, sl, 0)
        if Q.a > 0:
            Q.Ab.zero_()
        dptr = _lib.ptr(d)
        self._check(self.lib.bta_add_entries(self._stream(), self.nent, _lib.ptr(self.ent_dst),
                                             _lib.ptr(self.ent_off), _lib.ptr(self.ent_obs), _lib.ptr(self.ent_fac),
                                             dptr, float(dscale), _lib.ptr(Q.buf)), "add_entries")
        if Q.a > 0:
            self._check(self.lib.bta_arrow_tip(self._stream(), self.nobs, Q.a, _lib.ptr(self.X), dptr,
                                               self.fe_prec, float(dscale), _lib.ptr(self.part), self.nparts,
                                               _lib.ptr(Q.T)), "arrow_tip")

    def assemble_prior_bt(self, theta, sl=None):
        sl = self.slots[0] if sl is None else sl
        self._assemble_prior(theta, sl.Qp, sl, 1)

    def factor(self, M: BTAMatrix):
        self.work["factor"] += factor_flops(M.n, M.b, M.a)
        D, L, Ab, T = M.ptrs()
        self._check(self.lib.bta_pobtaf(self.h.bind_stream(), M.n, M.b, M.a, D, L, Ab, T, None), "pobtaf")

    def _batched_args(self, mats):
        k = len(mats)
        i64 = ctypes.c_int64 * k
        ptrs = ctypes.c_void_p * k
        n = i64(*[m.n for m in mats])
        b = i64(*[m.b for m in mats])
        a = i64(*[m.a for m in mats])
        P = [m.ptrs() for m in mats]
        D = ptrs(*[p[0].value for p in P])
        L = ptrs(*[p[1].value for p in P])
        Ab = ptrs(*[p[2].value for p in P])
        T = ptrs(*[p[3].value for p in P])
        return k, n, b, a, D, L, Ab, T

    def factor_batched(self, mats, precision="fp64"):
        """All matrices factored together, block column by block column;
        precision: arithmetic of the previous-column Schur updates."""
        self.work["factor"] += sum(factor_flops(m.n, m.b, m.a) for m in mats)
        if precision != "fp64":
            self.work["factor_schur"] += sum((m.n - 1) * (m.b ** 3 + 2 * m.a * m.b ** 2) for m in mats)
        k, n, b, a, D, L, Ab, T = self._batched_args(mats)
        self._check(self.lib.bta_pobtaf_batched_ex(self.h.bind_stream(), k, n, b, a, D, L, Ab, T, None,
                                                   _PRECISIONS[precision]), "pobtaf_batched")

    def selinv_batched(self, mats, precision="fp64", Vs=None):
        """Selected inversions of all matrices together; Vs (optional, entries
        may be None) supplies the inverses of their diagonal factor blocks,
        which the library otherwise computes chunk by chunk."""
        self.work["selinv_gemm"] += sum(selinv_gemm_flops(m.n, m.b, m.a) for m in mats)
        k, n, b, a, D, L, Ab, T = self._batched_args(mats)
        V = None if Vs is None else (ctypes.c_void_p * k)(*[None if v is None else v.data_ptr() for v in Vs])
        self._check(self.lib.bta_pobtasi_batched_v(self.h.bind_stream(), k, n, b, a, D, L, Ab, T, V,
                                                   _PRECISIONS[precision]), "pobtasi_batched")

    def block_inverses(self, mats, Vs):
        """V = inverses of the diagonal factor blocks of every matrix."""
        k, n, b, a, D, L, Ab, T = self._batched_args(mats)
        V = (ctypes.c_void_p * k)(*[v.data_ptr() for v in Vs])
        self._check(self.lib.bta_block_inverses(self.h.bind_stream(), k, n, b, D, V), "block_inverses")

    def sweep_inv_batched(self, mats, Vs, xs, trans):
        """Triangular sweeps through the block inverses (n dependent steps)."""
        k, n, b, a, D, L, Ab, T = self._batched_args(mats)
        V = (ctypes.c_void_p * k)(*[v.data_ptr() for v in Vs])
        X = (ctypes.c_void_p * k)(*[x.data_ptr() for x in xs])
        self._check(self.lib.bta_pobtas_inv_batched(self.h.bind_stream(), k, n, b, a, L, Ab, T, V, X, trans),
                    "pobtas_inv_batched")

    def _slot_inverses(self, sl):
        """Inverses of Q_c's diagonal factor blocks (n b^2 doubles), kept for
        the triangular sweeps and the selected inversion.  Q_prior needs no
        sweep: its selected inversion computes its block inverses chunk by
        chunk, so they never occupy n b^2 at once."""
        import torch

        if sl.Vc is None:
            sl.Vc = torch.empty(self.nt * self.b * self.b, dtype=torch.float64, device=self.device)
        return sl.Vc

    def logdet_to(self, M: BTAMatrix, out):
        D, _, _, T = M.ptrs()
        self._check(self.lib.bta_logdet(self.h.bind_stream(), M.n, M.b, M.a, D, T, 1 if M.a else 0, _lib.ptr(out),
                                        None), "logdet")

    def _inverses_fit(self, sls):
        """Whether the slots' Q_c block inverses are (or can be made)
        resident: n b^2 doubles per slot, kept for later use."""
        import torch

        missing = sum(1 for sl in sls if sl.Vc is None)
        if missing == 0:
            return True
        free, _ = torch.cuda.mem_get_info(self.device)
        return missing * self.nt * self.b * self.b * 8 + (4 << 30) < free

    def solve_in_place(self, sls, xs):
        """x <- Q_c^{-1} x for the factored Q_c of every slot: both triangular
        sweeps through the inverses of the diagonal factor blocks (computed
        once for both sweeps) when they fit in memory and the batch is small,
        else the library's sweep (which picks its own method)."""
        mats = [sl.Qc for sl in sls]
        if len(sls) <= 2 and self._inverses_fit(sls):
            Vs = [self._slot_inverses(sl) for sl in sls]
            self.block_inverses(mats, Vs)
            self.sweep_inv_batched(mats, Vs, xs, 0)
            self.sweep_inv_batched(mats, Vs, xs, 1)
        else:
            self.sweep_batched(mats, xs, 0)
            self.sweep_batched(mats, xs, 1)

    def sweep(self, M: BTAMatrix, x, trans):
        D, L, Ab, T = M.ptrs()
        self._check(self.lib.bta_pobtas(self.h.bind_stream(), M.n, M.b, M.a, D, L, Ab, T, _lib.ptr(x), trans),
                    "pobtas")

    def selinv(self, M: BTAMatrix):
        self.work["selinv_gemm"] += selinv_gemm_flops(M.n, M.b, M.a)
        D, L, Ab, T = M.ptrs()
        self._check(self.lib.bta_pobtasi(self.h.bind_stream(), M.n, M.b, M.a, D, L, Ab, T), "pobtasi")

    def dot_to(self, x, y, out):
        self._check(self.lib.bta_dot(self._stream(), x.numel(), _lib.ptr(x), _lib.ptr(y), _lib.ptr(self.part),
                                     self.nparts, _lib.ptr(out)), "dot")

    def sweep_batched(self, mats, xs, trans):
        k, n, b, a, D, L, Ab, T = self._batched_args(mats)
        X = (ctypes.c_void_p * k)(*[x.data_ptr() for x in xs])
        self._check(self.lib.bta_pobtas_batched(self.h.bind_stream(), k, n, b, a, D, L, Ab, T, X, trans),
                    "pobtas_batched")

    def spmv(self, rowptr, col, val, m, x, y, alpha=1.0, beta=0.0):
        self._check(self.lib.bta_csr_spmv(self._stream(), m, _lib.ptr(rowptr), _lib.ptr(col), _lib.ptr(val),
                                          _lib.ptr(x), float(alpha), float(beta), _lib.ptr(y)), "spmv")

    def status(self):
        info = ctypes.c_int64(0)
        rc = self.lib.bta_get_status(self.h.bind_stream(), ctypes.byref(info))
        if rc == _lib.BTA_ERR_NOT_SPD:
            raise np.linalg.LinAlgError(f"precision matrix not positive definite (pivot {info.value})")
        _lib.check(rc, "status")

    # ------------------------------------------------------------ objective
    def evaluate_f(self, theta):
        """f(theta) following ``DALIA._evaluate_f`` (``dalia.py:603-745``)."""
        theta = np.asarray(theta, dtype=np.float64)
        _lib.check(self.lib.bta_reset_status(self.h.bind_stream()), "reset")
        if self.gaussian:
            sl = self.slots[0]
            self._gauss_conditional(theta, sl)
            self.factor(sl.Qc)
            self.logdet_to(sl.Qc, sl.scal[0:1])
            # rhs = -Q_prior x + A^T grad(lik) at x = 0, eta = 0  ->  sum_v tau_v A_v^T y_v
            self._gauss_rhs(theta, sl)
            sl.x.copy_(sl.rhs)
            self.solve_in_place([sl], [sl.x])
            self.dot_to(sl.rhs, sl.x, sl.scal[1:2])  # mu^T Q_c mu = b^T mu
            self.assemble_prior_bt(theta, sl)
            self.factor(sl.Qp)
            self.logdet_to(sl.Qp, sl.scal[2:3])
            self.status()
            s = sl.scal[:3].cpu().numpy()
            cond = 0.5 * s[0] - 0.5 * s[1]
            f = cond - (self.log_prior_theta(theta) + self.lik0(theta) + 0.5 * s[2])
        else:
            f = self._evaluate_f_poisson(theta)
        if np.isnan(f):
            raise ValueError("f(theta) is NaN. Check what is happening.")
        return float(f)

    def objective_fd(self, theta):
        """(f, central finite-difference gradient): the reference's
        ``_objective_function`` (``dalia.py:513-601``), evaluated point by point
        in reverse order."""
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

    def evaluate_f_batched(self, thetas):
        """f at K theta points with all 2K factorisations (Q_c and Q_prior of
        every point) in one batched launch sequence (Gaussian likelihoods,
        whose evaluations carry no state from point to point).  model.x ends
        as the latent mean of the first point."""
        if not self.gaussian:
            raise NotImplementedError("batched f: Gaussian likelihoods (the Newton iteration is warm-started "
                                      "from point to point)")
        thetas = [np.asarray(t, dtype=np.float64) for t in thetas]
        sls = [self.slot(j) for j in range(len(thetas))]
        _lib.check(self.lib.bta_reset_status(self.h.bind_stream()), "reset")
        for sl, th in zip(sls, thetas):
            self._gauss_conditional(th, sl)
            self.assemble_prior_bt(th, sl)
        self.factor_batched([sl.Qc for sl in sls] + [sl.Qp for sl in sls])
        for sl, th in zip(sls, thetas):
            self.logdet_to(sl.Qc, sl.scal[0:1])
            self.logdet_to(sl.Qp, sl.scal[2:3])
            self._gauss_rhs(th, sl)
            sl.x.copy_(sl.rhs)
        self.sweep_batched([sl.Qc for sl in sls], [sl.x for sl in sls], 0)
        for sl in sls:
            self.dot_to(sl.x, sl.x, sl.scal[1:2])  # b^T Q_c^-1 b = mu^T Q_c mu
        self.sweep(sls[0].Qc, sls[0].x, 1)
        self.status()
        fs = []
        for sl, th in zip(sls, thetas):
            v = sl.scal[:3].cpu().numpy()
            f = 0.5 * v[0] - 0.5 * v[1] - (self.log_prior_theta(th) + self.lik0(th) + 0.5 * v[2])
            if np.isnan(f):
                raise ValueError("f(theta) is NaN. Check what is happening.")
            fs.append(float(f))
        return fs

    def points_that_fit(self, want, reserve_bytes=6 << 30):
        """How many theta points (of ``want``) can keep their device state --
        Q_c, Q_prior and their vectors -- at once: the slots that exist plus
        those the free device memory holds beyond ``reserve_bytes`` of
        library workspace."""
        import torch

        have = len(self.slots)
        if want <= have:
            return want
        free, _ = torch.cuda.mem_get_info(self.device)
        per = (self.Qc.buf.numel() + self.Qp.buf.numel() + 8 * self.N + 4 * self.nobs) * 8
        return int(max(1, min(want, have + max(0, free - reserve_bytes) // per)))

    def objective_fd_batched(self, theta, max_points=None):
        """The reference's central-difference objective (``dalia.py:513-601``)
        with the 2d+1 stencil points evaluated in batches of up to
        max_points (Gaussian likelihoods; default: as many as device memory
        holds, all 2d+1 when they fit -- one batched factorisation of the
        2(2d+1) matrices); the same values as ``objective_fd``."""
        theta = np.asarray(theta, dtype=np.float64)
        d = theta.size
        nf = 2 * d + 1
        if max_points is None:
            max_points = self.points_that_fit(min(nf, 32))
        tm = np.repeat(theta.reshape(-1, 1), nf, axis=1)
        tm[:, 1:1 + d] += self.eps * np.eye(d)
        tm[:, d + 1:nf] -= self.eps * np.eye(d)
        fv = np.zeros(nf)
        # the centre goes last and first in its batch, so that model.x is its latent mean
        order = list(range(1, nf)) + [0]
        for c0 in range(0, nf, max_points):
            idx = order[c0:c0 + max_points]
            if 0 in idx:
                idx = [0] + [i for i in idx if i != 0]
            fv[idx] = self.evaluate_f_batched([tm[:, i] for i in idx])
        return fv[0], (fv[1:1 + d] - fv[d + 1:nf]) / (2 * self.eps)

    def hessian_fd(self, theta, eps_hessian_f=5e-3, max_points=None):
        """Finite-difference Hessian of f (``DALIA._evaluate_hessian_f``,
        ``dalia.py:767-910``): f at theta, at theta +- eps e_i and at
        theta +- eps e_i +- eps e_j (i < j), 1 + 2d + 2d(d-1) points.  Gaussian
        likelihoods evaluate the points in batches of max_points; a Poisson
        likelihood evaluates them one by one in the reference's order, because
        each Newton iteration starts from the previous point's mode."""
        theta = np.asarray(theta, dtype=np.float64)
        d = theta.size
        h = float(eps_hessian_f)
        E = h * np.eye(d)
        pts = [theta.copy()]
        slot_of = {}
        for k in range(d * d):
            i, j = divmod(k, d)
            if i == j:
                slot_of[("+", i)] = len(pts)
                pts.append(theta + E[i])
                slot_of[("-", i)] = len(pts)
                pts.append(theta - E[i])
            elif i < j:
                for si, sj in ((1, 1), (1, -1), (-1, 1), (-1, -1)):
                    slot_of[(i, j, si, sj)] = len(pts)
                    pts.append(theta + si * E[i] + sj * E[j])
        if self.gaussian:
            if max_points is None:
                max_points = self.points_that_fit(min(len(pts), 32))
            fv = []
            for c0 in range(0, len(pts), max_points):
                fv += self.evaluate_f_batched(pts[c0:c0 + max_points])
        else:
            fv = [self.evaluate_f(p) for p in pts]
        H = np.zeros((d, d))
        for i in range(d):
            H[i, i] = (fv[slot_of[("+", i)]] - 2 * fv[0] + fv[slot_of[("-", i)]]) / h ** 2
            for j in range(i + 1, d):
                H[i, j] = H[j, i] = (fv[slot_of[(i, j, 1, 1)]] - fv[slot_of[(i, j, 1, -1)]]
                                     - fv[slot_of[(i, j, -1, 1)]] + fv[slot_of[(i, j, -1, -1)]]) / (4 * h * h)
        return H

    def covariance_theta(self, theta, eps_hessian_f=5e-3):
        """Covariance of the hyperparameters, the inverse of the FD Hessian
        (``DALIA.compute_covariance_hp``, ``dalia.py:747-765``)."""
        return np.linalg.inv(self.hessian_fd(theta, eps_hessian_f))

    def _dcoef(self, theta, k):
        th = np.asarray(theta, dtype=np.complex128).copy()
        th[k] += 1j * _CSTEP
        return np.imag(self.coef_blocks(th)) / _CSTEP

    def _dfun(self, fun, theta, k):
        th = np.asarray(theta, dtype=np.complex128).copy()
        th[k] += 1j * _CSTEP
        return float(np.imag(fun(th)) / _CSTEP)

    def objective_adjoint(self, theta):
        """(f, exact gradient) at one theta, see ``objective_adjoint_batched``."""
        f, g = self.objective_adjoint_batched([theta])
        return f[0], g[0]

    def _identity_residuals(self, theta, Ic, Ip, rest_c, tip_c):
        """Relative residuals of <S_c, Q_c> = N and <S_p, Q_st> = n b: the
        spatio-temporal parts from the block inner products with the
        Kronecker factors, rest_c = <S_c, A^T D A> and tip_c = <T(S_c), prior
        tip>."""
        mult = np.ones((2 * self.nt - 1, 1))
        mult[self.nt:] = 2.0
        cf = np.asarray(self.coef_blocks(theta), dtype=np.float64) * mult
        nst = self.nt * self.b
        rc = abs(float(np.sum(cf * Ic)) + rest_c + tip_c - self.N) / self.N
        rp = abs(float(np.sum(cf * Ip)) - nst) / nst
        return rc, rp

    def _mixed_fallback(self, thetas, fs, grads, precision, tok=None):
        """Recompute in FP64 the points whose selected-inverse check missed
        (and, for an evaluation at the model's own precision, run the next
        mixed_retry such evaluations in FP64 directly)."""
        demoted = bool(tok and tok.get("demoted"))
        if demoted:
            self.last_check = [dict(c, demoted=True) for c in self.last_check]
        if precision == "fp64":
            return fs, grads
        bad = [j for j, c in enumerate(self.last_check) if max(c["residual_c"], c["residual_p"]) > self.mixed_tol]
        if not bad:
            return fs, grads
        if tok is not None and tok.get("default"):
            self._demote_left = self.mixed_retry
        checks = list(self.last_check)
        f2, g2 = self.objective_adjoint_batched([thetas[j] for j in bad], precision="fp64")
        for j, f, g, c in zip(bad, f2, g2, self.last_check):
            fs[j], grads[j] = f, g
            # the reduced-precision residuals that triggered the recomputation stay reported
            checks[j] = dict(checks[j], fallback=True, fp64_residual_c=c["residual_c"],
                             fp64_residual_p=c["residual_p"])
        self.last_check = checks
        return fs, grads

    def objective_adjoint_batched(self, thetas, precision=None):
        """(f, exact gradient) at K theta points (e.g. the candidates of a line
        search), factorising and selected-inverting all 2K matrices (Q_c and
        Q_prior of every point) together:
        df/dth = 1/2 tr(S_c dQ_c) - 1/2 tr(S_p dQ_st) + 1/2 mu^T dQ_c mu
                 - mu^T db - d log p(theta) - d lik0,
        with tr(S dQ_st) and mu^T dQ_st mu contracted block by block against
        the Kronecker factors (c0, g1, g2, g3) and S = Q^{-1} on the BTA
        pattern.  The forward half (``adjoint_forward``: assembly,
        factorisations, log-determinants, latent mean) and the backward half
        (``adjoint_backward``: selected inversions and contractions) run back
        to back.  For a non-Gaussian likelihood see ``_poisson_forward``."""
        tok = self.adjoint_forward(thetas, precision, check=False)
        return self.adjoint_backward(tok)

    def adjoint_forward(self, thetas, precision=None, check=True):
        """Forward half of the adjoint gradient at K theta points: f(theta)
        with everything the backward half reuses left on the device (the
        factors of Q_c and Q_prior, the inverses of their diagonal factor
        blocks, the latent mean).  Returns a token for ``adjoint_backward``
        and ``f_device``; check=True synchronises and raises on a matrix
        that is not positive definite.  A later forward on this model
        invalidates the token (the backward then recomputes the forward)."""
        default = precision is None
        precision = self.selinv_precision if precision is None else precision
        if precision not in _PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_PRECISIONS)}")
        demoted = False
        if default and precision != "fp64" and self._demote_left > 0:
            self._demote_left -= 1
            precision, demoted = "fp64", True
        thetas = [np.asarray(t, dtype=np.float64) for t in thetas]
        if not self.gaussian:
            self._poisson_forward(thetas)
        else:
            self._gauss_forward(thetas, precision)
        self._fwd_gen = getattr(self, "_fwd_gen", 0) + 1
        tok = {"gen": self._fwd_gen, "thetas": thetas, "precision": precision, "fs": None, "default": default,
               "demoted": demoted}
        self._fwd_token = tok
        if check:
            self.status()
        if not self.gaussian:
            tok["fs"] = [self._f_poisson(sl, th) for sl, th in zip(self.slots, thetas)]
        return tok

    def f_device(self, tok):
        """f at the token's points as a device tensor (K,), without a host
        synchronisation for Gaussian likelihoods."""
        import torch

        if tok["fs"] is not None:
            return torch.tensor(tok["fs"], dtype=torch.float64, device=self.device)
        self._require_live(tok)
        K = len(tok["thetas"])
        parts = torch.stack([self.slots[j].scal[:3] for j in range(K)])
        c = torch.tensor([float(self.log_prior_theta(th) + self.lik0(th)) for th in tok["thetas"]],
                         dtype=torch.float64, device=self.device)
        return 0.5 * parts[:, 0] - 0.5 * parts[:, 1] - 0.5 * parts[:, 2] - c

    def _require_live(self, tok):
        if getattr(self, "_fwd_token", None) is not tok:
            raise RuntimeError("the device state of this forward evaluation was overwritten by a later one")

    def adjoint_backward(self, tok):
        """Backward half: (f, gradient) at the token's points from the
        selected inversions of Q_c and Q_prior and their contractions with
        dQ/dtheta (block inner products against the Kronecker factors, the
        quadratic and likelihood terms from the forward's latent mean).  A
        token whose device state was overwritten is recomputed first.  The
        selected inversion overwrites the factors, so the token is used up."""
        if getattr(self, "_fwd_token", None) is not tok:
            redo = self.adjoint_forward(tok["thetas"], tok["precision"], check=False)
            redo.update(default=tok.get("default", False), demoted=tok.get("demoted", False))
            tok = redo
        self._fwd_token = None
        if not self.gaussian:
            return self._poisson_backward(tok)
        return self._gauss_backward(tok)

    def _gauss_forward(self, thetas, precision="fp64"):
        _gauss_forward_group([(self, thetas)], _factor_arith(self.factor_precision, [self], precision))

    def _gauss_backward(self, tok):
        return _gauss_backward_group([(self, tok)])[0]

    def _gauss_gradients(self, thetas, precision, tok=None):
        """Host half of the Gaussian backward: f and the gradient of every
        point from the scalars and block contractions on the device."""
        K = len(thetas)
        n = self.nt
        sls = self.slots[:K]
        mult = np.ones((2 * n - 1, 1))
        mult[n:] = 2.0  # each sub-diagonal block appears twice in the symmetric matrix
        prior_idx = [k for k in range(len(self.theta_keys)) if k not in self.tau_idx]
        fs, grads = [], []
        self.last_check = []
        for sl, theta in zip(sls, thetas):
            s = sl.scal[:3].cpu().numpy()
            vs = sl.vscal.view(-1, 3).cpu().numpy()
            Ic = sl.inner_c.view(2 * n - 1, -1).cpu().numpy()
            Ip = sl.inner_p.view(2 * n - 1, -1).cpu().numpy()
            Qm = sl.quad_st.view(2 * n - 1, -1).cpu().numpy()
            Tsel = sl.Qc.T.cpu().numpy()
            f = 0.5 * s[0] - 0.5 * s[1] - (self.log_prior_theta(theta) + self.lik0(theta) + 0.5 * s[2])
            grad = np.zeros(theta.size)
            for k in prior_idx:
                dc = self._dcoef(theta, k) * mult
                grad[k] = 0.5 * np.sum(dc * (Ic - Ip + Qm)) - self._dfun(self.log_prior_theta, theta, k)
            rest_c = 0.0
            for j, k in enumerate(self.tau_idx):
                tau = math.exp(theta[k])
                tr_ata = vs[j, 0] + float(np.sum(Tsel * self.XtX_var[j]))
                rest_c += tau * tr_ata
                grad[k] = (0.5 * tau * tr_ata + 0.5 * tau * vs[j, 1] - tau * vs[j, 2]
                           - (0.5 * self.nobs_var[j] - 0.5 * tau * self.yty_var[j])
                           - self._dfun(self.log_prior_theta, theta, k))
            rc, rp = self._identity_residuals(theta, Ic, Ip, rest_c, self.fe_prec * float(np.trace(Tsel)))
            self.last_check.append({"precision": precision, "residual_c": rc, "residual_p": rp, "fallback": False})
            fs.append(float(f))
            grads.append(grad)
        return self._mixed_fallback(thetas, fs, grads, precision, tok)

    # --------------------------------------------------------- marginals
    def _covariance(self, theta, x_star):
        """Q_c(theta, eta = A x*) factorised and selected-inverted in place
        (``DALIA._compute_covariance_latent_parameters``, ``dalia.py:912-936``)."""
        import torch

        theta = np.asarray(theta, dtype=np.float64)
        sl = self.slots[0]
        _lib.check(self.lib.bta_reset_status(self.h.bind_stream()), "reset")
        if x_star is not None:
            sl.x.copy_(torch.as_tensor(np.asarray(x_star, dtype=np.float64)).to(self.device))
        if self.gaussian:
            self._gauss_conditional(theta, sl)
        else:
            self.spmv(self.A_rowptr, self.A_col, self.A_val, self.nobs, sl.x, sl.eta)
            self._check(self.lib.bta_poisson_terms(self._stream(), self.nobs, _lib.ptr(sl.eta), _lib.ptr(self.y),
                                                   _lib.ptr(self.e), _lib.ptr(sl.dvec), _lib.ptr(sl.gvec),
                                                   _lib.ptr(self.part), self.nparts, _lib.ptr(sl.scal[5:6])),
                        "poisson_terms")
            self.assemble_conditional(theta, sl.dvec, 1.0, sl)
        self.factor(sl.Qc)
        self.selinv(sl.Qc)
        self.status()
        return sl

    def marginal_variances_latent(self, theta, x_star=None):
        """diag(Q_c^{-1}) (``DALIA.get_marginal_variances_latent_parameters``,
        ``dalia.py:938-962``), as a device tensor of length N."""
        import torch

        sl = self._covariance(theta, x_star)
        d = torch.diagonal(sl.Qc.D, dim1=1, dim2=2).reshape(-1)
        return torch.cat([d, torch.diagonal(sl.Qc.T)]) if self.nb else d.clone()

    def marginal_variances_observations(self, theta, x_star=None):
        """diag(A Q_c^{-1} A^T) (``DALIA.get_marginal_variances_observations``,
        ``dalia.py:964-1021``), gathered from the selected inverse on the BTA
        pattern in one pass over the rows of A (the reference forms the sparse
        product A S A^T).  Unlike the reference, non-Gaussian likelihoods are
        supported (Q_c at eta = A x*)."""
        import torch

        sl = self._covariance(theta, x_star)
        out = torch.empty(self.nobs, dtype=torch.float64, device=self.device)
        self._check(self.lib.bta_obs_quad(self._stream(), self.nobs, _lib.ptr(self.obs_off), _lib.ptr(self.obs_dst),
                                          _lib.ptr(self.obs_w), _lib.ptr(sl.Qc.buf), self.nb, _lib.ptr(self.X),
                                          _lib.ptr(sl.Qc.T) if self.nb else None, None, _lib.ptr(out)), "obs_quad")
        return out

    # ------------------------------------------------------------- Poisson
    def _prior_apply(self, sl, x, out):
        """out = Q_prior x: the spatio-temporal block through its Kronecker
        structure (coefficients of the last prior assembly of ``sl``) and the
        fixed-effect block fe_prec I."""
        s = self._stream()
        nst = self.nt * self.ns
        self._check(self.lib.bta_kron_symv(s, self.nt, self.ns, _lib.ptr(sl.coef_dev[1]), _lib.ptr(self.u_rowptr),
                                           _lib.ptr(self.u_col), _lib.ptr(self.u_vals4), _lib.ptr(x), 1.0, 0.0,
                                           _lib.ptr(out)), "kron_symv")
        if self.nb > 0:
            self._check(self.lib.bta_axpby(s, self.nb, self.fe_prec, _lib.ptr(x[nst:]), 0.0, _lib.ptr(out[nst:])),
                        "axpby")

    def _newton(self, sls, thetas):
        """Newton inner iteration (``DALIA._inner_iteration``, ``dalia.py:1023-1072``)
        of every point, in lockstep: each step assembles Q_c(eta) with
        eta = A x*, factorises all unconverged points together, solves
        Q_c dx = -Q_prior x* + A^T (y - e exp(eta)) and stops a point once
        |dx|_2 < eps_inner_iteration.  As in the reference, x* (``sl.x``, warm
        started from its previous value) does not receive the final update,
        and Q_c, eta and the likelihood stay those of the last assembly.  The
        BT factorisation of Q_prior joins the first batch."""
        s = self._stream()
        K = len(sls)
        for sl, th in zip(sls, thetas):
            self.assemble_prior_bt(th, sl)
            sl.upd.zero_()
        active = list(range(K))
        counter = [0] * K
        first = True
        while active:
            for j in active:
                if counter[j] > self.max_inner:
                    raise ValueError(f"Inner iteration did not converge after {counter[j]} iterations.")
            for j in active:
                sl = sls[j]
                self._check(self.lib.bta_axpby(s, self.N, 1.0, _lib.ptr(sl.upd), 1.0, _lib.ptr(sl.x)), "axpby")
                self.spmv(self.A_rowptr, self.A_col, self.A_val, self.nobs, sl.x, sl.eta)
                self._check(self.lib.bta_poisson_terms(s, self.nobs, _lib.ptr(sl.eta), _lib.ptr(self.y),
                                                       _lib.ptr(self.e), _lib.ptr(sl.dvec), _lib.ptr(sl.gvec),
                                                       _lib.ptr(self.part), self.nparts, _lib.ptr(sl.scal[5:6])),
                            "poisson_terms")
                self.assemble_conditional(thetas[j], sl.dvec, 1.0, sl)
            mats = [sls[j].Qc for j in active] + ([sl.Qp for sl in sls] if first else [])
            self.factor_batched(mats)
            for j in active:
                sl = sls[j]
                self._prior_apply(sl, sl.x, sl.qpx)
                self.spmv(self.AT_rowptr, self.AT_col, self.AT_val, self.N, sl.gvec, sl.rhs)
                self._check(self.lib.bta_axpby(s, self.N, -1.0, _lib.ptr(sl.qpx), 1.0, _lib.ptr(sl.rhs)), "axpby")
                sl.upd.copy_(sl.rhs)
            self.solve_in_place([sls[j] for j in active], [sls[j].upd for j in active])
            for j in active:
                self.dot_to(sls[j].upd, sls[j].upd, sls[j].scal[6:7])
            self.status()
            import torch

            nrm = torch.stack([sls[j].scal[6] for j in active]).cpu().numpy()
            still = []
            for j, v in zip(active, nrm):
                counter[j] += 1
                self.work["newton_steps"] += 1
                if math.sqrt(max(float(v), 0.0)) >= self.eps_inner:
                    still.append(j)
            active = still
            first = False
        for sl in sls:
            self.logdet_to(sl.Qc, sl.scal[0:1])
            self.logdet_to(sl.Qp, sl.scal[2:3])
            self.dot_to(sl.x, sl.qpx, sl.scal[1:2])
        return counter

    def _f_poisson(self, sl, theta):
        """f = -(log p(theta) + lik(eta*) + 1/2 logdet_bt Q_st - 1/2 x*^T Q_prior x*
        - 1/2 logdet Q_c) (``dalia.py:699-729``), from the scalars of ``_newton``."""
        v = sl.scal[:7].cpu().numpy()
        return float(-(self.log_prior_theta(theta) + v[5] + 0.5 * v[2] - 0.5 * v[1] - 0.5 * v[0]))

    def _evaluate_f_poisson(self, theta):
        _lib.check(self.lib.bta_reset_status(self.h.bind_stream()), "reset")
        sl = self.slots[0]
        self._newton([sl], [theta])
        return self._f_poisson(sl, theta)

    def _poisson_forward(self, thetas):
        """Forward half for the Poisson likelihood: the Newton iteration of
        every point to its mode (``_newton``), warm-started from the current
        mode of slot 0; leaves Q_c (factored at the mode), the BT factor of
        Q_prior and the scalars of f on the device."""
        K = len(thetas)
        sls = [self.slot(j) for j in range(K)]
        for sl in sls[1:]:
            sl.x.copy_(sls[0].x)  # warm start every point from the current mode
        _lib.check(self.lib.bta_reset_status(self.h.bind_stream()), "reset")
        self._newton(sls, thetas)

    def _poisson_backward(self, tok):
        """(f, gradient) at K theta points for the Poisson likelihood.

        With x* the mode, Q_c = Q_prior + A^T diag(d) A, d = e exp(A x*),
        S_c = Q_c^{-1}, S_p = Q_st^{-1} and dQ = dQ_prior/dtheta_k:
          df = 1/2 x*^T dQ x* + 1/2 tr(S_c dQ) - 1/2 tr(S_p dQ_st) - d log p
               + (dx - 1/2 z)^T dQ x*,   z = Q_c^{-1} A^T (d * diag(A S_c A^T)).
        The z term is the change of 1/2 logdet Q_c through the mode,
        dx*/dtheta = -Q_c^{-1} dQ x*; the dx term (dx = the final Newton
        update, which the reference does not apply) is the first-order
        change of the objective's x*^T Q_prior x* / likelihood part at the
        unconverged x*, so the gradient matches the objective as evaluated."""
        import torch

        thetas, precision = tok["thetas"], tok["precision"]
        K = len(thetas)
        n, b = self.nt, self.ns
        s = self._stream()
        sls = self.slots[:K]
        for sl in sls:
            if sl.Sc is None:
                sl.Sc = BTAMatrix(n, b, self.nb, self._dev)
            sl.Sc.buf.copy_(sl.Qc.buf)
        # inverses of Q_c's diagonal factor blocks at the mode: the selected
        # inversion of its copy and the two sweeps of the z solve share them
        use_v = self._inverses_fit(sls)
        Vc = [self._slot_inverses(sl) for sl in sls] if use_v else [None] * K
        if use_v:
            self.block_inverses([sl.Qc for sl in sls], Vc)
        self.selinv_batched([sl.Sc for sl in sls] + [sl.Qp for sl in sls], precision, Vc + [None] * K)
        for sl in sls:
            self._check(self.lib.bta_obs_quad(s, self.nobs, _lib.ptr(self.obs_off), _lib.ptr(self.obs_dst),
                                              _lib.ptr(self.obs_w), _lib.ptr(sl.Sc.buf), self.nb, _lib.ptr(self.X),
                                              _lib.ptr(sl.Sc.T) if self.nb else None, _lib.ptr(sl.dvec),
                                              _lib.ptr(sl.hvec)), "obs_quad")
            self.spmv(self.AT_rowptr, self.AT_col, self.AT_val, self.N, sl.hvec, sl.z)
            self.dot_to(sl.hvec, self.ones_obs, sl.scal[7:8])  # <S_c, A^T diag(d) A>
        if use_v:
            self.sweep_inv_batched([sl.Qc for sl in sls], Vc, [sl.z for sl in sls], 0)
            self.sweep_inv_batched([sl.Qc for sl in sls], Vc, [sl.z for sl in sls], 1)
        else:
            self.sweep_batched([sl.Qc for sl in sls], [sl.z for sl in sls], 0)
            self.sweep_batched([sl.Qc for sl in sls], [sl.z for sl in sls], 1)
        for sl in sls:
            self._check(self.lib.bta_axpby(s, self.N, 1.0, _lib.ptr(sl.upd), -0.5, _lib.ptr(sl.z)), "axpby")
            args = (s, n, b, _lib.ptr(self.u_rowptr), _lib.ptr(self.u_col), _lib.ptr(self.u_vals4))
            self._check(self.lib.bta_block_bilinear(*args, _lib.ptr(sl.z), _lib.ptr(sl.x), _lib.ptr(sl.bil)),
                        "block_bilinear")
            self._check(self.lib.bta_block_quad(*args, _lib.ptr(sl.x), _lib.ptr(sl.quad_st)), "block_quad")
            Dc, Lc, _, _ = sl.Sc.ptrs()
            Dp, Lp, _, _ = sl.Qp.ptrs()
            self._check(self.lib.bta_block_inner(*args, Dc, Lc, _lib.ptr(sl.inner_c)), "block_inner")
            self._check(self.lib.bta_block_inner(*args, Dp, Lp, _lib.ptr(sl.inner_p)), "block_inner")
        self.status()
        mult = np.ones((2 * n - 1, 1))
        mult[n:] = 2.0
        fs, grads = [], []
        self.last_check = []
        for sl, theta in zip(sls, thetas):
            Ic = sl.inner_c.view(-1, 4).cpu().numpy()
            Ip = sl.inner_p.view(-1, 4).cpu().numpy()
            Qm = sl.quad_st.view(-1, 4).cpu().numpy()
            Bm = sl.bil.view(-1, 4).cpu().numpy()
            grad = np.zeros(theta.size)
            for k in range(theta.size):
                dc = self._dcoef(theta, k)
                grad[k] = (0.5 * np.sum(dc * mult * (Ic - Ip + Qm)) + np.sum(dc * Bm)
                           - self._dfun(self.log_prior_theta, theta, k))
            rest = float(sl.scal[7].item())
            tip = self.fe_prec * float(torch.trace(sl.Sc.T).item()) if self.nb else 0.0
            rc, rp = self._identity_residuals(theta, Ic, Ip, rest, tip)
            self.last_check.append({"precision": precision, "residual_c": rc, "residual_p": rp, "fallback": False})
            grads.append(grad)
        fs = list(tok["fs"])
        return self._mixed_fallback(thetas, fs, grads, precision, tok)


# ------------------------------------------------------------------ groups
# The Gaussian adjoint of several models at once: every launch of the forward
# (factorisations, block inverses, sweeps) and of the backward (selected
# inversions) takes the matrices of all models together, so instances of
# different block sizes -- e.g. bivariate and univariate models -- share the
# launches.  A group with one model is the ordinary batched evaluation.

def _gauss_forward_group(jobs, factor_precision="fp64"):
    """jobs: [(model, thetas)] with Gaussian likelihoods on one device;
    factor_precision: arithmetic of the factorisations' Schur updates."""
    lead = jobs[0][0]
    parts = []
    _lib.check(lead.lib.bta_reset_status(lead.h.bind_stream()), "reset")
    for m, thetas in jobs:
        sls = [m.slot(j) for j in range(len(thetas))]
        for sl, th in zip(sls, thetas):
            m._gauss_conditional(th, sl)
            m.assemble_prior_bt(th, sl)
        parts.append((m, sls, thetas))
    Qc = [sl.Qc for _, sls, _ in parts for sl in sls]
    Qp = [sl.Qp for _, sls, _ in parts for sl in sls]
    lead.factor_batched(Qc + Qp, factor_precision)
    # inverses of Q_c's diagonal factor blocks: the sweeps become n dependent
    # matrix-vector steps, and the selected inversion reuses them
    Vc = [m._slot_inverses(sl) for m, sls, _ in parts for sl in sls]
    lead.block_inverses(Qc, Vc)
    xs = []
    for m, sls, thetas in parts:
        for sl, th in zip(sls, thetas):
            m.logdet_to(sl.Qc, sl.scal[0:1])
            m.logdet_to(sl.Qp, sl.scal[2:3])
            m._gauss_rhs(th, sl)
            sl.x.copy_(sl.rhs)
            xs.append(sl.x)
    lead.sweep_inv_batched(Qc, Vc, xs, 0)
    for m, sls, _ in parts:
        for sl in sls:
            m.dot_to(sl.x, sl.x, sl.scal[1:2])  # b^T Q^-1 b = |L^-1 b|^2
    lead.sweep_inv_batched(Qc, Vc, xs, 1)  # mu
    return parts


def _gauss_backward_group(jobs):
    """jobs: [(model, token)] whose forwards ran together (or alone) and are
    still on the device, all with the same precision; returns [(fs, grads)]."""
    lead = jobs[0][0]
    precision = jobs[0][1]["precision"]
    mats, Vs = [], []
    for m, tok in jobs:
        K = len(tok["thetas"])
        n, ns, nv = m.nt, m.ns, m.nv
        stream = m._stream()
        pat = (_lib.ptr(m.u_rowptr), _lib.ptr(m.u_col), _lib.ptr(m.u_vals4))
        for sl in m.slots[:K]:
            # per variate |A_v mu|^2 and (A_v mu)^T y_v; mu^T (E_tt' (x) K) mu per sub-block
            m.spmv(m.A_rowptr, m.A_col, m.A_val, m.nobs, sl.x, sl.eta)
            for j, (lo, hi) in enumerate(m.var_ranges):
                m.dot_to(sl.eta[lo:hi], sl.eta[lo:hi], sl.vscal[3 * j + 1:3 * j + 2])
                m.dot_to(sl.eta[lo:hi], m.y[lo:hi], sl.vscal[3 * j + 2:3 * j + 3])
            m._check(m.lib.bta_block_quad_mv(stream, n, ns, nv, *pat, _lib.ptr(sl.x), _lib.ptr(sl.quad_st)),
                     "block_quad")
        mats += [sl.Qc for sl in m.slots[:K]] + [sl.Qp for sl in m.slots[:K]]
        Vs += [sl.Vc for sl in m.slots[:K]] + [None] * K
    # selected inverses of every matrix of the group, then their contractions
    lead.selinv_batched(mats, precision, Vs)
    for m, tok in jobs:
        K = len(tok["thetas"])
        n, ns, nv = m.nt, m.ns, m.nv
        stream = m._stream()
        pat = (_lib.ptr(m.u_rowptr), _lib.ptr(m.u_col), _lib.ptr(m.u_vals4))
        for sl in m.slots[:K]:
            Dc, Lc, _, _ = sl.Qc.ptrs()
            Dp, Lp, _, _ = sl.Qp.ptrs()
            for (Dm, Lm, out) in ((Dc, Lc, sl.inner_c), (Dp, Lp, sl.inner_p)):
                m._check(m.lib.bta_block_inner_mv(stream, n, ns, nv, *pat, Dm, Lm, _lib.ptr(out)), "block_inner")
            for j in range(len(m.var_ranges)):
                m._check(m.lib.bta_gather_dot(stream, m.nent, _lib.ptr(m.ent_dst), _lib.ptr(m.ata_w_var[j]),
                                              _lib.ptr(sl.Qc.buf), _lib.ptr(m.part), m.nparts,
                                              _lib.ptr(sl.vscal[3 * j:3 * j + 1])), "gather_dot")
    lead.status()
    return [m._gauss_gradients(tok["thetas"], precision, tok) for m, tok in jobs]


def adjoint_group(jobs, precision="fp64"):
    """(f, exact gradient) of several Gaussian models at once:
    jobs = [(model, thetas)], each model on the same device with its own
    points.  All factorisations, block inverses, sweeps and selected
    inversions of every model's Q_c and Q_prior share their launches (the
    instances may have different block and arrowhead sizes).  Returns
    [(fs, grads)] per job; the per-point accuracy check and FP64 fallback
    of each model apply as in ``objective_adjoint_batched``."""
    if precision not in _PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(_PRECISIONS)}")
    jobs = [(m, [np.asarray(t, dtype=np.float64) for t in ths]) for m, ths in jobs]
    if any(not m.gaussian for m, _ in jobs):
        raise NotImplementedError("grouped adjoint evaluation: Gaussian likelihoods")
    if len({id(m) for m, _ in jobs}) != len(jobs):
        raise ValueError("each model may appear once in a group")
    fp = _factor_arith(jobs[0][0].factor_precision, [m for m, _ in jobs], precision)
    _gauss_forward_group(jobs, fp)
    toks = []
    for m, thetas in jobs:
        m._fwd_gen = getattr(m, "_fwd_gen", 0) + 1
        m._fwd_token = None  # consumed by the backward below
        toks.append((m, {"gen": m._fwd_gen, "thetas": thetas, "precision": precision, "fs": None}))
    return _gauss_backward_group(toks)
