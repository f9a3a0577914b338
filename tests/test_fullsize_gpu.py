"""FP64 parity at the benchmarked sizes: the device path against the CPU
oracle (the reference's Serinv-path algorithm restated in NumPy/SciPy LAPACK,
pinned to DALIA's own outputs by the golden fixtures) on the same seeded
synthetic problems.  Every result the plain FP64 path produces is compared
within 1e-10 relative: log-determinants of Q_conditional and of Q_prior
(BT), the latent mean, f(theta), the selected inverse on the BTA pattern and
the marginal variances.

gst_1500x20 is the profiled mid-size case (block 1500, 20 blocks);
gst_1500x100 is the benchmark workload itself.  The oracle needs about a
minute of host time for the larger one."""
import numpy as np
import pytest

from golden_util import rel
from oracle import bta_ref, model_ref

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _oracle_parts(prob, theta, selinv):
    """logdet Q_c, logdet_bt Q_st, mu, f and (optionally) the selected
    inverse of Q_c, each step as ``OracleModel.evaluate_f`` /
    ``marginal_variances`` takes it, with one factorisation per matrix."""
    om = model_ref.OracleModel(prob)
    eta = np.zeros(len(prob.y))
    Qc = om.q_cond(theta, eta)
    D, L, Ab, T = om._factor_bta(Qc)
    ld_c = bta_ref.logdet(D, T, "bta")
    ld_p = om._logdet_prior_bt(theta)
    rhs = om.AT @ om.grad_lik(theta, eta)
    mu = om._solve((D, L, Ab, T), rhs)
    f = 0.5 * ld_c - 0.5 * mu @ (Qc @ mu) - (om.log_prior_theta(theta) + om.lik(theta, eta) + 0.5 * ld_p)
    sel = None
    if selinv:
        bta_ref.pobtasi(D, L, Ab, T)
        sel = (D, L, Ab, T)
    return ld_c, ld_p, mu, float(f), sel


@pytest.mark.parametrize("name", ["gst_1500x20", "gst_1500x100"])
def test_fp64_path_matches_oracle_at_full_size(name):
    from dalia_b200 import synth
    from dalia_b200.model import SpatioTemporalModel

    cfg = synth.CONFIGS[name]
    prob = synth.make_config(name, seed=0)
    theta = np.asarray(cfg["theta"], dtype=np.float64)
    ld_c, ld_p, mu, f_ref, sel = _oracle_parts(prob, theta, selinv=True)

    m = SpatioTemporalModel(prob)
    f = m.evaluate_f(theta)
    s = m.scal[:3].cpu().numpy()
    assert abs(s[0] - ld_c) <= TOL * abs(ld_c)
    assert abs(s[2] - ld_p) <= TOL * abs(ld_p)
    assert rel(m.x.cpu().numpy(), mu) < TOL
    assert abs(f - f_ref) <= TOL * abs(f_ref)

    mv = m.marginal_variances_latent(theta).cpu().numpy()
    D, L, Ab, T = sel
    mv_ref = np.concatenate([np.concatenate([np.diagonal(D[i]) for i in range(m.nt)]), np.diagonal(T)])
    assert rel(mv, mv_ref) < TOL
    # entry by entry the smallest variances (1e-6 of the largest) carry the
    # rounding of the recurrence relative to their own size: measured up to
    # 1e-9 between two FP64 evaluations in different operation orders
    assert float(np.max(np.abs(mv - mv_ref) / np.abs(mv_ref))) < 1e-8
    # the selected inverse on the BTA pattern (DALIA reads the lower
    # triangles of the diagonal blocks, the sub-diagonal and arrow blocks)
    # the selected inverse on the BTA pattern as a whole (DALIA reads the lower
    # triangles of the diagonal blocks, the sub-diagonal and arrow blocks, the
    # tip); array by array and block by block (condition numbers up to 1e9)
    # two FP64 evaluations in different operation orders differ by up to
    # 1.1e-10, so those are held to 3e-10
    Q = m.slots[0].Qc
    got = [np.tril(Q.D.cpu().numpy()), Q.L.cpu().numpy(), Q.Ab.cpu().numpy(), Q.T.cpu().numpy()]
    ref = [np.tril(D), L, Ab, T]
    assert rel(np.concatenate([g.ravel() for g in got]), np.concatenate([r.ravel() for r in ref])) < TOL
    for g, r in zip(got, ref):
        assert rel(g, r) < 3 * TOL
    for i in range(m.nt):
        assert rel(got[0][i], ref[0][i]) < 3 * TOL, i


def test_adjoint_and_mixed_gradient_at_mid_size():
    """At gst_1500x20 (too large for the dense adjoint oracle) the FP64
    adjoint gradient is checked against fourth-order central differences of
    the device f (h = 1e-3; f itself matches the oracle above), and the
    8-bit-slice backward against the FP64 one within 1e-6."""
    from dalia_b200 import synth
    from dalia_b200.model import SpatioTemporalModel

    name = "gst_1500x20"
    prob = synth.make_config(name, seed=0)
    theta = np.asarray(synth.CONFIGS[name]["theta"], dtype=np.float64)
    m = SpatioTemporalModel(prob)
    f64, g64 = m.objective_adjoint(theta)
    h = 1e-3
    fd = np.zeros_like(theta)
    for k in range(theta.size):
        e = np.zeros_like(theta)
        e[k] = h
        d1 = m.evaluate_f(theta + e) - m.evaluate_f(theta - e)
        d2 = m.evaluate_f(theta + 2 * e) - m.evaluate_f(theta - 2 * e)
        fd[k] = (8 * d1 - d2) / (12 * h)
    # f carries ~1e-7 absolute rounding (its quadratic term is ~1e5), so the
    # quotient resolves the gradient to ~1e-6 relative (measured 3e-7)
    assert rel(g64, fd) < 1e-6
    fi8, gi8 = m.objective_adjoint_batched([theta], precision="i8slice")
    assert abs(fi8[0] - f64) <= 1e-13 * abs(f64)
    assert rel(gi8[0], g64) < 1e-6
    assert not m.last_check[0]["fallback"]
