"""Parity of the CUDA BTA kernels with the CPU oracle, through the C ABI
(Serinv-compatible wrappers).  Tolerance: 1e-10 relative (norm-wise), the
bar the reference's FP64 results are held to."""
import numpy as np
import pytest

from golden_util import load, rel
from oracle import bta_ref

pytestmark = pytest.mark.gpu

TOL = 1e-10

SHAPES = [
    (1, 7, 0), (1, 64, 3), (2, 33, 1), (3, 65, 5), (4, 64, 3), (3, 130, 2),
    (5, 48, 0), (2, 96, 70), (6, 200, 6), (3, 1, 1), (2, 129, 0),
]


def _cuda(*arrs):
    import torch

    return [None if a is None else torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrs]


def _np(*ts):
    return [None if t is None else t.cpu().numpy() for t in ts]


@pytest.mark.parametrize("n,b,a", SHAPES)
def test_pobtaf_logdet_solve_selinv(n, b, a):
    from dalia_b200 import serinv_compat as sc

    rng = np.random.default_rng(100 * n + b + a)
    D, L, Ab, T = bta_ref.random_bta(n, b, a, rng)
    M = bta_ref.bta_to_dense(D, L, Ab, T)
    ref = [x.copy() for x in (D, L, Ab, T)]
    bta_ref.pobtaf(*ref)
    d = _cuda(D, L, Ab, T)
    if a == 0:
        sc.pobtf(d[0], d[1])
    else:
        sc.pobtaf(*d)
    got = _np(*d)
    assert rel(got[0], ref[0]) < TOL
    if n > 1:
        assert rel(got[1], ref[1]) < TOL
    if a:
        assert rel(got[2], ref[2]) < TOL and rel(got[3], ref[3]) < TOL
    # upper triangles of the factor blocks are zero
    assert np.all(np.triu(got[0], 1) == 0)
    ld = sc.logdet(d[0], d[3] if a else None, "bta")
    sign, ld_ref = np.linalg.slogdet(M)
    assert sign > 0 and abs(ld - ld_ref) < TOL * abs(ld_ref) + 1e-9
    # solve
    rhs = rng.standard_normal(n * b + a)
    x = _cuda(rhs)[0]
    sc.pobtas(d[0], d[1], d[2] if a else None, d[3] if a else None, x, "N")
    sc.pobtas(d[0], d[1], d[2] if a else None, d[3] if a else None, x, "C")
    assert rel(x.cpu().numpy(), np.linalg.solve(M, rhs)) < TOL
    # selected inversion
    if a == 0:
        sc.pobtsi(d[0], d[1])
    else:
        sc.pobtasi(*d)
    got = _np(*d)
    Sref = bta_ref.dense_to_bta(np.linalg.inv(M), n, b, a)
    assert rel(got[0], Sref[0]) < TOL
    if n > 1:
        assert rel(got[1], Sref[1]) < TOL
    if a:
        assert rel(got[2], Sref[2]) < TOL and rel(got[3], Sref[3]) < TOL


@pytest.mark.parametrize("name", ["gst_small", "gst_ragged"])
def test_b200solver_on_reference_precision_matrices(name):
    """Q_conditional assembled by the reference; results vs the reference's
    dense LAPACK solver (DenseSolver) stored in the fixture."""
    import scipy.sparse as sps
    from dalia_b200.solver import B200Solver

    g = load(name)
    ns, nt, nb = (int(v) for v in g["shape"][:3])
    N = ns * nt + nb
    Qc = sps.coo_matrix((g["qc_data"], (g["qc_row"], g["qc_col"])), shape=(N, N)).tocsc()
    s = B200Solver(None, diagonal_blocksize=ns, n_diag_blocks=nt, arrowhead_blocksize=nb)
    s.cholesky(Qc, sparsity="bta")
    assert abs(s.logdet("bta") - float(g["logdet_qc"])) < TOL * abs(float(g["logdet_qc"]))
    x = s.solve(g["rhs"].copy(), "bta")
    assert rel(x, g["x_solve"]) < TOL
    s.selected_inversion("bta")
    for k, arr in (("sel_D", s.A_diagonal_blocks), ("sel_L", s.A_lower_diagonal_blocks),
                   ("sel_Ab", s.A_arrow_bottom_blocks), ("sel_T", s.A_arrow_tip_block)):
        assert rel(arr.cpu().numpy(), g[k]) < TOL, k
    mv = s._structured_to_spmatrix(sps.eye(N), "bta").diagonal()
    assert rel(mv, np.diag(bta_ref.bta_to_dense(g["sel_D"], g["sel_L"], g["sel_Ab"], g["sel_T"]))) < TOL


def test_serinv_compat_numpy_host_arrays():
    from dalia_b200 import serinv_compat as sc

    rng = np.random.default_rng(5)
    D, L, Ab, T = bta_ref.random_bta(3, 40, 4, rng)
    ref = [x.copy() for x in (D, L, Ab, T)]
    bta_ref.pobtaf(*ref)
    sc.pobtaf(D, L, Ab, T)
    for g_, r_ in zip((D, L, Ab, T), ref):
        assert rel(g_, r_) < TOL


def test_not_positive_definite_raises():
    from dalia_b200 import serinv_compat as sc

    rng = np.random.default_rng(7)
    D, L, Ab, T = bta_ref.random_bta(3, 70, 2, rng)
    D[1, 5, 5] = -1e6
    d = _cuda(D, L, Ab, T)
    with pytest.raises(np.linalg.LinAlgError):
        sc.pobtaf(*d)
    # the handle stays usable
    D2, L2, Ab2, T2 = bta_ref.random_bta(2, 30, 1, rng)
    d2 = _cuda(D2, L2, Ab2, T2)
    sc.pobtaf(*d2)


def test_batched_factor_and_selinv_match_single():
    """Instances of different sizes in one batched launch give the results of
    separate calls."""
    import ctypes

    import torch

    from dalia_b200 import _lib

    lib = _lib.load()
    h = _lib.handle()
    shapes = [(4, 130, 3), (3, 64, 0), (5, 70, 6), (2, 200, 1)]
    rng = np.random.default_rng(11)
    mats = [bta_ref.random_bta(n, b, a, rng) for n, b, a in shapes]
    single = [_cuda(*m) for m in mats]
    batch = [_cuda(*m) for m in mats]
    for (n, b, a), t in zip(shapes, single):
        assert lib.bta_pobtaf(h.bind_stream(), n, b, a, *[_lib.ptr(x if x.numel() else None) for x in t], None) == 0
    k = len(shapes)
    I64, P = ctypes.c_int64 * k, ctypes.c_void_p * k
    args = (I64(*[s[0] for s in shapes]), I64(*[s[1] for s in shapes]), I64(*[s[2] for s in shapes]),
            *[P(*[(t[j].data_ptr() if t[j].numel() else None) for t in batch]) for j in range(4)])
    info = ctypes.c_int64(-1)
    assert lib.bta_pobtaf_batched(h.bind_stream(), k, *args, ctypes.byref(info)) == 0 and info.value == 0
    for s_, b_ in zip(single, batch):
        for x, y in zip(s_, b_):
            if x.numel():
                assert rel(y.cpu().numpy(), x.cpu().numpy()) < TOL
    for (n, b, a), t in zip(shapes, single):
        assert lib.bta_pobtasi(h.bind_stream(), n, b, a, *[_lib.ptr(x if x.numel() else None) for x in t]) == 0
    assert lib.bta_pobtasi_batched(h.bind_stream(), k, *args) == 0
    torch.cuda.synchronize()
    for (n, b, a), m, s_, b_ in zip(shapes, mats, single, batch):
        S = bta_ref.dense_to_bta(np.linalg.inv(bta_ref.bta_to_dense(*m)), n, b, a)
        for j, (x, y) in enumerate(zip(s_, b_)):
            if x.numel():
                assert rel(y.cpu().numpy(), x.cpu().numpy()) < TOL
                assert rel(y.cpu().numpy(), S[j]) < TOL


def test_whole_factorisation_launch_is_bit_identical_to_column_launches(monkeypatch):
    """The FP64 factorisation as one launch over every block column
    (DALIA_B200_PANEL_PERSIST=1, arrows of at most 64 rows) and as one launch per block
    column give bit-identical factors (the same tile tasks, each summing in
    the same order), both within 1e-10 of the oracle; instances of different
    block and arrow sizes and block counts share the launch."""
    import ctypes

    import torch

    from dalia_b200 import _lib

    lib = _lib.load()
    h = _lib.handle()
    shapes = [(4, 130, 3), (3, 64, 0), (6, 70, 6), (1, 200, 1), (5, 200, 64)]
    rng = np.random.default_rng(23)
    mats = [bta_ref.random_bta(n, b, a, rng) for n, b, a in shapes]
    k = len(shapes)
    I64, P = ctypes.c_int64 * k, ctypes.c_void_p * k
    outs = {}
    for mode in ("1", "0"):
        monkeypatch.setenv("DALIA_B200_PANEL_PERSIST", mode)
        dev = [_cuda(*m) for m in mats]
        args = (I64(*[s[0] for s in shapes]), I64(*[s[1] for s in shapes]), I64(*[s[2] for s in shapes]),
                *[P(*[(t[j].data_ptr() if t[j].numel() else None) for t in dev]) for j in range(4)])
        info = ctypes.c_int64(-1)
        assert lib.bta_pobtaf_batched(h.bind_stream(), k, *args, ctypes.byref(info)) == 0 and info.value == 0
        torch.cuda.synchronize()
        outs[mode] = [[x.cpu().numpy() for x in t] for t in dev]
    for m, one, cols in zip(mats, outs["1"], outs["0"]):
        ref = [x.copy() for x in m]
        bta_ref.pobtaf(*ref)
        for x, y, r in zip(one, cols, ref):
            if x.size:
                assert np.array_equal(x, y)
                assert rel(x, r) < TOL


@pytest.mark.parametrize("n,b,a", SHAPES)
def test_block_inverse_sweeps_and_selinv(n, b, a):
    """bta_block_inverses + bta_pobtas_inv_batched (two sweeps) against a dense
    solve, and bta_pobtasi_batched_v with those inverses against the oracle."""
    import ctypes

    import torch

    from dalia_b200 import _lib

    lib = _lib.load()
    h = _lib.handle()
    rng = np.random.default_rng(11 * n + b + a)
    D, L, Ab, T = bta_ref.random_bta(n, b, a, rng)
    M = bta_ref.bta_to_dense(D, L, Ab, T)
    d = _cuda(D, L, Ab, T)
    V = torch.empty(n * b * b, dtype=torch.float64, device="cuda")
    arr = lambda t: (ctypes.c_void_p * 1)(t.data_ptr() if (t is not None and t.numel()) else None)
    i64 = lambda v: (ctypes.c_int64 * 1)(v)
    sz = (i64(n), i64(b), i64(a))
    _lib.check(lib.bta_pobtaf_batched(h.bind_stream(), 1, *sz, arr(d[0]), arr(d[1]), arr(d[2]), arr(d[3]), None),
               "pobtaf")
    _lib.check(lib.bta_block_inverses(h.bind_stream(), 1, sz[0], sz[1], arr(d[0]), arr(V)), "inverses")
    rhs = rng.standard_normal(n * b + a)
    x = _cuda(rhs)[0]
    for trans in (0, 1):
        _lib.check(lib.bta_pobtas_inv_batched(h.bind_stream(), 1, *sz, arr(d[1]), arr(d[2]), arr(d[3]), arr(V),
                                              arr(x), trans), "sweep")
    st = ctypes.c_int64(0)
    _lib.check(lib.bta_get_status(h.bind_stream(), ctypes.byref(st)), "status")
    assert rel(x.cpu().numpy(), np.linalg.solve(M, rhs)) < TOL
    ref = [v.copy() for v in (D, L, Ab, T)]
    bta_ref.pobtaf(*ref)
    bta_ref.pobtasi(*ref)
    _lib.check(lib.bta_pobtasi_batched_v(h.bind_stream(), 1, *sz, arr(d[0]), arr(d[1]), arr(d[2]), arr(d[3]), arr(V),
                                         _lib.BTA_PREC_FP64), "pobtasi_v")
    got = _np(*d)
    assert rel(got[0], ref[0]) < TOL
    if n > 1:
        assert rel(got[1], ref[1]) < TOL
    if a:
        assert rel(got[2], ref[2]) < TOL and rel(got[3], ref[3]) < TOL


class _SerinvSolverCalls:
    """The calling sequence of DALIA's ``SerinvSolver`` against ``serinv.algs``
    (``src/dalia/solvers/structured_solver.py:72-190``): the four arrays
    passed positionally, one sweep per ``pobtas`` call with ``trans="N"``
    then ``trans="C"`` as keywords, the log-determinant read from the factor's
    diagonals in place, the selected inversion in place."""

    def __init__(self, algs, D, L, Ab, T):
        self.algs = algs
        self.A_diagonal_blocks, self.A_lower_diagonal_blocks = D, L
        self.A_arrow_bottom_blocks, self.A_arrow_tip_block = Ab, T

    def cholesky(self, sparsity):
        if sparsity == "bta":
            self.algs.pobtaf(self.A_diagonal_blocks, self.A_lower_diagonal_blocks, self.A_arrow_bottom_blocks,
                             self.A_arrow_tip_block)
        else:
            self.algs.pobtf(self.A_diagonal_blocks, self.A_lower_diagonal_blocks)

    def solve(self, rhs, sparsity):
        if sparsity == "bta":
            for tr in ("N", "C"):
                self.algs.pobtas(self.A_diagonal_blocks, self.A_lower_diagonal_blocks, self.A_arrow_bottom_blocks,
                                 self.A_arrow_tip_block, rhs, trans=tr)
        else:
            for tr in ("N", "C"):
                self.algs.pobts(self.A_diagonal_blocks, self.A_lower_diagonal_blocks, rhs, trans=tr)
        return rhs

    def logdet(self, sparsity, xp):
        ld = 0.0
        for i in range(self.A_diagonal_blocks.shape[0]):
            ld += float(xp.sum(xp.log(xp.diagonal(self.A_diagonal_blocks[i]))))
        if sparsity == "bta":
            ld += float(xp.sum(xp.log(xp.diagonal(self.A_arrow_tip_block))))
        return 2 * ld

    def selected_inversion(self, sparsity):
        if sparsity == "bta":
            self.algs.pobtasi(self.A_diagonal_blocks, self.A_lower_diagonal_blocks, self.A_arrow_bottom_blocks,
                              self.A_arrow_tip_block)
        else:
            self.algs.pobtsi(self.A_diagonal_blocks, self.A_lower_diagonal_blocks)


@pytest.mark.parametrize("arrays", ["numpy", "torch"])
@pytest.mark.parametrize("sparsity", ["bta", "bt"])
def test_serinv_solver_calling_sequence(arrays, sparsity):
    import torch

    from dalia_b200 import serinv_compat as sc

    n, b, a = 5, 150, 4
    rng = np.random.default_rng(11)
    D, L, Ab, T = bta_ref.random_bta(n, b, a, rng)
    if sparsity == "bt":
        Ab, T = np.zeros((n, 0, b)), np.zeros((0, 0))
    M = bta_ref.bta_to_dense(D, L, Ab, T) if a and sparsity == "bta" else bta_ref.bta_to_dense(
        D, L, np.zeros((n, 0, b)), np.zeros((0, 0)))
    N = M.shape[0]
    if arrays == "numpy":
        arrs, xp = [x.copy() for x in (D, L, Ab, T)], np
    else:
        arrs, xp = [torch.from_numpy(x.copy()).cuda() for x in (D, L, Ab, T)], torch
    solver = _SerinvSolverCalls(sc, *arrs)
    solver.cholesky(sparsity)
    assert abs(solver.logdet(sparsity, xp) - np.linalg.slogdet(M)[1]) < 1e-10 * abs(np.linalg.slogdet(M)[1])
    rhs0 = rng.standard_normal(N)
    rhs = rhs0.copy() if arrays == "numpy" else torch.from_numpy(rhs0.copy()).cuda()
    out = solver.solve(rhs, sparsity)
    assert out is rhs
    got = out if arrays == "numpy" else out.cpu().numpy()
    assert rel(got, np.linalg.solve(M, rhs0)) < 1e-10
    solver.selected_inversion(sparsity)
    S = np.linalg.inv(M)
    Dg = arrs[0] if arrays == "numpy" else arrs[0].cpu().numpy()
    Lg = arrs[1] if arrays == "numpy" else arrs[1].cpu().numpy()
    for i in range(n):
        assert rel(Dg[i], S[i * b:(i + 1) * b, i * b:(i + 1) * b]) < 1e-10
    for i in range(n - 1):
        assert rel(Lg[i], S[(i + 1) * b:(i + 2) * b, i * b:(i + 1) * b]) < 1e-10


def test_handle_on_second_device():
    """Kernel attributes and grid sizes are per device: a handle on device 1
    after device 0 was used factors correctly (skipped on one GPU)."""
    import torch

    from dalia_b200 import serinv_compat as sc

    if torch.cuda.device_count() < 2:
        pytest.skip("one GPU")
    D, L, Ab, T = bta_ref.random_bta(3, 130, 3, np.random.default_rng(2))
    ref = [x.copy() for x in (D, L, Ab, T)]
    bta_ref.pobtaf(*ref)
    for dev in (0, 1):
        with torch.cuda.device(dev):
            d = [torch.from_numpy(x.copy()).cuda(dev) for x in (D, L, Ab, T)]
            sc.pobtaf(*d)
            for g, r in zip(d, ref):
                assert rel(g.cpu().numpy(), r) < 1e-10
