"""Queue of a whole FP64 factorisation in one launch (host logic, no GPU).

``bta_pobtaf_batched`` runs every block column of every matrix of a batch as
one launch when every arrow is at most 64 rows and DALIA_B200_PANEL_PERSIST=1:
the one-column queues of
columns 0, 1, ... follow one another, a column's previous-column tasks wait
per source tile for the previous column's block below (and arrow rows), the
tip tasks of a matrix's columns run in column order, and one chain CTA per
matrix finishes the chain tiles of its columns in order.  These tests read
the queue through ``bta_panel_task_list_all`` and check it against those
rules the way ``test_panel_queue.py`` checks one column: every tile once,
a topological order, and draining with any number of CTAs."""
import ctypes

import pytest

from dalia_b200 import _lib

DIAG, SUB, TRSM, TIP, PREV = 3, 4, 5, 6, 7


class Mat:
    def __init__(self, b, a, n, tip=True):
        self.b, self.a, self.n = b, a, n
        self.nq = (b + 63) // 64
        self.tip = tip and 0 < a <= 64

    def rows(self, c):
        """Tile rows of column c: diagonal block, block below (not in the last
        column), arrow."""
        return self.nq + (self.nq if c < self.n - 1 else 0) + (self.a + 63) // 64

    def has_prev(self, c, p):
        if c == 0:
            return False
        if p < self.nq:
            return True
        if c < self.n - 1 and p < 2 * self.nq:
            return False
        return self.a > 0

    def prev_row(self, c, p):
        """Row of column c-1 holding the previous-column source of row p."""
        if p < self.nq:
            return self.nq + p
        return 2 * self.nq + (p - self.nq - (self.nq if c < self.n - 1 else 0))


def task_list(mats, look=2, order=1):
    lib = _lib.load()
    k = len(mats)
    arr = lambda vals: (ctypes.c_int * k)(*vals)  # noqa: E731
    args = (k, arr([m.b for m in mats]), arr([m.a for m in mats]), arr([8 if m.tip else 0 for m in mats]),
            arr([m.n for m in mats]), look, order)
    cnt = ctypes.c_int(0)
    assert lib.bta_panel_task_list_all(*args, None, 0, ctypes.byref(cnt)) == _lib.BTA_ERR_INVALID
    out = (ctypes.c_int * (4 * cnt.value))()
    assert lib.bta_panel_task_list_all(*args, out, cnt.value, ctypes.byref(cnt)) == _lib.BTA_OK
    where = [(k, c) for k, m in enumerate(mats) for c in range(m.n)]
    tasks = []
    for i in range(cnt.value):
        g, kind, p, r = out[4 * i:4 * i + 4]
        mk, c = where[g]
        tasks.append((mk, c, kind, p, r))
    return tasks


def deps(m, c, kind, p, r):
    """What a task waits on: ('flag' | 'prv' | 'upd' | 'tip', column, p, r)."""
    if kind == PREV:
        return [("flag", c - 1, m.prev_row(c, q), k) for q in (p, r) for k in range(m.nq)]
    if kind == TIP:
        pa = m.rows(c) - 1
        return [("flag", c, pa, k) for k in range(m.nq)] + [("tip", c2, 0, 0) for c2 in range(c)]
    kmax = r - 1 if kind == DIAG else r
    d = []
    for k in range(max(kmax, 0)):
        d += [("flag", c, p, k), ("flag", c, r, k)]
    if m.has_prev(c, p):
        d.append(("prv", c, p, r))
    if kind == TRSM:
        d.append(("flag", c, r, r))
    return d


def produces(c, kind, p, r):
    return {PREV: ("prv", c, p, r), DIAG: ("upd", c, p, r), SUB: ("upd", c, p, r), TRSM: ("flag", c, p, r),
            TIP: ("tip", c, 0, 0)}[kind]


CASES = [
    [Mat(200, 6, 4) for _ in range(3)],
    [Mat(129, 5, 3), Mat(300, 0, 4), Mat(64, 6, 2)],
    [Mat(70, 3, 5), Mat(48, 2, 1)],
    [Mat(130, 64, 3, tip=True)],
]
LOOK_ORDER = [(look, order) for look in (1, 2, 4) for order in (0, 1)]


@pytest.mark.parametrize("ci", range(len(CASES)))
def test_every_tile_of_every_column_once(ci):
    mats = CASES[ci]
    tasks = task_list(mats)
    pos = {}
    for i, (mk, c, kind, p, r) in enumerate(tasks):
        key = (mk, c, "prev" if kind == PREV else ("tip" if kind == TIP else "tile"), p, r)
        assert key not in pos, f"duplicate {key}"
        pos[key] = i
    for mk, m in enumerate(mats):
        for c in range(m.n):
            for r in range(m.nq):
                for p in range(r, m.rows(c)):
                    t = pos.get((mk, c, "tile", p, r))
                    assert t is not None, (mk, c, p, r)
                    want = DIAG if p == r else (SUB if p == r + 1 and p < m.nq else TRSM)
                    assert tasks[t][2] == want
                    assert ((mk, c, "prev", p, r) in pos) == m.has_prev(c, p)
            assert ((mk, c, "tip", 0, 0) in pos) == m.tip


@pytest.mark.parametrize("look,order", LOOK_ORDER)
@pytest.mark.parametrize("ci", range(len(CASES)))
def test_whole_factorisation_queue_is_topological(ci, look, order):
    """Every input is produced earlier in the queue, directly or through the
    chain, which finishes (q, q-1) and (q, q) of its columns in order."""
    mats = CASES[ci]
    tasks = task_list(mats, look, order)
    where = {}
    for i, (mk, c, kind, p, r) in enumerate(tasks):
        where[(mk,) + produces(c, kind, p, r)] = i

    def chain_ready(mk, c, q):
        m = mats[mk]
        need = []
        for c2 in range(c + 1):
            for s in range(m.nq if c2 < c else q + 1):
                need.append(where[(mk, "upd", c2, s, s)])
                if s > 0:
                    need.append(where[(mk, "upd", c2, s, s - 1)])
        return max(need)

    for i, (mk, c, kind, p, r) in enumerate(tasks):
        m = mats[mk]
        for what, c2, dp, dr in deps(m, c, kind, p, r):
            if what == "flag" and (dp == dr or (dp == dr + 1 and dp < m.nq)):
                ready = chain_ready(mk, c2, dp)
            else:
                ready = where[(mk, what, c2, dp, dr)]
            assert ready < i, f"task {i} {(mk, c, kind, p, r)} waits on {(what, c2, dp, dr)}"


def simulate(mats, tasks, workers):
    done = set()
    chain = [[0, 0, 0] for _ in mats]  # column, step q, phase
    held, nxt, finished = [], 0, 0
    while True:
        moved = False
        while len(held) < workers and nxt < len(tasks):
            held.append(nxt)
            nxt += 1
            moved = True
        keep = []
        for i in held:
            mk, c, kind, p, r = tasks[i]
            if all((mk,) + d in done for d in deps(mats[mk], c, kind, p, r)):
                done.add((mk,) + produces(c, kind, p, r))
                finished += 1
                moved = True
            else:
                keep.append(i)
        held = keep
        for mk, m in enumerate(mats):
            c, q, ph = chain[mk]
            if c >= m.n:
                continue
            if ph == 0 and (q == 0 or (mk, "upd", c, q, q - 1) in done):
                if q > 0:
                    done.add((mk, "flag", c, q, q - 1))
                chain[mk][2] = ph = 1
                moved = True
            if ph == 1 and (mk, "upd", c, q, q) in done:
                done.add((mk, "flag", c, q, q))
                chain[mk] = [c, q + 1, 0] if q + 1 < m.nq else [c + 1, 0, 0]
                moved = True
        if finished == len(tasks) or not moved:
            return finished


@pytest.mark.parametrize("look,order", [(2, 1), (1, 0), (4, 1)])
@pytest.mark.parametrize("ci", range(len(CASES)))
@pytest.mark.parametrize("workers", [1, 2, 3, 7, 40, 148, 437])
def test_whole_factorisation_queue_drains_with_any_number_of_ctas(ci, workers, look, order):
    mats = CASES[ci]
    tasks = task_list(mats, look, order)
    assert simulate(mats, tasks, workers) == len(tasks)


def test_one_column_matrices_match_the_one_column_queue():
    """A batch of one-column matrices is the one-column queue itself."""
    from test_panel_queue import HAS_TIP, Inst
    from test_panel_queue import task_list as one_column

    mats = [Mat(200, 6, 1), Mat(129, 0, 1)]
    ref = one_column([Inst(200, 6, HAS_TIP), Inst(129, 0, 0)], 2, 1)
    assert [(mk, kind, p, r) for mk, c, kind, p, r in task_list(mats, 2, 1)] == ref


def test_rejects_bad_arguments():
    lib = _lib.load()
    n = ctypes.c_int(0)
    one = (ctypes.c_int * 1)(64)
    zero = (ctypes.c_int * 1)(0)
    big = (ctypes.c_int * 1)(65)
    assert lib.bta_panel_task_list_all(1, one, big, zero, one, 2, 1, None, 0, ctypes.byref(n)) == \
        _lib.BTA_ERR_INVALID  # arrows above 64 rows launch column by column
    assert lib.bta_panel_task_list_all(1, one, zero, zero, zero, 2, 1, None, 0, ctypes.byref(n)) == \
        _lib.BTA_ERR_INVALID
    assert lib.bta_panel_task_list_all(1, one, zero, zero, one, 2, 3, None, 0, ctypes.byref(n)) == \
        _lib.BTA_ERR_INVALID
