"""Task queue of the factorisation's block-column kernel (host logic, no GPU).

One launch factors a block column of every matrix of a batch as a tile DAG:
a chain CTA per matrix finishes the tiles (q, q-1) and (q, q) in order, and
the other CTAs claim tile tasks from a queue in a fixed order and wait, by
release/acquire flags, for the tiles they read.  A claimed task that waits on
a task nobody can claim any more would hang the launch (the kernel's waits
are bounded and then raise an error), so the order must let every task
finish whatever the number of CTAs.  These tests read the queue through
``bta_panel_task_list`` and check it against the kernel's dependency rules:

* every tile at or below the diagonal has exactly one task of the right kind,
  and the previous block column's term of a tile (a task without
  dependencies) exactly when that tile receives one, queued before it;
* every task's inputs come from tasks earlier in the queue or from the chain,
  whose own inputs are earlier still (a topological order);
* claiming in queue order with 1 to 437 CTAs always drains the queue.
"""
import ctypes

import pytest

from dalia_b200 import _lib

DIAG, SUB, TRSM, TIP, PREV = 3, 4, 5, 6, 7
HAS_L, HAS_PREV, HAS_ABPREV, HAS_TIP = 1, 2, 4, 8


class Inst:
    def __init__(self, b, a, flags):
        self.b, self.a, self.flags = b, a, flags
        self.nq = (b + 63) // 64
        self.has_l = bool(flags & HAS_L)
        self.rows = self.nq + (self.nq if self.has_l else 0) + (a + 63) // 64
        self.tip = bool(flags & HAS_TIP) and 0 < a <= 64

    def has_prev(self, p):
        """Whether tile row p receives the previous block column's term."""
        if not self.flags & HAS_PREV:
            return False
        if p < self.nq:
            return True
        if self.has_l and p < 2 * self.nq:
            return False
        return bool(self.flags & HAS_ABPREV) and self.a > 0


# queue lookaheads the autotuner chooses from (2 is the default), and the two
# queue orders (0: column by column, 1: the chain's critical tasks ahead)
LOOKAHEADS = [1, 2, 4]
ORDERS = [0, 1]
LOOK_ORDER = [(look, order) for look in LOOKAHEADS for order in ORDERS]


def task_list(insts, lookahead=None, order=0):
    lib = _lib.load()
    k = len(insts)
    b = (ctypes.c_int * k)(*[i.b for i in insts])
    a = (ctypes.c_int * k)(*[i.a for i in insts])
    f = (ctypes.c_int * k)(*[i.flags for i in insts])
    n = ctypes.c_int(0)
    if lookahead is None:
        call = lambda out, cap: lib.bta_panel_task_list(k, b, a, f, out, cap, ctypes.byref(n))  # noqa: E731
    else:
        call = lambda out, cap: lib.bta_panel_task_list_ex(k, b, a, f, lookahead, order, out, cap,  # noqa: E731
                                                            ctypes.byref(n))
    assert call(None, 0) == _lib.BTA_ERR_INVALID
    out = (ctypes.c_int * (4 * n.value))()
    assert call(out, n.value) == _lib.BTA_OK
    return [tuple(out[4 * i:4 * i + 4]) for i in range(n.value)]


def deps(inst, kind, p, r):
    """Flags a task reads: ('flag', p, k) final tiles, ('prv', p, r) terms."""
    d = []
    if kind == PREV:
        return d
    if kind == TIP:
        pa = inst.rows - 1
        return [("flag", pa, k) for k in range(inst.nq)]
    kmax = r - 1 if kind == DIAG else r
    for k in range(max(kmax, 0)):
        d.append(("flag", p, k))
        d.append(("flag", r, k))
    if inst.has_prev(p):
        d.append(("prv", p, r))
    if kind == TRSM:
        d.append(("flag", r, r))
    return d


def produces(kind, p, r):
    return {PREV: ("prv", p, r), DIAG: ("upd", p, r), SUB: ("upd", p, r), TRSM: ("flag", p, r)}.get(kind)


CASES = [
    [Inst(320, 6, HAS_L | HAS_PREV | HAS_ABPREV | HAS_TIP) for _ in range(6)],
    [Inst(320, 6, HAS_L | HAS_TIP)],
    [Inst(320, 6, HAS_PREV | HAS_ABPREV | HAS_TIP)],
    [Inst(129, 70, HAS_L | HAS_PREV | HAS_ABPREV), Inst(300, 0, HAS_L | HAS_PREV), Inst(64, 6, HAS_TIP)],
    [Inst(70, 3, HAS_L | HAS_PREV | HAS_ABPREV | HAS_TIP), Inst(48, 2, HAS_PREV | HAS_ABPREV | HAS_TIP)],
]


@pytest.mark.parametrize("look,order", LOOK_ORDER)
@pytest.mark.parametrize("ci", range(len(CASES)))
def test_queue_covers_every_tile_once(ci, look, order):
    insts = CASES[ci]
    tasks = task_list(insts, look, order)
    pos = {}
    for i, (m, kind, p, r) in enumerate(tasks):
        key = (m, "prev" if kind == PREV else ("tip" if kind == TIP else "tile"), p, r)
        assert key not in pos, f"duplicate task {key}"
        pos[key] = i
    for m, inst in enumerate(insts):
        for r in range(inst.nq):
            for p in range(r, inst.rows):
                t = pos.get((m, "tile", p, r))
                assert t is not None, f"tile ({p}, {r}) of matrix {m} has no task"
                kind = tasks[t][1]
                want = DIAG if p == r else (SUB if p == r + 1 and p < inst.nq else TRSM)
                assert kind == want
                pv = pos.get((m, "prev", p, r))
                assert (pv is not None) == inst.has_prev(p)
                if pv is not None:
                    assert pv < t
        assert ((m, "tip", 0, 0) in pos) == inst.tip
    n_tiles = sum(sum(inst.rows - r for r in range(inst.nq)) for inst in insts)
    n_prev = sum(sum(inst.has_prev(p) for r in range(inst.nq) for p in range(r, inst.rows)) for inst in insts)
    assert len(tasks) == n_tiles + n_prev + sum(inst.tip for inst in insts)


@pytest.mark.parametrize("look,order", LOOK_ORDER)
@pytest.mark.parametrize("ci", range(len(CASES)))
def test_queue_is_topological(ci, look, order):
    """Inputs of every task are produced earlier in the queue, directly or
    through the chain (whose step q consumes the tasks of tiles (q, q-1) and
    (q, q))."""
    insts = CASES[ci]
    tasks = task_list(insts, look, order)
    where = {}
    for i, (m, kind, p, r) in enumerate(tasks):
        out = produces(kind, p, r)
        if out:
            where[(m,) + out] = i

    def ready_at(m, dep):
        """Queue position by which the flag `dep` is produced (chain flags:
        by the chain-input tasks of their step and everything before)."""
        what, p, r = dep
        if what == "flag" and (p == r or p == r + 1 and p < insts[m].nq):
            q = p  # chain step q finishes (q, q-1) and (q, q)
            needed = [where[(m, "upd", s, s)] for s in range(q + 1)]
            needed += [where[(m, "upd", s, s - 1)] for s in range(1, q + 1)]
            return max(needed)
        return where[(m, what, p, r)]

    for i, (m, kind, p, r) in enumerate(tasks):
        for dep in deps(insts[m], kind, p, r):
            assert ready_at(m, dep) < i, f"task {i} {kind, p, r} waits on {dep}"


def simulate(insts, tasks, workers):
    """Claim in queue order with `workers` CTAs; a claimed task finishes once
    all its inputs exist; the chains advance whenever their inputs exist.
    Returns the number of finished tasks when nothing can move any more."""
    done = set()
    chain = [0] * len(insts)
    phase = [0] * len(insts)
    held = []
    nxt = 0
    finished = 0
    while True:
        moved = False
        while len(held) < workers and nxt < len(tasks):
            held.append(nxt)
            nxt += 1
            moved = True
        keep = []
        for i in held:
            m, kind, p, r = tasks[i]
            if all((m,) + d in done for d in deps(insts[m], kind, p, r)):
                out = produces(kind, p, r)
                if out:
                    done.add((m,) + out)
                finished += 1
                moved = True
            else:
                keep.append(i)
        held = keep
        for m, inst in enumerate(insts):
            q = chain[m]
            if q >= inst.nq:
                continue
            if phase[m] == 0:
                if q == 0 or (m, "upd", q, q - 1) in done:
                    if q > 0:
                        done.add((m, "flag", q, q - 1))
                    phase[m] = 1
                    moved = True
            if phase[m] == 1 and (m, "upd", q, q) in done:
                done.add((m, "flag", q, q))
                phase[m] = 0
                chain[m] += 1
                moved = True
        if finished == len(tasks) or not moved:
            return finished


@pytest.mark.parametrize("look,order", LOOK_ORDER)
@pytest.mark.parametrize("ci", range(len(CASES)))
@pytest.mark.parametrize("workers", [1, 2, 3, 7, 40, 148, 296, 437])
def test_queue_drains_with_any_number_of_ctas(ci, workers, look, order):
    insts = CASES[ci]
    tasks = task_list(insts, look, order)
    assert simulate(insts, tasks, workers) == len(tasks)


def test_default_lookahead_is_two():
    for insts in CASES:
        assert task_list(insts) == task_list(insts, 2, 0)


def test_chain_ahead_order_puts_critical_tasks_first():
    """In the chain-ahead order, the solve of tile (r+2, r) and the chain's
    inputs of step r+2 precede every other solve of column r."""
    insts = CASES[0]
    tasks = task_list(insts, 2, 1)
    pos = {(m, kind, p, r): i for i, (m, kind, p, r) in enumerate(tasks)}
    for m, inst in enumerate(insts):
        for r in range(inst.nq - 2):
            crit = max(pos[(m, TRSM, r + 2, r)], pos[(m, SUB, r + 2, r + 1)], pos[(m, DIAG, r + 2, r + 2)])
            for p in range(r + 3, inst.rows):
                assert crit < pos[(m, TRSM, p, r)]


def test_task_list_rejects_bad_arguments():
    lib = _lib.load()
    n = ctypes.c_int(0)
    one = (ctypes.c_int * 1)(64)
    zero = (ctypes.c_int * 1)(0)
    assert lib.bta_panel_task_list(0, one, zero, zero, None, 0, ctypes.byref(n)) == _lib.BTA_ERR_INVALID
    assert lib.bta_panel_task_list(1, zero, zero, zero, None, 0, ctypes.byref(n)) == _lib.BTA_ERR_INVALID
    assert lib.bta_panel_task_list_ex(1, one, zero, zero, 0, 0, None, 0, ctypes.byref(n)) == _lib.BTA_ERR_INVALID
    assert lib.bta_panel_task_list_ex(1, one, zero, zero, 2, 2, None, 0, ctypes.byref(n)) == _lib.BTA_ERR_INVALID


def noalloc_order(b, a, has_l):
    """The closed form the allocation-free factorisation writes on the device
    (``write_tasks_kernel`` in ``noalloc.cu``): tile column r holds the
    diagonal tile, then tiles r+1 .. rows-1 in order, the tile right below the
    diagonal tile going to the chain CTA."""
    inst = Inst(b, a, HAS_L if has_l else 0)
    out = []
    for r in range(inst.nq):
        out.append((0, DIAG, r, r))
        for p in range(r + 1, inst.rows):
            out.append((0, SUB if (p == r + 1 and p < inst.nq) else TRSM, p, r))
    assert len(out) == inst.nq * inst.rows - inst.nq * (inst.nq - 1) // 2
    return out


@pytest.mark.parametrize("b", [1, 63, 64, 65, 200, 1500, 2048])
@pytest.mark.parametrize("a", [0, 5, 64, 100, 128])
@pytest.mark.parametrize("has_l", [False, True])
def test_noalloc_device_task_order_matches_queue(b, a, has_l):
    assert task_list([Inst(b, a, HAS_L if has_l else 0)]) == noalloc_order(b, a, has_l)
