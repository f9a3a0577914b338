"""Load the golden fixtures written by ``tests/golden/make_golden.py``."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz"), allow_pickle=False))


def problem(g):
    from dalia_b200 import synth

    ns, nt, nb, no, seed = (int(v) for v in g["shape"])
    prob = synth.make_problem(ns, nt, nb, no, tuple(g["theta"]), str(g["likelihood"]), seed=seed)
    # the generator must reproduce the inputs the fixture was made from
    for nm in ("c0", "g1", "g2", "g3", "m0", "m1", "m2", "a_st"):
        d = getattr(prob, nm).tocsc().data
        np.testing.assert_allclose([d.sum(), (d * d).sum(), d.size], g[f"chk_{nm}"], rtol=1e-12)
    np.testing.assert_allclose(
        [prob.y.sum(), (prob.y ** 2).sum(), prob.y.size], g["chk_y"], rtol=1e-12)
    return prob


def coreg_problem(g):
    from dalia_b200 import synth

    ns, nt, nv, nb, no, seed = (int(v) for v in g["shape"])
    prob = synth.make_coregional_problem(ns, nt, nv, nb, no, tuple(g["theta"]), seed=seed)
    for nm in ("c0", "g1", "g2", "g3", "m0", "m1", "m2"):
        d = getattr(prob, nm).tocsc().data
        np.testing.assert_allclose([d.sum(), (d * d).sum(), d.size], g[f"chk_{nm}"], rtol=1e-12)
    for v in range(nv):
        d = prob.a_st[v].tocsc().data
        np.testing.assert_allclose([d.sum(), (d * d).sum(), d.size], g[f"chk_a_st{v}"], rtol=1e-12)
        np.testing.assert_allclose([prob.y[v].sum(), (prob.y[v] ** 2).sum(), prob.y[v].size], g[f"chk_y{v}"],
                                   rtol=1e-12)
    return prob


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
