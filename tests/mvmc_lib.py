"""Loads the product binding (mvmc-rs_b200/mvmc_b200.py) for the tests."""
import importlib.util
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_MOD = None


def mvmc():
    global _MOD
    if _MOD is None:
        spec = importlib.util.spec_from_file_location(
            "mvmc_b200", os.path.join(ROOT, "mvmc-rs_b200", "mvmc_b200.py"))
        _MOD = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(_MOD)
    return _MOD


def read_triples(path, npara):
    """Parameter means of a zqp_opt.dat / initial.def file (last 6 + 3·NPara floats)."""
    vals = np.array([float(t) for t in open(path).read().split()])
    vals = vals[len(vals) - (6 + 3 * npara):]
    return vals[6::3][:npara]


def lattice():
    """The synthetic Hubbard input generator (mvmc-rs_b200/lattice.py)."""
    spec = importlib.util.spec_from_file_location("lattice", os.path.join(ROOT, "mvmc-rs_b200", "lattice.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def write_green_lists(src_inputs, dst, one=(), two=(), ex=()):
    """Copy an Expert-mode input directory and give it OneBodyG / TwoBodyG / TwoBodyGEx
    lists: one = [(i, s, j, t)], two and ex = [(i, s, j, t, k, u, l, v)]. Returns the
    new namelist path."""
    import shutil
    os.makedirs(dst, exist_ok=True)
    for name in os.listdir(src_inputs):
        if name not in ("greenone.def", "greentwo.def", "greentwoex.def"):
            shutil.copyfile(os.path.join(src_inputs, name), os.path.join(dst, name))
    lines = [line for line in open(os.path.join(dst, "namelist.def"))
             if line.split()[:1] not in (["OneBodyG"], ["TwoBodyG"], ["TwoBodyGEx"])]
    for key, fname, rows in (("OneBodyG", "greenone.def", one), ("TwoBodyG", "greentwo.def", two),
                             ("TwoBodyGEx", "greentwoex.def", ex)):
        if not rows:
            continue
        with open(os.path.join(dst, fname), "w") as f:
            f.write("=" * 30 + f"\nN{key} {len(rows)}\n" + "=" * 30 + "\n" + "=" * 30 + "\n" + "=" * 30 + "\n")
            for r in rows:
                f.write(" ".join(f"{v:5d}" for v in r) + "\n")
        lines.append(f"{key} {fname}\n")
    with open(os.path.join(dst, "namelist.def"), "w") as f:
        f.writelines(lines)
    return os.path.join(dst, "namelist.def")


def green_term_mix(ns, rng, n_two=300):
    """One-body terms over every (i, s, j, t) and TwoBodyG terms that reach every branch of
    the two-body reduction: random index tuples plus tuples with each coincidence."""
    one = [(i, s, j, t) for s in (0, 1) for t in (0, 1) for i in range(ns) for j in range(ns)]
    two = []
    for _ in range(n_two):
        i, j, k, l = (int(v) for v in rng.integers(0, ns, 4))
        s, u = (int(v) for v in rng.integers(0, 2, 2))
        two.append((i, s, j, s, k, u, l, u))
    for s in (0, 1):
        for u in (0, 1):
            a, b, c = (int(v) for v in rng.choice(ns, 3, replace=False))
            for i, j, k, l in ((a, b, c, c), (a, b, c, b), (a, b, c, a), (a, b, b, a), (a, b, b, c),
                               (a, b, a, c), (a, a, b, c), (a, a, b, b), (a, b, c, c)):
                two.append((i, s, j, s, k, u, l, u))
    ex = [one[int(rng.integers(len(one)))][:4] + one[int(rng.integers(len(one)))][:4] for _ in range(10)]
    return one, two, ex
