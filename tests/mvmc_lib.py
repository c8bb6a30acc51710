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
