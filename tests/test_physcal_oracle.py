"""PhysCal Green functions of the oracle against the native C mVMC 1.4.0 outputs of the
reference's fixture tests/fixtures/native_c_physcal_181/hubbard_chain_real (and its
_mpi2 / _mpi4 runs: the same inputs on 2 and 4 chains seeded RndSeed + rank).

Bounds are the reference's own for this scenario (abs 1e-13, rel 1e-10,
crates/mvmc-cli/tests/issue181_native_c_physcal.rs:91-109); the files the oracle writes
carry the C layout (term columns, token count, terminal blank line)."""
import os

import numpy as np
import pytest

import oracle_lib as ol

D = os.path.join(ol.GOLDEN, "physcal_hubbard_chain_real")
NL = os.path.join(D, "inputs", "namelist.def")
ZQP = os.path.join(D, "zqp_opt.dat")


def close(got, ref):
    return np.all(np.abs(got - ref) <= np.maximum(1e-13, 1e-10 * np.abs(ref)))


@pytest.mark.parametrize("walkers,sub", [(1, "expected"), (2, "expected_mpi2"), (4, "expected_mpi4")])
def test_green_functions_match_native_c(walkers, sub):
    g, out = ol.physcal_green(NL, ZQP, 1, walkers)
    assert (g["one"], g["ex"], g["two"], g["blocks"]) == (12, 3, 36, 2)
    for b, idx in enumerate((7, 8)):
        ref = ol.read_physcal_expected(os.path.join(D, sub), idx)
        for key in ("energy", "one", "ex", "two"):
            assert close(out[key][b], ref[key]), (walkers, idx, key)


def test_physcal_files_have_the_c_layout(tmp_path):
    ol.physcal_green(NL, ZQP, 1, 1, out_dir=str(tmp_path))
    for idx in (7, 8):
        for kind in ("out", "var", "cisajs", "cisajscktalt", "cisajscktaltex"):
            name = f"zvo_{kind}_{idx:03d}.dat"
            got = open(tmp_path / name).read().split("\n")
            ref = open(os.path.join(D, "expected", name)).read().split("\n")
            assert len(got) == len(ref), name
            for a, b in zip(got, ref):
                ta, tb = a.split(), b.split()
                assert len(ta) == len(tb), (name, a, b)
                for x, y in zip(ta, tb):
                    if "e" in y or "." in y:
                        assert abs(float(x) - float(y)) <= max(1e-13, 1e-10 * abs(float(y))), (name, x, y)
                    else:
                        assert x == y, (name, a, b)
