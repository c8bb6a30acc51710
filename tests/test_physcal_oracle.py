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


def test_green_ratios_match_recomputed_amplitudes(tmp_path):
    """The one-electron and two-hop ratios of the Green functions against exp(Σ α Δc)·
    IP(x')/IP(x) with IP(x') from a fresh CalculateMAll of every moved configuration
    (the fixture's TwoBodyG list has no general two-hop term; this list reaches them)."""
    from mvmc_lib import green_term_mix, write_green_lists
    one, two, ex = green_term_mix(6, np.random.default_rng(3))
    nl = write_green_lists(os.path.join(D, "inputs"), str(tmp_path / "in"), one, two, ex)
    worst, n1, n2 = ol.green_identity(nl, ZQP)
    assert n1 > 1000 and n2 > 1000, (n1, n2)
    assert worst < 1e-11, worst


def test_two_body_ex_canonical_map(tmp_path):
    """OneBodyG is de-duplicated when TwoBodyGEx is present, and the factors that it lacks
    are appended in TwoBodyGEx order (types.rs:1169-1215)."""
    from mvmc_lib import write_green_lists
    one = [(0, 0, 1, 0), (0, 0, 1, 0), (2, 1, 3, 1)]
    ex = [(0, 0, 1, 0, 4, 1, 5, 1), (2, 1, 3, 1, 0, 0, 1, 0)]
    nl = write_green_lists(os.path.join(D, "inputs"), str(tmp_path / "in"), one, [], ex)
    g = ol.green_dims(nl)
    # (0 0 1 0), (2 1 3 1), then (5 1 4 1) and (1 0 0 0) from the factored terms
    assert (g["one"], g["ex"], g["two"]) == (4, 2, 0)
    ol.physcal_green(nl, ZQP, 1, 1, out_dir=str(tmp_path))
    rows = [line.split()[:4] for line in open(tmp_path / "zvo_cisajs_007.dat") if line.strip()]
    assert rows == [["0", "0", "1", "0"], ["2", "1", "3", "1"], ["5", "1", "4", "1"], ["1", "0", "0", "0"]]
