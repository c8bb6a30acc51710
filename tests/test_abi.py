"""CPU checks of the product boundary: the C ABI library loads and exports every entry
point include/mvmc_b200.h declares; the input generator round-trips through the reader."""
import ctypes
import os
import re
import sys

import pytest

import oracle_lib as ol
from mvmc_lib import ROOT, mvmc


def declared_functions():
    text = open(os.path.join(ROOT, "include", "mvmc_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mvmc_b200_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_entry_point():
    lib = mvmc().lib()
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) <= set(mvmc().EXPORTS) | set(names)


def test_binding_lists_every_declared_entry_point():
    assert set(declared_functions()) == set(mvmc().EXPORTS)


def test_default_options():
    o = mvmc().default_options()
    assert o.walkers == 1 and o.precision == 64 and o.seed < 0


@pytest.mark.parametrize("name", ["chain16", "square8", "square16", "square16_sr", "physcal8"])
def test_lattice_inputs_parse(tmp_path, name):
    sys.path.insert(0, os.path.join(ROOT, "mvmc-rs_b200"))
    import lattice
    nl, ini, dims = lattice.write_inputs(str(tmp_path / name), **lattice.CONFIGS[name])
    d = ol.model_dims(nl)
    assert d["nsite"] == dims["nsite"] and d["npara"] == dims["npara"] and d["nqp"] == dims["nqp"]
    assert 2 * d["ne"] == dims["n"]


def test_lattice_chain_runs_on_the_oracle(tmp_path):
    sys.path.insert(0, os.path.join(ROOT, "mvmc-rs_b200"))
    import lattice
    nl, ini, dims = lattice.write_inputs(str(tmp_path / "c"), **lattice.CONFIGS["chain16"])
    d, out = ol.opt_step1_walkers(nl, 2, seed=12345, initial_def=ini)
    assert out["energy"][0] == 2.0
    assert -20.0 < out["energy"][1] / 2 < 20.0


def test_entry_points_reject_bad_arguments_before_any_device_call():
    """Argument checks of the ABI (status < 0, no CUDA call): odd or non-positive matrix
    sides, missing pointers and handles."""
    m = mvmc()
    lib = m.lib()
    buf = (ctypes.c_double * 64)()
    st = (ctypes.c_int * 4)()
    assert lib.mvmc_b200_pfinv_batch(buf, 3, 1, buf, buf, st) == -1  # odd n
    assert lib.mvmc_b200_pfinv_batch(buf, 0, 1, buf, buf, st) == -1
    assert lib.mvmc_b200_pfinv_batch(None, 4, 1, buf, buf, st) == -1
    sizes = (ctypes.c_int * 2)(4, 5)
    assert lib.mvmc_b200_pfinv_batch_mixed(buf, sizes, 2, 64, buf, buf, st) == -1
    assert lib.mvmc_b200_pfinv_batch_mixed(buf, None, 2, 64, buf, buf, st) == -1
    dims = (ctypes.c_int * 8)()
    assert lib.mvmc_b200_dims(None, dims) == -1
    assert lib.mvmc_b200_green_dims(None, dims) == -1
    out = ctypes.c_void_p()
    assert lib.mvmc_b200_create(None, None, None, ctypes.byref(out)) == -1
    assert lib.mvmc_b200_physcal_create(None, None, None, ctypes.byref(out)) == -1
    assert lib.mvmc_b200_run_physcal(None, None, None, None) == -1


def test_reader_rejects_inputs_outside_the_path(tmp_path):
    """The Expert-mode reader (shared by the library and the oracle) refuses terms the real
    sz-conserved path does not cover and malformed Green lists, with a message."""
    from mvmc_lib import write_green_lists
    d = os.path.join(ol.GOLDEN, "physcal_hubbard_chain_real", "inputs")
    nl = write_green_lists(d, str(tmp_path / "a"))
    with open(nl, "a") as f:
        f.write("PairHop pairhop.def\n")
    with pytest.raises(RuntimeError, match="PairHop"):
        ol.green_dims(nl)
    nl = write_green_lists(d, str(tmp_path / "b"), one=[(0, 0, 1, 0)])
    path = os.path.join(str(tmp_path / "b"), "greenone.def")
    text = open(path).read().replace("NOneBodyG 1", "NOneBodyG 2")
    open(path, "w").write(text)
    with pytest.raises(RuntimeError, match="row count"):
        ol.green_dims(nl)
    nl = write_green_lists(d, str(tmp_path / "c"), one=[(0, 2, 1, 0)])
    with pytest.raises(RuntimeError, match="out of range"):
        ol.green_dims(nl)
