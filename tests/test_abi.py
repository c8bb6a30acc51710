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


@pytest.mark.parametrize("name", ["chain16", "square8", "square16", "square16_sr"])
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
