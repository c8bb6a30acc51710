"""The oracle's teacher-forced stage replay (the CPU stage arithmetic of
sampling/stage.rs:134-240) against from-scratch recomputation: every proposal's pf_new is
the Pfaffian of the candidate configuration, and the inverse after a chain of accepted
rank-2 / rank-4 updates is the inverse of the final configuration."""
import numpy as np
import pytest

import oracle_lib as ol
import stage_moves as sm
from mvmc_lib import lattice, read_triples


def model(tmp_path, name, **over):
    lat = lattice()
    cfg = dict(lat.CONFIGS[name])
    cfg.update(over)
    nl, init, dims = lat.write_inputs(str(tmp_path / name), **cfg)
    d = ol.model_dims(nl)
    params = read_triples(init, d["npara"])
    return nl, d, params


@pytest.mark.parametrize("name,over", [("chain16", {}), ("square8", {}), ("square8", {"tp": -0.2, "n_up": 28})])
def test_oracle_stage_replay_matches_recomputation(tmp_path, name, over):
    nl, d, params = model(tmp_path, name, **over)
    ns, ne = d["nsite"], d["ne"]
    n = 2 * ne
    rng = np.random.default_rng(3)
    idx0 = sm.random_configuration(rng, ns, ne)
    ops, seq, final = sm.random_sequence(rng, idx0, ns, ne, 40)
    nqp = d["nqp"]
    out, inv = ol.stage_replay(nl, params, idx0, ops, seq, nqp, n)
    kinds = set()
    for k, op in enumerate(ops):
        if op[0] in (sm.PROPOSE_HOP, sm.PROPOSE_EX):
            kinds.add(int(op[0]))
            fresh, _ = ol.stage_replay(nl, params, seq[k], [[4, 0, 0, 0, 0, 0, 0]], seq[k][None, :], nqp, n)
            assert np.allclose(out[k], fresh[0], rtol=1e-9, atol=1e-12 * np.abs(fresh[0]).max()), k
    assert kinds == {sm.PROPOSE_HOP, sm.PROPOSE_EX}
    assert np.sum(ops[:, 0] == sm.ACCEPT_HOP) > 0 and np.sum(ops[:, 0] == sm.ACCEPT_EX) > 0
    _, fresh_inv = ol.stage_replay(nl, params, final, [[4, 0, 0, 0, 0, 0, 0]], final[None, :], nqp, n)
    assert np.allclose(inv, fresh_inv, rtol=1e-8, atol=1e-9 * np.abs(fresh_inv).max())
