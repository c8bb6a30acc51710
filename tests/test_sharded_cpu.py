"""Walker-sharded SR across ranks (mvmc-rs_b200/sharded.py) on CPU: two gloo ranks, each
with its own chains from the oracle, reduce the measurement sums and every CG product;
both ranks reach the same update, equal to one process holding all chains and to the
oracle's CG on the union of the samples."""
import os
import sys
import tempfile

import numpy as np
import pytest

import oracle_lib as ol
from mvmc_lib import ROOT, lattice

sys.path.insert(0, os.path.join(ROOT, "mvmc-rs_b200"))
import sharded  # noqa: E402

CFG = dict(nsrcg=1, red_cut=1e-8, step_dt=0.02, sta_del=0.02, cg_tol=1e-9, cg_max_iter=500, diag_scale=0,
           cg_fallback=0, cg_abort=0)


class OracleLocal:
    """One rank's chains measured by the oracle (step 1 of an optimisation)."""

    def __init__(self, nl, init, walkers, seed):
        dims, ref = ol.opt_step1_walkers(nl, walkers, seed=seed, initial_def=init)
        self.npara = dims["npara"]
        wc = ref["energy"][0]
        tot = np.concatenate([ref["energy"], ref["ho"], ref["oo"]])
        self.sums = np.concatenate([[wc], tot[1:] * wc])
        self.store = ref["ostore"]
        self.applied = None

    def measure_sums(self):
        return self.sums.copy()

    def sr_config(self):
        return dict(CFG, npara=self.npara), np.ones(2 * self.npara, dtype=np.int32)

    def sr_gather(self, mapping):
        self.oa = self.store[:, np.asarray(mapping) + 1]

    def sr_local_product(self, v):
        return self.oa.T @ (self.oa @ v)

    def sr_local_product_device(self, v, z, stream):
        import torch
        z.copy_(torch.from_numpy(self.oa.T @ (self.oa @ v.numpy())))

    def sr_apply(self, mapping, x):
        self.applied = (np.asarray(mapping), np.asarray(x))


def inputs(tmp):
    lat = lattice()
    cfg = dict(lat.CONFIGS["chain16"])
    cfg.update(samples=4, interval=2)
    nl, init, _ = lat.write_inputs(os.path.join(tmp, "in"), **cfg)
    return nl, init


def _rank(rank, world, port, nl, init, out, device_form=False):
    import torch
    import torch.distributed as dist
    import datetime
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local = OracleLocal(nl, init, 2, 100 + 2 * rank)

        def reduce(a):
            t = torch.from_numpy(np.array(a, dtype=np.float64))
            dist.all_reduce(t)
            return t.numpy()

        if device_form:
            info = sharded.sr_step_device(local, reduce, dist.all_reduce, "cpu")
        else:
            info = sharded.sr_step(local, reduce)
        np.savez(os.path.join(out, f"rank{rank}.npz"), mapping=local.applied[0], x=local.applied[1],
                 info=np.array([info["nsmat"], info["info"]]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_one_process_and_the_oracle():
    import torch.multiprocessing as mp
    tmp = tempfile.mkdtemp()
    nl, init = inputs(tmp)
    port = 29500 + os.getpid() % 1000
    mp.spawn(_rank, args=(2, port, nl, init, tmp), nprocs=2, join=True)
    r0 = np.load(os.path.join(tmp, "rank0.npz"))
    r1 = np.load(os.path.join(tmp, "rank1.npz"))
    assert np.array_equal(r0["mapping"], r1["mapping"])
    assert np.array_equal(r0["x"], r1["x"])  # identical numbers on every rank
    one = OracleLocal(nl, init, 4, 100)
    info = sharded.sr_step(one, lambda a: a)
    assert np.array_equal(one.applied[0], r0["mapping"])
    assert info["info"] >= 0 and int(r0["info"][1]) >= 0
    # both solves stop at |r| < n·tol (tol 1e-9); the summation order of the ranks' sums
    # moves the solution only within that tolerance
    scale = np.abs(one.applied[1]).max()
    assert np.allclose(r0["x"], one.applied[1], rtol=1e-6, atol=1e-6 * scale)
    # the oracle's CG on the union of the samples (fixed operands)
    ops = sharded.operands(one.sums)
    m = one.applied[0]
    idx = m + 1
    var = ops["diag"][idx] - ops["mean"][idx] ** 2
    g = -2.0 * CFG["step_dt"] * (ops["ho"][idx] - ops["ho"][0] * ops["mean"][idx])
    st, x, _ = ol.cg_fixed(ops["mean"][idx], var, one.store[:, idx], g, 1.0 / ops["wc"], CFG["sta_del"],
                           CFG["cg_tol"], CFG["cg_max_iter"], False)
    assert abs(st - info["info"]) <= 2  # iteration counts at the same tolerance
    assert np.allclose(one.applied[1], x, rtol=1e-6, atol=1e-6 * scale)


def test_cg_recurrence_statuses_match_oracle_on_fixed_operands():
    rng = np.random.default_rng(3)
    ns, na = 60, 12
    o = rng.normal(size=(ns, na))
    mean, diag = o.mean(0), o.var(0)
    g = rng.normal(size=na)
    for limit in (1, 3, 25):
        def apply(v):
            return (o.T @ (o @ v)) / ns - float(mean @ v) * mean + 1e-5 * diag * v
        x, st = sharded.cg_solve(apply, g, diag, 1e-5, 0.0, limit, False)
        sto, xo, _ = ol.cg_fixed(mean, diag, o, g, 1.0 / ns, 1e-5, 0.0, limit, False)
        assert st == sto
        assert np.allclose(x, xo, rtol=1e-9, atol=1e-12)


def _rank_device_form(rank, world, port, nl, init, out):
    _rank(rank, world, port, nl, init, out, device_form=True)


def test_two_gloo_ranks_with_tensor_vectors_match_the_array_form():
    """sr_step_device (CG vectors as torch tensors, z reduced in place by all_reduce on the
    tensor): both ranks apply identical updates, equal within the CG tolerance to the
    array form on one process holding all chains, with the same active set."""
    import torch.multiprocessing as mp
    tmp = tempfile.mkdtemp()
    nl, init = inputs(tmp)
    port = 29600 + os.getpid() % 1000
    mp.spawn(_rank_device_form, args=(2, port, nl, init, tmp), nprocs=2, join=True)
    r0 = np.load(os.path.join(tmp, "rank0.npz"))
    r1 = np.load(os.path.join(tmp, "rank1.npz"))
    assert np.array_equal(r0["mapping"], r1["mapping"])
    assert np.array_equal(r0["x"], r1["x"])
    one = OracleLocal(nl, init, 4, 100)
    info = sharded.sr_step(one, lambda a: a)
    assert np.array_equal(one.applied[0], r0["mapping"]) and info["info"] >= 0 and int(r0["info"][1]) >= 0
    scale = np.abs(one.applied[1]).max()
    assert np.allclose(r0["x"], one.applied[1], rtol=1e-6, atol=1e-6 * scale)
