"""Benchmark of the VMC sampling + SR hot path on one or more B200s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config square8]
                    [--precision 32|64] [--impl ours|reference]

Engine workloads (chain16, square8, square16, square16_sr; mvmc-rs_b200/lattice.py): a
step is one SR step — resident sampling (burn-in chain of NVMCSample + 1 blocks of
NVMCInterval sweeps per walker), measurement with the adjoint O rows, SR-CG and the
parameter update. `value` is Metropolis sweeps/s of the whole job with the model resident
on the device. The default line is the plain FP64 path; the mixed path (FP32 inverse
updates, FP64 refresh every --refresh sweeps and after guard-tripping moves) is timed
beside it on the same workload and seeds (`mixed_path`), and `accuracy` compares one
fresh sample + measurement of the two.

PhysCal workload (physcal8): the square8 model with fixed parameters; a step is one data
block — resident sampling of one sample per walker, then the measurement in the PhysCal
form: energy plus the one-body Green function of every same-spin site pair and the
density-density function of every site pair (8192 + 16384 terms); `value` is samples/s.

Pfaffian workloads (pfinv64, pfinv_mix): a step is one batched Pfaffian + inverse launch
over B = 8192 (8190 for the five-size mix) seeded skew planes; `value` is planes/s.

`e2e` times the same steps through the public C ABI calls with host buffers, host↔device
copies inside the timed region. For N > 1 (torchrun) every rank samples and measures its
own walker ensemble (seeds offset by rank × walkers, no collective on that path) and the
SR step is sharded: the measurement sums and every CG product are added across ranks
over NCCL (mvmc-rs_b200/sharded.py), so all ranks apply the same update.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "mvmc-rs_b200"))

WALKERS = {"chain16": 256, "square8": 4096, "square16": 2048, "square16_sr": 8192}
PFINV = {"pfinv64": [64] * 8192, "pfinv_mix": [32, 48, 64, 96, 128] * 1638}
METRIC = "Metropolis sweeps/s & SR-step time: mixed vs FP64 path on 1 B200 at |dE|/N<=1e-6"
# DRAM bytes (read + write) per walker-sweep of k_sample from an ncu capture of a small
# case of the same kernel instance (profiles/k_sample_fp64_square8_w296.txt: 2.594 GB over
# 296 walkers x 4 sweeps), scaled to a launch by walker-sweeps.
SAMPLE_DRAM_PER_WALKER_SWEEP = {("square8", 64): 2.607e9 / (296 * 4)}
PFINV_METRIC = "Pfaffian+inverse/s (batched skew FP64)"
PHYSCAL = {"physcal8": 4096}
PHYSCAL_METRIC = "PhysCal samples/s (energy + one- and two-body Green functions, FP64)"


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def start_clock_sampler(path):
    try:
        return subprocess.Popen(
            ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
             "--format=csv,noheader,nounits", "-lms", "200"],
            stdout=open(path, "w"), stderr=subprocess.DEVNULL)
    except OSError:
        return None


def stop_clock_sampler(sampler):
    if sampler is not None:
        sampler.terminate()
        sampler.wait()


def summarize_clocks(path, device):
    rows = []
    try:
        for line in open(path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9 and parts[0] == str(device):
                rows.append(parts)
    except OSError:
        return None
    if not rows:
        return None
    sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
    reasons = set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for r in rows:
        for k, name in enumerate(names):
            if r[5 + k].lower().startswith("active"):
                reasons.add(name)
    return {"sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
            "reasons": sorted(reasons), "samples": len(rows)}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ----------------------------------------------------------------------------------------
# CPU legs: the oracle (C++ restatement of the reference CPU path) on the host cores.
# ----------------------------------------------------------------------------------------
def _oracle_lib():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    ol.lib()
    return ol


def _engine_job(args):
    namelist, initial_def, walkers, seed = args
    _oracle_lib().opt_step1_walkers(namelist, walkers, seed=seed, initial_def=initial_def)
    return 0


_PF_DATA = []


def _pfinv_init(sizes, per):
    """Worker set-up: this process's own seeded planes (generated once, not timed)."""
    global _PF_DATA
    _oracle_lib()
    rng = np.random.default_rng(os.getpid())
    _PF_DATA = [(skew_planes(rng, n, per).ravel(), n, per) for n in sorted(set(sizes))]


def _pfinv_job(_):
    ol = _oracle_lib()
    for x, n, per in _PF_DATA:
        ol.pfinv_batch(x, n, per)
    return 0


class CpuPool:
    """One oracle process per host core (spawned before any GPU work, so no process is
    forked from a CUDA context); only the map over the jobs is timed."""

    def __init__(self, procs, initializer=None, initargs=()):
        import multiprocessing as mp
        self.procs = procs
        self.pool = mp.get_context("spawn").Pool(procs, initializer=initializer, initargs=initargs)

    def time(self, fn, jobs):
        t0 = time.perf_counter()
        self.pool.map(fn, jobs, chunksize=1)
        return time.perf_counter() - t0

    def close(self):
        self.pool.close()
        self.pool.join()


def cpu_engine_time(namelist, initial_def, walkers):
    """One process, `walkers` chains of one SR step of the oracle."""
    _oracle_lib()
    t0 = time.perf_counter()
    _engine_job((namelist, initial_def, walkers, 12345))
    return time.perf_counter() - t0


def cpu_pfinv_time(sizes, per):
    """One process, `per` planes of each size."""
    _pfinv_init(sizes, per)
    t0 = time.perf_counter()
    _pfinv_job(0)
    return time.perf_counter() - t0


def skew_planes(rng, n, planes):
    """A_ij ~ N(0,1) for i < j, A_ji = -A_ij, plus 0.5·J (J = diag of [[0,1],[-1,0]] blocks);
    column-major planes (the transpose of a skew matrix is its negative, so the row-major
    draw is stored negated)."""
    u = np.triu(rng.standard_normal((planes, n, n)), 1)
    x = u - np.transpose(u, (0, 2, 1))
    i = np.arange(0, n, 2)
    x[:, i, i + 1] += 0.5
    x[:, i + 1, i] -= 0.5
    return np.ascontiguousarray(np.transpose(x, (0, 2, 1)))


# ----------------------------------------------------------------------------------------
# Engine workloads.
# ----------------------------------------------------------------------------------------
def engine_inputs(args, rank):
    import lattice
    cfg = dict(lattice.CONFIGS[args.config])
    if args.interval:
        cfg["interval"] = args.interval
    if args.direct:
        cfg["nsrcg"] = 0
    tmp = tempfile.mkdtemp(prefix=f"mvmc_bench_{rank}_")
    namelist, initial_def, dims = lattice.write_inputs(os.path.join(tmp, "in"), **cfg)
    return cfg, tmp, namelist, initial_def, dims


def reference_engine(args):
    cfg, tmp, namelist, initial_def, dims = engine_inputs(args, 0)
    procs = os.cpu_count() or 1
    per = 64 if args.config == "chain16" else 2
    S = cfg["samples"]
    sweeps = procs * per * (cfg["warmup"] + S) * cfg["interval"]  # the oracle's step 1 runs warm-up + S blocks
    pool = CpuPool(procs, initializer=_oracle_lib)
    jobs = [(namelist, initial_def, per, 12345 + k * per) for k in range(procs)]
    for _ in range(args.warmup):
        pool.time(_engine_job, jobs)
    times = [pool.time(_engine_job, jobs) for _ in range(args.steps)]
    pool.close()
    t = sum(times) / len(times)
    value = sweeps / t
    return {"metric": METRIC, "value": value, "unit": "sweeps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": args.config, "walkers": procs * per,
                       "sweeps_per_walker": (cfg["warmup"] + S) * cfg["interval"]},
            "cpu_baseline": {"value": value, "unit": "sweeps/s", "cores": procs, "kind": "port",
                             "sample": f"{procs * per} chains x one SR step (warm-up + {S} sample blocks) "
                                       f"of {args.config}, one process per core"},
            "e2e": {"value": value, "unit": "sweeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def time_engine(args, precision, W, namelist, initial_def, cfg, dims, rank, local, ws, dist, timed_hook=None,
                sr_precision=0):
    """Warm-up + K timed SR steps of one engine; returns the timing record."""
    import torch
    import mvmc_b200 as mb
    eng = mb.Engine(namelist, initial_def, walkers=W, precision=precision, seed=12345 + rank * W,
                    device=local, refresh_sweeps=args.refresh if precision == 32 else 0,
                    refresh_guard=args.guard if precision == 32 else 0.0, sr_precision=sr_precision,
                    sr_gram=1 if args.sr_gram else 0, measure_resident=1 if args.resident else 0)
    stream = torch.cuda.ExternalStream(eng.stream())
    energy = None
    if ws > 1:
        # walker-sharded SR: the sums and every CG product are added across ranks (NCCL)
        import sharded

        def reduce(a):
            t = torch.as_tensor(np.asarray(a, dtype=np.float64), device="cuda")
            dist.all_reduce(t)
            return t.cpu().numpy()

        def sr_step():
            # CG vectors stay on the GPU: z is added across ranks by an NCCL all-reduce of the
            # device tensor; the measurement sums go through `reduce` once per step
            info = sharded.sr_step_device(eng, reduce, dist.all_reduce, "cuda",
                                          torch.cuda.current_stream().cuda_stream)
            return 0, np.array([info[k] for k in ("npara", "nsmat", "opt_cut", "diag_cut", "sdiag_max",
                                                  "sdiag_min", "rmax", "imax", "info")], dtype=np.float64)
    else:
        sr_step = eng.sr_cg
    for _ in range(args.warmup):
        eng.sample()
        eng.measure()
        sr_step()
    torch.cuda.synchronize()
    if timed_hook:
        timed_hook("start")
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    marks = []
    h0, d0 = eng.transfer_bytes()
    t_wall0 = time.perf_counter()
    ev0.record(stream)
    cg_iters = []
    for _ in range(args.steps):
        a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        a.record(stream)
        eng.sample()
        b.record(stream)
        e, ho, oo = eng.measure()
        c.record(stream)
        rc, sri = sr_step()
        energy = float(e[1])
        cg_iters.append(int(sri[8]))
        marks.append((a, b, c))
    ev1.record(stream)
    torch.cuda.synchronize()
    t_wall = time.perf_counter() - t_wall0
    if timed_hook:
        timed_hook("stop")
    h1, d1 = eng.transfer_bytes()
    ms = ev0.elapsed_time(ev1)
    samp = [a.elapsed_time(b) for a, b, _ in marks]
    meas = [b.elapsed_time(c) for _, b, c in marks]
    if ws > 1:
        t = torch.tensor([ms, t_wall * 1e3], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, t_wall_ms = float(t[0]), float(t[1])
    else:
        t_wall_ms = t_wall * 1e3
    samples = eng.samples()
    c = samples["counter"].reshape(-1, 6).sum(axis=0)
    drift = eng.refresh_stats()
    eng.close()
    return {"ms": ms, "t_wall_ms": t_wall_ms, "sample_ms": sum(samp) / len(samp),
            "measure_ms": sum(meas) / len(meas), "h2d": h1 - h0, "d2h": d1 - d0, "energy": energy,
            "acceptance": (c[1] + c[3]) / max(1, c[0] + c[2]), "cg_iters": cg_iters, "drift": drift}


def accuracy_check(args, W, namelist, initial_def, local):
    """One fresh sample + measurement of the mixed and the plain FP64 path with the same
    seeds and parameters: chains that saw no Metropolis decision flip hold identical
    configurations (and energies to FP64 rounding, since measurement is FP64)."""
    import mvmc_b200 as mb
    out = {}
    for prec in (64, 32):
        eng = mb.Engine(namelist, initial_def, walkers=W, precision=prec, seed=12345, device=local,
                        refresh_sweeps=args.refresh if prec == 32 else 0,
                        refresh_guard=args.guard if prec == 32 else 0.0)
        eng.sample()
        e, _, _ = eng.measure()
        out[prec] = (e, eng.samples()["ele_idx"].reshape(W, -1), eng.local_energies(), eng.refresh_stats())
        eng.close()
    e64, idx64, el64, _ = out[64]
    e32, idx32, el32, drift = out[32]
    same = np.all(idx64 == idx32, axis=1)
    return {"walkers": W, "identical_chains": float(same.mean()),
            "energy_fp64": float(e64[1]), "energy_mixed": float(e32[1]),
            "dE": float(e32[1] - e64[1]),
            "stat_err": float(np.std(el64) / np.sqrt(len(el64))),
            "max_dEloc_identical": float(np.max(np.abs(el64[same] - el32[same]), initial=0.0)),
            "refresh_drift_max": drift["drift_max"], "refresh_drift_mean": drift["drift_mean"]}


def l2_ceiling_gbs():
    """Bandwidth of a working set that stays in L2, two ways (CUDA events, best of 20 after
    warm-up): a copy of 24 MB into 24 MB (read + write bytes, ten launches per event pair),
    and one reduction launch that reads the same 24 MB 64 times through a stride-0 view
    (1.6 GB of L2 reads in one launch, so launch gaps do not count). The larger is the
    ceiling for a kernel whose planes are L2-resident."""
    import torch
    n = 24 * (1 << 20) // 4
    a = torch.randn(n, device="cuda")
    b = torch.empty_like(a)
    rep = a.expand(64, n)
    out = torch.empty(64, device="cuda")

    def best_ms(fn, inner):
        for _ in range(5):
            fn()
        best = 1e30
        for _ in range(20):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(inner):
                fn()
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1) / inner)
        return best

    copy = 2 * 4 * n / (best_ms(lambda: b.copy_(a), 10) / 1e3) / 1e9
    read = 64 * 4 * n / (best_ms(lambda: torch.sum(rep, dim=1, out=out), 1) / 1e3) / 1e9
    return {"copy": copy, "read": read}


def sr16_record(args, local, timed=3):
    """The 2D 16×16 SR workload (t' = -0.2, U = 6, 112 + 112 electrons, n = 224, 4×4-sublattice
    f: 4226 parameters, 8192 walkers, SR-CG): SR-step time split into sampling, measurement
    and SR-CG for the plain FP64 path and the mixed path (FP32 inverse updates with FP64
    refresh; SR-CG through the tensor-core Gram of the centred, column-scaled samples with
    TF32 inputs), and the mixed path's errors on the first step from the same seeds and
    parameters: energy per site, variance, <O_k> and the SR parameter update; the update
    error of each reduced-precision SR operator alone on the FP64 path's samples; and the FP64
    path with the resident measurement (Pf and X⁻¹ of each saved sample as the sampler held
    them, not recomputed)."""
    import torch
    import lattice
    import mvmc_b200 as mb
    cfg = dict(lattice.CONFIGS["square16_sr"])
    tmp = tempfile.mkdtemp(prefix="mvmc_sr16_")
    nl, init, dims = lattice.write_inputs(os.path.join(tmp, "in"), **cfg)
    W = WALKERS["square16_sr"]

    def run(precision, sr_precision, steps, sr_gram=0, resident=0):
        eng = mb.Engine(nl, init, walkers=W, precision=precision, seed=12345,
                        refresh_sweeps=args.refresh if precision == 32 else 0,
                        refresh_guard=args.guard if precision == 32 else 0.0, sr_precision=sr_precision,
                        sr_gram=sr_gram, measure_resident=resident)
        stream = torch.cuda.ExternalStream(eng.stream())
        p0 = eng.parameters()
        eng.sample()
        e, ho, oo = eng.measure()
        idx = eng.samples()["ele_idx"].reshape(W, -1)
        _, info = eng.sr_cg()
        first = {"e": e, "oo": oo, "dp": eng.parameters() - p0, "idx": idx, "cg_info": int(info[8])}
        if steps == 0:
            eng.close()
            return first, None
        split = []
        for k in range(1 + steps):  # one untimed warm step, then the timed ones
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            ev[0].record(stream)
            eng.sample()
            ev[1].record(stream)
            eng.measure()
            ev[2].record(stream)
            eng.sr_cg()
            ev[3].record(stream)
            torch.cuda.synchronize()
            if k:
                split.append([ev[i].elapsed_time(ev[i + 1]) for i in range(3)])
        eng.close()
        s = np.mean(np.array(split), axis=0)
        return first, {"sample_ms": float(s[0]), "measure_ms": float(s[1]), "sr_cg_ms": float(s[2]),
                       "sr_step_ms": float(s.sum())}

    a_first, a_t = run(64, 64, timed)
    c_first, c_t = run(32, 32, timed, sr_gram=1)
    # FP64 path whose measurement reads the sampler's resident Pf and X⁻¹
    r_first, r_t = run(64, 64, timed, resident=1)
    op_err = {}
    for name, srp, gram in (("tf32_gram", 32, 1), ("bf16_gram", 16, 1), ("bf16_gemv", 16, 0)):
        f, _ = run(64, srp, 0, sr_gram=gram)
        op_err[name] = float(np.linalg.norm(f["dp"] - a_first["dp"]) / max(np.linalg.norm(a_first["dp"]), 1e-300))
    ns = dims["nsite"]
    size = 1 + dims["npara"]
    var = lambda f: float(f["e"][2] - f["e"][1] ** 2)
    rel = lambda x, y: float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))
    return {
        "workload": "square16_sr", "walkers": W, "n": dims["n"], "npara": dims["npara"],
        "sweeps_per_walker_step": (cfg["samples"] + 1) * cfg["interval"],
        "fp64": a_t, "mixed": c_t,
        "fp64_resident_measurement": dict(r_t, dE_per_site_first_step=float(
            abs(r_first["e"][1] - a_first["e"][1]) / ns), identical_chains_first_step=float(
            np.mean(np.all(r_first["idx"] == a_first["idx"], axis=1)))),
        "mixed_over_fp64": {"sr_step": a_t["sr_step_ms"] / c_t["sr_step_ms"],
                            "sweeps": a_t["sample_ms"] / c_t["sample_ms"],
                            "measure": a_t["measure_ms"] / c_t["measure_ms"],
                            "sr_cg": a_t["sr_cg_ms"] / c_t["sr_cg_ms"]},
        "mixed_precision": {"sampler": "f32 updates + f64 refresh", "refresh_sweeps": args.refresh,
                            "refresh_guard": args.guard,
                            "sr_operator": "Gram of the centred, column-scaled samples on the tensor cores "
                                           "(tcgen05, TF32 inputs, FP32 accumulation), FP64 CG"},
        "cg_status_first_step": {"fp64": a_first["cg_info"], "mixed": c_first["cg_info"]},
        "accuracy_first_step": {
            "identical_chains": float(np.mean(np.all(a_first["idx"] == c_first["idx"], axis=1))),
            "dE_per_site": float(abs(c_first["e"][1] - a_first["e"][1]) / ns),
            "variance_fp64": var(a_first), "dvariance": abs(var(c_first) - var(a_first)),
            "max_dO_mean": float(np.max(np.abs(c_first["oo"][:size] - a_first["oo"][:size]))),
            "update_rel_err_mixed": rel(c_first["dp"], a_first["dp"]),
            "update_rel_err_operator_only": op_err},
    }


def pfinv_records(local, steps=10, warmup=3):
    """Batched Pfaffian + inverse on device buffers: B = 8192 planes of n = 64 and the
    five-size mix {32, 48, 64, 96, 128} (8190 planes), FP64 and FP32 sweeps: planes/s and
    the fraction of the measured cuBLAS FP64 GEMM rate (2n³ flops per plane)."""
    import ctypes
    import torch
    import mvmc_b200 as mb
    L = mb.lib()
    peak = fp64_gemm_peak()
    out = {"fp64_gemm_tflops": peak}
    for name in ("pfinv64", "pfinv_mix"):
        sizes = PFINV[name]
        rng = np.random.default_rng(2024)
        uniq = sorted(set(sizes))
        by_n = {n: skew_planes(rng, n, sizes.count(n)) for n in uniq}
        cur = {n: 0 for n in uniq}
        chunks = []
        for n in sizes:
            chunks.append(by_n[n][cur[n]].ravel())
            cur[n] += 1
        x = torch.from_numpy(np.concatenate(chunks)).cuda()
        inv = torch.empty_like(x)
        B = len(sizes)
        pf = torch.zeros(B, dtype=torch.float64, device="cuda")
        st = torch.zeros(B, dtype=torch.int32, device="cuda")
        szs = np.asarray(sizes, dtype=np.int32)
        sz = torch.from_numpy(szs).cuda()
        off = torch.from_numpy(np.concatenate([[0], np.cumsum(szs.astype(np.int64) ** 2)[:-1]])).cuda()
        uniform = len(uniq) == 1
        P = lambda t: ctypes.c_void_p(t.data_ptr())
        stream = torch.cuda.current_stream()
        rec = {"planes": B, "sizes": uniq}
        for prec in (64, 32):
            def launch():
                rc = L.mvmc_b200_pfinv_batch_device(P(x), None if uniform else P(sz), None if uniform else P(off),
                                                    uniq[0] if uniform else 0, B, max(uniq), P(pf), P(inv), P(st),
                                                    prec, ctypes.c_void_p(stream.cuda_stream))
                if rc < 0:
                    raise RuntimeError(L.mvmc_b200_last_error().decode())
            for _ in range(warmup):
                launch()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(steps):
                launch()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / steps
            flops = float(sum(2 * n ** 3 for n in sizes))
            rec[f"fp{prec}"] = {"planes_per_s": B / (ms / 1e3), "ms": ms, "tflops": flops / (ms / 1e3) / 1e12,
                                "frac_of_fp64_gemm": flops / (ms / 1e3) / 1e12 / peak,
                                "singular": int((st != 0).sum())}
        out[name] = rec
        del x, inv
    return out


def engine_bench(args, ws, rank, local):
    import torch
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    cfg, tmp, namelist, initial_def, dims = engine_inputs(args, rank)
    W = args.walkers or WALKERS[args.config]
    S = cfg["samples"]
    sweeps_per_walker_step = (S + 1) * cfg["interval"]
    clocks_path = os.path.join(tmp, "clocks.csv")
    state = {}

    def hook(what):
        if rank != 0:
            return
        if what == "start":
            state["sampler"] = start_clock_sampler(clocks_path)
        else:
            stop_clock_sampler(state.pop("sampler", None))

    main_rec = time_engine(args, args.precision, W, namelist, initial_def, cfg, dims, rank, local, ws, dist, hook,
                           sr_precision=args.sr_precision)
    other = None
    other_prec = 32 if args.precision == 64 else 64
    if not args.no_compare:
        other = time_engine(args, other_prec, W, namelist, initial_def, cfg, dims, rank, local, ws, dist,
                            sr_precision=args.sr_precision)
    sweeps_total = ws * W * sweeps_per_walker_step * args.steps
    value = sweeps_total / (main_rec["ms"] / 1e3)
    n, nqp, ns = dims["n"], dims["nqp"], dims["nsite"]
    s_bytes = 8 if args.precision == 64 else 4
    p_acc = main_rec["acceptance"]
    # algorithmic bytes per walker-sweep of the resident sampler (InvM row + gathered Slater
    # row per proposal, rank-2 read+write per accepted move)
    per_sweep = ns * (nqp * n * s_bytes + nqp * n * 8) + ns * p_acc * nqp * (2 * n * n * s_bytes)
    launch_bytes = W * sweeps_per_walker_step * per_sweep
    achieved = launch_bytes / (main_rec["sample_ms"] / 1e3) / 1e9
    per_ws = SAMPLE_DRAM_PER_WALKER_SWEEP.get((args.config, args.precision))
    traffic = per_ws * W * sweeps_per_walker_step if per_ws and not args.interval else None
    peak, peak_kind = measured_peaks()
    if rank != 0:
        if ws > 1:
            dist.destroy_process_group()
        return
    acc = accuracy_check(args, min(W, 1024), namelist, initial_def, local) if other else None
    base_t = cpu_engine_time(namelist, initial_def, 1)
    base_sweeps = (cfg["warmup"] + S) * cfg["interval"]
    out = {
        "metric": METRIC, "value": value, "unit": "sweeps/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": main_rec["ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == 64 else "f32+f64refresh", "data": "synthetic",
        "config": {"workload": args.config, "walkers_per_gpu": W, "nsite": ns, "n": n, "nqp": nqp,
                   "npara": dims["npara"], "sweeps_per_walker_step": sweeps_per_walker_step,
                   "precision": args.precision, "parallelism": f"walker-sharded{ws}" if ws > 1 else "1",
                   "refresh_sweeps": args.refresh if args.precision == 32 else None,
                   "refresh_guard": args.guard if args.precision == 32 else None,
                   "sr_precision": args.sr_precision or 64, "sr": "direct" if args.direct else "cg",
                   "sr_gram": bool(args.sr_gram),
                   "measurement": "resident" if args.resident else "recomputed",
                   "l2": "inputs larger than L2 between steps (walker planes + O matrix)"},
        "sr_step_ms": main_rec["ms"] / args.steps, "sample_ms": main_rec["sample_ms"],
        "measure_ms": main_rec["measure_ms"], "energy": main_rec["energy"], "acceptance": p_acc,
        "cg_iterations": main_rec["cg_iters"],
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "kernel": "k_sample",
                     "peak_kind": peak_kind, "algorithmic_bytes_per_launch": launch_bytes},
        "cpu_baseline": {"value": base_sweeps / base_t, "unit": "sweeps/s", "cores": 1, "kind": "port",
                         "sample": f"1 chain x one SR step (warm-up + {S} blocks, {base_sweeps} sweeps) "
                                   f"of {args.config}"},
        "e2e": {"value": sweeps_total / (main_rec["t_wall_ms"] / 1e3), "unit": "sweeps/s",
                "h2d_bytes_per_step": main_rec["h2d"] // args.steps,
                "d2h_bytes_per_step": main_rec["d2h"] // args.steps},
        "gpu_launches": 8 * args.steps,
        "headline": ("plain FP64 path" if args.precision == 64 else "mixed path") +
                    "; the other path is timed beside it with its measured error against FP64",
        "residency": os.environ.get("MVMC_B200_RESIDENCY", "auto"),
        "clocks": summarize_clocks(clocks_path, local),
    }
    if args.precision == 32:
        out["refresh"] = {"sweeps": args.refresh, "guard": args.guard, **main_rec["drift"]}
    if other:
        rec = {"precision": other_prec, "value": sweeps_total / (other["ms"] / 1e3),
               "sr_step_ms": other["ms"] / args.steps, "sample_ms": other["sample_ms"],
               "energy": other["energy"], "acceptance": other["acceptance"]}
        if other_prec == 32:
            rec["refresh"] = {"sweeps": args.refresh, "guard": args.guard, **other["drift"]}
        out["mixed_path" if other_prec == 32 else "fp64_path"] = rec
        mixed_ms, fp64_ms = (other["ms"], main_rec["ms"]) if other_prec == 32 else (main_rec["ms"], other["ms"])
        out["mixed_over_fp64"] = {"sweeps": fp64_ms / mixed_ms, "sr_step": fp64_ms / mixed_ms}
        out["accuracy"] = acc
        if acc:
            out["accuracy"]["dE_per_site"] = acc["dE"] / ns
    if os.environ.get("MVMC_B200_TIMERS") == "1":
        out["timers"] = "phase cycles: run the engine directly for mvmc_b200_sampler_timers"
    if not args.no_extra and args.config == "square8" and ws == 1:
        # the sampler's planes are served from L2: its effective bandwidth against a measured
        # L2-resident copy as well as against HBM
        l2 = l2_ceiling_gbs()
        out["roofline"]["l2_peak"] = max(l2.values())
        out["roofline"]["l2_frac"] = achieved / max(l2.values())
        out["roofline"]["l2_peak_kind"] = (
            "measured in this run: max of a 24 MB -> 24 MB copy (%.0f GB/s) and one reduction "
            "reading a 24 MB buffer 64 times (%.0f GB/s)" % (l2["copy"], l2["read"]))
        out["square16_sr"] = sr16_record(args, local)
        out["pfinv"] = pfinv_records(local)
    print(json.dumps(out), flush=True)
    if ws > 1:
        dist.destroy_process_group()


# ----------------------------------------------------------------------------------------
# PhysCal workload.
# ----------------------------------------------------------------------------------------
def _physcal_job(args):
    namelist, zqp, walkers, seed = args
    _oracle_lib().physcal_green(namelist, zqp, seed, walkers)
    return 0


def physcal_flops(dims, nterm_one, samples):
    """Algorithmic FP64 flops of the PhysCal measurement of the given samples: per QP plane
    the Pfaffian + inverse (2n³) and 2n per allowed one-body hop (same spin, destination
    empty, source occupied), from the terms (i, s, j, t) of the one-body list."""
    n, nqp, ns = dims["n"], dims["nqp"], dims["nsite"]
    num = samples["ele_num"].reshape(-1, 2 * ns)
    occ_up, occ_dn = num[:, :ns].sum(axis=1), num[:, ns:].sum(axis=1)
    # the list holds every same-spin pair (i, j), so the allowed hops are empty × occupied
    hops = (ns - occ_up) * occ_up + (ns - occ_dn) * occ_dn
    assert nterm_one == 2 * ns * ns
    return float(np.sum(nqp * (2.0 * n ** 3 + 2.0 * n * hops)))


def reference_physcal(args):
    cfg, tmp, namelist, initial_def, dims = engine_inputs(args, 0)
    procs = os.cpu_count() or 1
    per = 2
    pool = CpuPool(procs, initializer=_oracle_lib)
    jobs = [(namelist, initial_def, per, 12345 + k * per) for k in range(procs)]
    for _ in range(args.warmup):
        pool.time(_physcal_job, jobs)
    times = [pool.time(_physcal_job, jobs) for _ in range(args.steps)]
    pool.close()
    t = sum(times) / len(times)
    value = procs * per * cfg["samples"] / t
    return {"metric": PHYSCAL_METRIC, "value": value, "unit": "samples/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": args.config, "walkers": procs * per},
            "cpu_baseline": {"value": value, "unit": "samples/s", "cores": procs, "kind": "port",
                             "sample": f"{procs * per} chains x one PhysCal block (warm-up + {cfg['samples']} "
                                       f"sample) of {args.config}, one process per core"},
            "e2e": {"value": value, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def physcal_bench(args, ws, rank, local):
    import torch
    import mvmc_b200 as mb
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    cfg, tmp, namelist, initial_def, dims = engine_inputs(args, rank)
    W = args.walkers or PHYSCAL[args.config]
    S = cfg["samples"]
    eng = mb.Engine(namelist, physcal_zqp=initial_def, walkers=W, precision=64, seed=12345 + rank * W, device=local)
    stream = torch.cuda.ExternalStream(eng.stream())

    def block():
        eng.sample()
        e, one, ex, two = eng.measure_green()
        if ws > 1:
            # chains on other GPUs: energy sums and the per-rank averaged Green functions
            sums = np.concatenate([[e[0]], e[1:] * e[0]])
            t = torch.as_tensor(np.concatenate([sums, one, ex, two]), device="cuda")
            dist.all_reduce(t)
            t = t.cpu().numpy()
            e = np.concatenate([[t[0]], t[1:5] / t[0]])
            one = t[5:5 + len(one)] / ws
        return e, one

    for _ in range(args.warmup):
        block()
    torch.cuda.synchronize()
    clocks_path = os.path.join(tmp, "clocks.csv")
    sampler = start_clock_sampler(clocks_path) if rank == 0 else None
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    h0, d0 = eng.transfer_bytes()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    marks = []
    t0 = time.perf_counter()
    ev0.record(stream)
    flops = 0.0
    for _ in range(args.steps):
        a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        a.record(stream)
        eng.sample()
        b.record(stream)
        e, one, ex, two = eng.measure_green()
        c.record(stream)
        marks.append((a, b, c))
        energy = float(e[1])
    ev1.record(stream)
    torch.cuda.synchronize()
    t_wall = time.perf_counter() - t0
    stop_clock_sampler(sampler)
    h1, d1 = eng.transfer_bytes()
    ms = ev0.elapsed_time(ev1)
    if ws > 1:
        t = torch.tensor([ms, t_wall * 1e3], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, t_wall = float(t[0]), float(t[1]) / 1e3
    samp = [a.elapsed_time(b) for a, b, _ in marks]
    meas = [b.elapsed_time(c) for _, b, c in marks]
    flops = physcal_flops(dims, eng.green_dims["one"], eng.samples())
    eng.close()
    if rank != 0:
        if ws > 1:
            dist.destroy_process_group()
        return
    total = ws * W * S * args.steps
    meas_ms = sum(meas) / len(meas)
    achieved = flops / (meas_ms / 1e3) / 1e12
    peak = fp64_gemm_peak()
    _oracle_lib()
    t_cpu = time.perf_counter()
    _physcal_job((namelist, initial_def, 2, 12345))
    t_cpu = time.perf_counter() - t_cpu
    out = {
        "metric": PHYSCAL_METRIC, "value": total / (ms / 1e3), "unit": "samples/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.config, "walkers_per_gpu": W, "samples_per_walker": S, "nsite": dims["nsite"],
                   "n": dims["n"], "nqp": dims["nqp"], "green_one": eng.green_dims["one"],
                   "green_two": eng.green_dims["two"], "parallelism": f"walker-sharded{ws}" if ws > 1 else "1",
                   "l2": "inputs larger than L2 between steps (walker planes and Green rows)"},
        "sample_ms": sum(samp) / len(samp), "measure_ms": meas_ms, "energy": energy,
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": None, "kernel": "k_measure (PhysCal form)",
                     "peak_kind": "measured cuBLAS FP64 GEMM on this GPU",
                     "algorithmic_flops_per_launch": flops},
        "cpu_baseline": {"value": 2 * S / t_cpu, "unit": "samples/s", "cores": 1, "kind": "port",
                         "sample": f"2 chains x one PhysCal block (warm-up + {S} sample) of {args.config}"},
        "e2e": {"value": total / t_wall, "unit": "samples/s", "h2d_bytes_per_step": (h1 - h0) // args.steps,
                "d2h_bytes_per_step": (d1 - d0) // args.steps},
        "gpu_launches": 6 * args.steps,
        "clocks": summarize_clocks(clocks_path, local),
    }
    print(json.dumps(out), flush=True)
    if ws > 1:
        dist.destroy_process_group()


# ----------------------------------------------------------------------------------------
# Pfaffian workloads.
# ----------------------------------------------------------------------------------------
def fp64_gemm_peak():
    """cuBLAS FP64 GEMM throughput (TFLOP/s) on this GPU, best of 5: the FP64 denominator."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2 * n ** 3 / (best / 1e3) / 1e12


def reference_pfinv(args):
    sizes = PFINV[args.config]
    procs = os.cpu_count() or 1
    per = 1024 if len(set(sizes)) == 1 else 128
    planes = procs * per * len(set(sizes))
    pool = CpuPool(procs, initializer=_pfinv_init, initargs=(sizes, per))
    for _ in range(args.warmup):
        pool.time(_pfinv_job, range(procs))
    times = [pool.time(_pfinv_job, range(procs)) for _ in range(args.steps)]
    pool.close()
    t = sum(times) / len(times)
    value = planes / t
    return {"metric": PFINV_METRIC, "value": value, "unit": "planes/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": args.config, "sizes": sorted(set(sizes))},
            "cpu_baseline": {"value": value, "unit": "planes/s", "cores": procs, "kind": "port",
                             "sample": f"{per} planes of each size per process, one process per core"},
            "e2e": {"value": value, "unit": "planes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def pfinv_bench(args, ws, rank, local):
    import ctypes
    import torch
    import mvmc_b200 as mb
    torch.cuda.set_device(local)
    sizes = PFINV[args.config]
    B = len(sizes)
    rng = np.random.default_rng(2024 + rank)
    uniq = sorted(set(sizes))
    planes_by_n = {n: skew_planes(rng, n, sizes.count(n)) for n in uniq}
    cursor = {n: 0 for n in uniq}
    chunks = []
    for n in sizes:
        chunks.append(planes_by_n[n][cursor[n]].ravel())
        cursor[n] += 1
    x_host = np.concatenate(chunks)
    sizes_host = np.asarray(sizes, dtype=np.int32)
    offsets_host = np.concatenate([[0], np.cumsum(sizes_host.astype(np.int64) ** 2)[:-1]]).astype(np.int64)
    n_max = max(sizes)
    uniform = len(uniq) == 1
    dev = torch.device("cuda", local)
    x = torch.from_numpy(x_host).to(dev)
    inv = torch.empty_like(x)
    pf = torch.zeros(B, dtype=torch.float64, device=dev)
    st = torch.zeros(B, dtype=torch.int32, device=dev)
    sz = torch.from_numpy(sizes_host).to(dev)
    off = torch.from_numpy(offsets_host).to(dev)
    stream = torch.cuda.current_stream(dev)
    P = lambda t: ctypes.c_void_p(t.data_ptr())
    L = mb.lib()

    def launch():
        rc = L.mvmc_b200_pfinv_batch_device(P(x), None if uniform else P(sz), None if uniform else P(off),
                                            n_max if uniform else 0, B, n_max, P(pf), P(inv), P(st),
                                            args.precision, ctypes.c_void_p(stream.cuda_stream))
        if rc < 0:
            raise RuntimeError(L.mvmc_b200_last_error().decode())

    for _ in range(args.warmup):
        launch()
    torch.cuda.synchronize()
    if int((st != 0).sum()) != 0:
        raise RuntimeError("singular planes in the Pfaffian workload")
    clocks_path = os.path.join(tempfile.mkdtemp(prefix="mvmc_pf_"), "clocks.csv")
    sampler = start_clock_sampler(clocks_path) if rank == 0 else None
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    ev[0].record(stream)
    for k in range(args.steps):
        launch()
        ev[k + 1].record(stream)
    torch.cuda.synchronize()
    stop_clock_sampler(sampler)
    per = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    ms = sum(per) / len(per)
    # end to end through the host-buffer entry points, inputs and results in pinned host
    # memory (the library pipelines its copies with the sweeps in ~32 MB chunks)
    def pinned(shape, dtype):
        return torch.empty(shape, dtype=dtype, pin_memory=True).numpy()
    x_pin = pinned(x_host.shape, torch.float64)
    x_pin[...] = x_host
    x_host = x_pin
    pf_h = pinned((B,), torch.float64)
    inv_h = pinned(x_host.shape, torch.float64)
    st_h = pinned((B,), torch.int32)
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    for _ in range(2):  # the first call sizes the library's device buffers and streams
        if uniform:
            L.mvmc_b200_pfinv_batch(vp(x_host), n_max, B, vp(pf_h), vp(inv_h), vp(st_h))
        else:
            L.mvmc_b200_pfinv_batch_mixed(vp(x_host), vp(sizes_host), B, args.precision, vp(pf_h), vp(inv_h),
                                          vp(st_h))
    t0 = time.perf_counter()
    for _ in range(args.steps):
        if uniform:
            rc = L.mvmc_b200_pfinv_batch(vp(x_host), n_max, B, vp(pf_h), vp(inv_h), vp(st_h))
        else:
            rc = L.mvmc_b200_pfinv_batch_mixed(vp(x_host), vp(sizes_host), B, args.precision, vp(pf_h),
                                               vp(inv_h), vp(st_h))
        if rc < 0:
            raise RuntimeError(L.mvmc_b200_last_error().decode())
    e2e_s = (time.perf_counter() - t0) / args.steps
    flops = float(sum(2 * n ** 3 for n in sizes))
    bytes_ = float(sum(16 * n * n for n in sizes))
    peak_tf = fp64_gemm_peak()
    achieved = flops / (ms / 1e3) / 1e12
    hbm, hbm_kind = measured_peaks()
    base_planes = 256 if uniform else 32
    base_t = cpu_pfinv_time(sizes, base_planes)
    base_value = base_planes * len(uniq) / base_t
    out = {
        "metric": PFINV_METRIC, "value": ws * B / (ms / 1e3), "unit": "planes/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == 64 else "f32sweep",
        "data": "synthetic",
        "config": {"workload": args.config, "planes": B, "sizes": uniq, "precision": args.precision,
                   "l2": "inputs larger than L2 (x + inverse > 126 MB)"},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak_tf, "unit": "TFLOP/s",
                     "frac": achieved / peak_tf, "traffic": None, "kernel": "k_pfinv_pp/k_pfinv_batch",
                     "peak_kind": "cuBLAS FP64 GEMM measured in this run",
                     "hbm_gbs": bytes_ / (ms / 1e3) / 1e9, "hbm_peak": hbm, "hbm_peak_kind": hbm_kind},
        "cpu_baseline": {"value": base_value, "unit": "planes/s", "cores": 1, "kind": "port",
                         "sample": f"{base_planes} planes of each size {uniq}"},
        "e2e": {"value": ws * B / e2e_s, "unit": "planes/s", "h2d_bytes_per_step": int(x_host.nbytes + 4 * B),
                "d2h_bytes_per_step": int(inv_h.nbytes + 8 * B + 4 * B)},
        "gpu_launches": args.steps,
        "clocks": summarize_clocks(clocks_path, local),
    }
    if rank == 0:
        print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="square8", choices=sorted(WALKERS) + sorted(PFINV) + sorted(PHYSCAL))
    ap.add_argument("--precision", type=int, default=64, choices=(32, 64),
                    help="64: plain FP64 path (default); 32: mixed path (FP32 inverses, FP64 refresh)")
    ap.add_argument("--walkers", type=int, default=0)
    ap.add_argument("--interval", type=int, default=0, help="override NVMCInterval (sweeps per sample block)")
    ap.add_argument("--refresh", type=int, default=32,
                    help="mixed path: FP64 refresh every this many sweeps (0: the C accept-window rule)")
    ap.add_argument("--guard", type=float, default=0.03,
                    help="mixed path: FP64 refresh after an accepted move with a plane ratio outside [g, 1/g]")
    ap.add_argument("--no-compare", action="store_true", help="time one path only (no other precision beside it)")
    ap.add_argument("--sr-precision", type=int, default=0, choices=(0, 64, 32, 16),
                    help="SR operator storage of the timed engine (0: FP64)")
    ap.add_argument("--direct", action="store_true", help="direct SR (NSRCG 0): Gram + Cholesky instead of SR-CG")
    ap.add_argument("--sr-gram", action="store_true",
                    help="with --sr-precision 32/16: SR-CG through the tensor-core Gram of the samples")
    ap.add_argument("--resident", action="store_true",
                    help="FP64 path: measure from the sampler's resident Pf and inverse (not recomputed)")
    ap.add_argument("--no-extra", action="store_true",
                    help="square8: skip the 16x16 SR-step record, the Pfaffian records and the L2 ceiling")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    args = ap.parse_args()
    ws, rank, local = dist_env()
    pf = args.config in PFINV
    pc = args.config in PHYSCAL
    if args.impl == "reference":
        if rank != 0:
            return
        ref = reference_pfinv(args) if pf else (reference_physcal(args) if pc else reference_engine(args))
        print(json.dumps(ref), flush=True)
        return
    if pf:
        pfinv_bench(args, ws, rank, local)
    elif pc:
        physcal_bench(args, ws, rank, local)
    else:
        engine_bench(args, ws, rank, local)


if __name__ == "__main__":
    main()
