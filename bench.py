"""Benchmark: one VMC optimisation step (resident sampling → measurement → SR-CG) per
timed step, on the synthetic Hubbard workloads of mvmc-rs_b200/lattice.py.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config square8]
                    [--precision 64|32] [--impl ours|reference]

Prints one JSON line (rank 0). `value` is Metropolis sweeps/s of the whole job with the
model resident on the device; `e2e` times the same steps through the public C ABI calls
including their host↔device copies. For N > 1 (torchrun) every rank runs its own walker
ensemble (seeds offset by rank × walkers): replicas, no data-path collective.
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "mvmc-rs_b200"))

WALKERS = {"chain16": 256, "square8": 4096, "square16": 2048, "square16_sr": 8192}
METRIC = "Metropolis sweeps/s & SR-step time: mixed vs FP64 path on 1 B200 at |dE|/N<=1e-6"


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


def summarize_clocks(path, device):
    import statistics
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
            "reasons": sorted(reasons)}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def cpu_baseline(namelist, initial_def, walkers_per_proc, procs, seconds_hint=10.0):
    """The oracle (C++ restatement of the reference CPU path) on host cores."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    ol.lib()
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    if procs == 1:
        _oracle_chunk((namelist, initial_def, walkers_per_proc, 12345))
    else:
        with ctx.Pool(procs) as pool:
            pool.map(_oracle_chunk, [(namelist, initial_def, walkers_per_proc, 12345 + k * walkers_per_proc)
                                     for k in range(procs)])
    return time.perf_counter() - t0


def _oracle_chunk(args):
    namelist, initial_def, walkers, seed = args
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    ol.opt_step1_walkers(namelist, walkers, seed=seed, initial_def=initial_def)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="square8")
    ap.add_argument("--precision", type=int, default=64)
    ap.add_argument("--walkers", type=int, default=0)
    ap.add_argument("--refresh", type=int, default=32,
                    help="mixed path: FP64 refresh every this many sweeps (0: the C accept-window rule)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    args = ap.parse_args()
    ws, rank, local = dist_env()

    import lattice
    cfg = dict(lattice.CONFIGS[args.config])
    W = args.walkers or WALKERS[args.config]
    tmp = tempfile.mkdtemp(prefix=f"mvmc_bench_{rank}_")
    namelist, initial_def, dims = lattice.write_inputs(os.path.join(tmp, "in"), **cfg)
    S = cfg["samples"]
    sweeps_per_walker_step = (S + 1) * cfg["interval"]  # burn-in chain: NVMCSample + 1 blocks

    if args.impl == "reference":
        if rank != 0:
            return
        procs = os.cpu_count() or 1
        per = max(1, 2 if args.config != "chain16" else 64)
        # the oracle's first step includes warm-up blocks: (warmup + S) blocks per walker
        sweeps = procs * per * (cfg["warmup"] + S) * cfg["interval"]
        times = []
        for _ in range(args.warmup):
            cpu_baseline(namelist, initial_def, per, procs)
        for _ in range(args.steps):
            times.append(cpu_baseline(namelist, initial_def, per, procs))
        t = sum(times) / len(times)
        value = sweeps / t
        line = {"metric": METRIC, "value": value, "unit": "sweeps/s", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "impl": "reference",
                "config": {"workload": args.config, "walkers": procs * per, "sweeps_per_walker": (cfg["warmup"] + S) * cfg["interval"]},
                "cpu_baseline": {"value": value, "unit": "sweeps/s", "cores": procs, "kind": "port",
                                 "sample": f"{procs * per} chains x one SR step (warm-up + {S} sample blocks) of {args.config}"},
                "e2e": {"value": value, "unit": "sweeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    import mvmc_b200 as mb
    if ws > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    eng = mb.Engine(namelist, initial_def, walkers=W, precision=args.precision, seed=12345 + rank * W,
                    device=local, refresh_sweeps=args.refresh if args.precision == 32 else 0)
    stream = torch.cuda.ExternalStream(eng.stream())
    info = {}

    def sr_step():
        eng.sample()
        e, ho, oo = eng.measure()
        rc, sri = eng.sr_cg()
        info["energy"] = float(e[1])
        info["cg_info"] = int(sri[8])
        return e

    for _ in range(args.warmup):
        sr_step()
    torch.cuda.synchronize()
    clocks_path = os.path.join(tmp, "clocks.csv")
    sampler = start_clock_sampler(clocks_path) if rank == 0 else None
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    samp_ms = []
    h0, d0 = eng.transfer_bytes()
    t_wall0 = time.perf_counter()
    ev0.record(stream)
    for _ in range(args.steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        eng.sample()
        b.record(stream)
        e, ho, oo = eng.measure()
        rc, sri = eng.sr_cg()
        info["energy"] = float(e[1])
        samp_ms.append((a, b))
    ev1.record(stream)
    torch.cuda.synchronize()
    t_wall = time.perf_counter() - t_wall0
    h1, d1 = eng.transfer_bytes()
    if sampler is not None:
        sampler.terminate()
        sampler.wait()
    ms = ev0.elapsed_time(ev1)
    samp = [a.elapsed_time(b) for a, b in samp_ms]
    if ws > 1:
        t = torch.tensor([ms, t_wall * 1e3], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, t_wall_ms = float(t[0]), float(t[1])
    else:
        t_wall_ms = t_wall * 1e3
    sweeps_total = ws * W * sweeps_per_walker_step * args.steps
    value = sweeps_total / (ms / 1e3)
    samples = eng.samples()
    c = samples["counter"].reshape(-1, 6).sum(axis=0)
    proposals = int(c[0] + c[2])
    p_acc = (c[1] + c[3]) / max(1, proposals)
    n, nqp, ns = dims["n"], dims["nqp"], dims["nsite"]
    s_bytes = 8 if args.precision == 64 else 4
    # algorithmic bytes per walker-sweep of the resident sampler (row reads per proposal,
    # rank-2 read+write per accepted move)
    per_sweep = ns * (nqp * n * s_bytes + nqp * n * 8) + ns * p_acc * nqp * (2 * n * n * s_bytes)
    launch_bytes = W * sweeps_per_walker_step * per_sweep
    samp_avg_ms = sum(samp) / len(samp)
    achieved = launch_bytes / (samp_avg_ms / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    out = None
    if rank == 0:
        base_t = cpu_baseline(namelist, initial_def, 1, 1)
        base_sweeps = (cfg["warmup"] + S) * cfg["interval"]
        clocks = summarize_clocks(clocks_path, local)
        out = {
            "metric": METRIC, "value": value, "unit": "sweeps/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.precision == 64 else "f32+f64refresh",
            "data": "synthetic",
            "config": {"workload": args.config, "walkers_per_gpu": W, "nsite": ns, "n": n, "nqp": nqp,
                       "npara": dims["npara"], "sweeps_per_walker_step": sweeps_per_walker_step,
                       "precision": args.precision, "parallelism": f"replicas{ws}",
                       "refresh_sweeps": args.refresh if args.precision == 32 else None,
                       "l2": "inputs larger than L2 between steps (walker planes + O matrix)"},
            "sr_step_ms": ms / args.steps, "sample_ms": samp_avg_ms, "energy": info.get("energy"),
            "acceptance": p_acc,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "kernel": "k_sample",
                         "peak_kind": peak_kind},
            "cpu_baseline": {"value": base_sweeps / base_t, "unit": "sweeps/s", "cores": 1, "kind": "port",
                             "sample": f"1 chain x one SR step (warm-up + {S} blocks, {base_sweeps} sweeps) of {args.config}"},
            "e2e": {"value": sweeps_total / (t_wall_ms / 1e3), "unit": "sweeps/s",
                    "h2d_bytes_per_step": (h1 - h0) // args.steps, "d2h_bytes_per_step": (d1 - d0) // args.steps},
            "gpu_launches": 8 * args.steps,
            "residency": os.environ.get("MVMC_B200_RESIDENCY", "auto"),
            "phase_cycles_per_walker": ({k: v / W for k, v in eng.sampler_timers().items()}
                                        if os.environ.get("MVMC_B200_TIMERS") == "1" else None),
            "clocks": clocks,
        }
        print(json.dumps(out), flush=True)
    eng.close()
    if ws > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
