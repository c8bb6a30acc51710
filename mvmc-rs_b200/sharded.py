"""Walker-sharded SR step across ranks.

Each rank samples and measures its own walkers (seeds RndSeed + global walker index,
multichain.rs:88). The SR step has one real exchange: the measurement sums (Wc, E, E²,
Sz, Sz², HO, ⟨O⟩, ⟨O²⟩) are added across ranks before the weight average, and every CG
product z = Σ_ranks Σ_s O_s (O_s·v) is added across ranks — the placement of the
reference's Reducer (crates/mvmc-core/src/reducer.rs:20-168) in
stochastic_opt_cg_with_reducer (sr_cg.rs:201-490): the sampled operator is reduced before
the weight, mean and shift terms (apply_with_product, sr_cg.rs:952-1009). Every rank then
runs the same C recurrence (sr_cg.rs:700-880) on identical numbers and applies the same
update, so the parameters stay identical without a broadcast.

`local` is any object with measure_sums(), sr_config(), sr_gather(map),
sr_local_product(v) and sr_apply(map, x) — the device Engine of mvmc_b200.py, or a CPU
stand-in in the tests. `reduce(array) -> array` adds an array across ranks (identity on
one rank; torch.distributed all_reduce over NCCL in bench.py, gloo in the tests).

sr_step_device keeps the CG vectors in torch tensors on the local product's device: the
product is `local.sr_local_product_device(v, z, stream)` on device buffers and
`reduce_(z)` adds z across ranks in place (an NCCL all-reduce of the device tensor), so no
vector leaves the GPU during the solve; only the recurrence's scalars (the dots that decide
its branches) are read on the host, as the reference's per-iteration Reducer does.
"""
import numpy as np


def _dot(a, b):
    """Single-threaded pairwise sum: the same bits on every rank whatever the BLAS
    threading, so every rank takes the same CG branch."""
    return float(np.sum(a * b))


def operands(sums):
    """Weight average of the reduced sums (weight_average_sr_opt_real, average.rs:50)."""
    size = (len(sums) - 5) // 3
    tot = np.array(sums, dtype=np.float64)
    wc = tot[0]
    if abs(wc) >= 1e-15:
        tot[1:] /= wc
    return dict(wc=wc, energy=tot[:5], ho=tot[5:5 + size], mean=tot[5 + size:5 + 2 * size],
                diag=tot[5 + 2 * size:5 + 3 * size])


def active_set(ops, npara, flags, red_cut):
    """Redundancy cut of the CG path (sr_cg.rs:201-300): variances ⟨O²⟩ − ⟨O⟩² of the
    optimised parameters against red_cut × their maximum."""
    var = ops["diag"][1:npara + 1] - ops["mean"][1:npara + 1] ** 2
    if np.isnan(var).any():
        vmax = vmin = float("nan")
    else:
        vmax, vmin = float(np.max(var)), float(np.min(var))
    threshold = vmax * red_cut
    mapping, opt_cut, diag_cut = [], 0, 0
    for pi in range(npara):
        if not (2 * pi < len(flags) and flags[2 * pi] == 1):
            opt_cut += 1
        elif var[pi] < threshold:
            diag_cut += 1
        else:
            mapping.append(pi)
    return np.array(mapping, dtype=np.int32), var, opt_cut, diag_cut, vmax, vmin


def cg_solve(apply, g, diag, shift, tol, max_iter, diag_scale):
    """The C recurrence of SampledSrOperator::solve_with_product (sr_cg.rs:700-880):
    threshold tol²·n², δ = β·δ (plain) or δ = δ_new (DiagScale), r = g − S·x every 20th
    iteration, breakdown |d·q| < 1e-20; returns (x, status) with status = iterations or
    −(iter+1)."""
    n = len(g)
    threshold = tol * tol * float(n) * float(n)
    dq_pre = (1.0 + shift) * diag
    dq_pre = np.where(np.isfinite(dq_pre) & (np.abs(dq_pre) >= 1e-12), dq_pre,
                      np.where(dq_pre < 0.0, -1e-12, 1e-12))

    def precond(r):
        return r / dq_pre

    x = np.zeros(n)
    r = g.copy()
    if diag_scale:
        r = g - apply(x)
        d = precond(r)
        delta = _dot(r, d)
    else:
        d = g.copy()
        delta = _dot(r, r)
    status, it, done = 0, 0, False
    if not np.isfinite(delta):
        return x, -1
    while it < max_iter:
        failed = -(it + 1)
        if not np.isfinite(delta):
            status, done = failed, True
            break
        if abs(delta) < threshold:
            break
        q = apply(d)
        dq = _dot(d, q)
        if not np.isfinite(dq) or abs(dq) < 1e-20:
            status, done = failed, True
            break
        alpha = delta / dq
        if not np.isfinite(alpha):
            status, done = failed, True
            break
        x = x + alpha * d
        if (it + 1) % 20 == 0:
            r = g - apply(x)
        else:
            r = r - alpha * q
        if diag_scale:
            q = precond(r)
            delta_new = _dot(r, q)
        else:
            delta_new = _dot(r, r)
        if not np.isfinite(delta_new) or abs(delta) < 1e-20:
            status, done = failed, True
            break
        beta = delta_new / delta
        if not np.isfinite(beta):
            status, done = failed, True
            break
        if diag_scale:
            delta = delta_new
            d = q + beta * d
        else:
            delta *= beta
            d = r + beta * d
        it += 1
    if not done:
        status = -(max_iter + 1) if (it == max_iter and abs(delta) >= threshold) else it
    return x, status


def sr_step(local, reduce):
    """One SR-CG step over all ranks; returns the SRinfo values
    {npara, nsmat, opt_cut, diag_cut, sdiag_max, sdiag_min, rmax, imax, info}."""
    cfg, flags = local.sr_config()
    if int(cfg["nsrcg"]) == 0:
        raise NotImplementedError("the sharded SR step runs SR-CG (NSRCG 1)")
    npara = int(cfg["npara"])
    ops = operands(reduce(local.measure_sums()))
    mapping, var, opt_cut, diag_cut, vmax, vmin = active_set(ops, npara, flags, cfg["red_cut"])
    info = dict(npara=npara, nsmat=len(mapping), opt_cut=opt_cut, diag_cut=diag_cut, sdiag_max=vmax,
                sdiag_min=vmin, rmax=0.0, imax=0, info=0)
    if len(mapping) == 0:
        return info
    idx = mapping + 1
    mean, diag = ops["mean"][idx], var[mapping]
    g = -2.0 * cfg["step_dt"] * (ops["ho"][idx] - ops["ho"][0] * ops["mean"][idx])
    inv_w = 1.0 / ops["wc"]
    shift = cfg["sta_del"]
    local.sr_gather(mapping)

    def apply(v):
        z = reduce(local.sr_local_product(v))
        return inv_w * z - _dot(mean, v) * mean + shift * diag * v

    max_iter = int(cfg["cg_max_iter"]) if cfg["cg_max_iter"] > 0 else len(mapping)
    diag_scale = bool(cfg["diag_scale"])
    x, status = cg_solve(apply, g, diag, shift, cfg["cg_tol"], max_iter, diag_scale)
    code = status
    if status < 0:
        fallback_iter = max(-status - 1, 0)
        if cfg["cg_fallback"]:
            x, st2 = cg_solve(apply, g, diag, shift, cfg["cg_tol"], max_iter, not diag_scale)
            code = -(fallback_iter + 1)
            if st2 < 0 and cfg["cg_abort"]:
                raise RuntimeError("fallback SR-CG failed")
        else:
            if cfg["cg_abort"]:
                raise RuntimeError("SR-CG failed and fallback is disabled")
            code = -(fallback_iter + 1)
    imax = int(np.argmax(np.abs(x)))  # first maximum, as the C loop
    info.update(rmax=float(x[imax]), imax=int(mapping[imax]), info=int(code))
    if not np.all(np.isfinite(x)):
        if cfg["cg_abort"]:
            raise RuntimeError("SR-CG produced non-finite updates")
        return info
    local.sr_apply(mapping, x)
    return info


def cg_solve_t(apply, g, diag, shift, tol, max_iter, diag_scale):
    """cg_solve on torch tensors (any device): the same recurrence, statuses and elementwise
    operation order; dots are tensor sums read on the host for the branch decisions."""
    import torch
    n = g.numel()
    threshold = tol * tol * float(n) * float(n)
    dq_pre = (1.0 + shift) * diag
    ok = torch.isfinite(dq_pre) & (dq_pre.abs() >= 1e-12)
    dq_pre = torch.where(ok, dq_pre, torch.where(dq_pre < 0.0, torch.full_like(dq_pre, -1e-12),
                                                  torch.full_like(dq_pre, 1e-12)))

    def dot(a, b):
        return float((a * b).sum())

    x = torch.zeros_like(g)
    r = g.clone()
    if diag_scale:
        r = g - apply(x)
        d = r / dq_pre
        delta = dot(r, d)
    else:
        d = g.clone()
        delta = dot(r, r)
    status, it, done = 0, 0, False
    if not np.isfinite(delta):
        return x, -1
    while it < max_iter:
        failed = -(it + 1)
        if not np.isfinite(delta):
            status, done = failed, True
            break
        if abs(delta) < threshold:
            break
        q = apply(d)
        dq = dot(d, q)
        if not np.isfinite(dq) or abs(dq) < 1e-20:
            status, done = failed, True
            break
        alpha = delta / dq
        if not np.isfinite(alpha):
            status, done = failed, True
            break
        x = x + alpha * d
        if (it + 1) % 20 == 0:
            r = g - apply(x)
        else:
            r = r - alpha * q
        if diag_scale:
            q = r / dq_pre
            delta_new = dot(r, q)
        else:
            delta_new = dot(r, r)
        if not np.isfinite(delta_new) or abs(delta) < 1e-20:
            status, done = failed, True
            break
        beta = delta_new / delta
        if not np.isfinite(beta):
            status, done = failed, True
            break
        if diag_scale:
            delta = delta_new
            d = q + beta * d
        else:
            delta *= beta
            d = r + beta * d
        it += 1
    if not done:
        status = -(max_iter + 1) if (it == max_iter and abs(delta) >= threshold) else it
    return x, status


def sr_step_device(local, reduce, reduce_, device, stream=0):
    """sr_step with the CG vectors on `device` (torch tensors): the local product on device
    buffers, z added across ranks in place by `reduce_(tensor)`. `reduce` adds the
    measurement sums (host arrays, once per SR step)."""
    import torch
    cfg, flags = local.sr_config()
    if int(cfg["nsrcg"]) == 0:
        raise NotImplementedError("the sharded SR step runs SR-CG (NSRCG 1)")
    npara = int(cfg["npara"])
    ops = operands(reduce(local.measure_sums()))
    mapping, var, opt_cut, diag_cut, vmax, vmin = active_set(ops, npara, flags, cfg["red_cut"])
    info = dict(npara=npara, nsmat=len(mapping), opt_cut=opt_cut, diag_cut=diag_cut, sdiag_max=vmax,
                sdiag_min=vmin, rmax=0.0, imax=0, info=0)
    if len(mapping) == 0:
        return info
    idx = mapping + 1
    as_t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=device)
    mean, diag = as_t(ops["mean"][idx]), as_t(var[mapping])
    g = as_t(-2.0 * cfg["step_dt"] * (ops["ho"][idx] - ops["ho"][0] * ops["mean"][idx]))
    inv_w = 1.0 / ops["wc"]
    shift = cfg["sta_del"]
    local.sr_gather(mapping)

    def apply(v):
        v = v.contiguous()
        z = torch.empty_like(v)
        local.sr_local_product_device(v, z, stream)
        reduce_(z)
        return inv_w * z - (mean * v).sum() * mean + shift * diag * v

    max_iter = int(cfg["cg_max_iter"]) if cfg["cg_max_iter"] > 0 else len(mapping)
    diag_scale = bool(cfg["diag_scale"])
    x, status = cg_solve_t(apply, g, diag, shift, cfg["cg_tol"], max_iter, diag_scale)
    code = status
    if status < 0:
        fallback_iter = max(-status - 1, 0)
        if cfg["cg_fallback"]:
            x, st2 = cg_solve_t(apply, g, diag, shift, cfg["cg_tol"], max_iter, not diag_scale)
            code = -(fallback_iter + 1)
            if st2 < 0 and cfg["cg_abort"]:
                raise RuntimeError("fallback SR-CG failed")
        else:
            if cfg["cg_abort"]:
                raise RuntimeError("SR-CG failed and fallback is disabled")
            code = -(fallback_iter + 1)
    x = x.cpu().numpy()
    imax = int(np.argmax(np.abs(x)))
    info.update(rmax=float(x[imax]), imax=int(mapping[imax]), info=int(code))
    if not np.all(np.isfinite(x)):
        if cfg["cg_abort"]:
            raise RuntimeError("SR-CG produced non-finite updates")
        return info
    local.sr_apply(mapping, x)
    return info
