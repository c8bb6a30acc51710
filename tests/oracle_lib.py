"""ctypes loader for the oracle (test infrastructure: the CPU checker of the CUDA path)."""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(ROOT, "oracle", "_build", "liboracle.so")
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
        _LIB = ctypes.CDLL(path)
    return _LIB


def ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def err_buf():
    return ctypes.create_string_buffer(1024)


def model_dims(namelist):
    dims = (ctypes.c_int * 8)()
    err = err_buf()
    if lib().oracle_model_dims(namelist.encode(), dims, err, 1024) != 0:
        raise RuntimeError(err.value.decode())
    keys = ["nsite", "ne", "nqp", "nproj", "npara", "nvmc_sample", "data_qty_smp", "n_orb"]
    return dict(zip(keys, list(dims)))


def sfmt_words(seed, count):
    out = (ctypes.c_uint32 * count)()
    lib().oracle_sfmt_words(ctypes.c_uint32(seed), count, out)
    return list(out)


def pfinv_batch(x_colmajor, n, planes):
    x = np.ascontiguousarray(x_colmajor, dtype=np.float64)
    pf = np.zeros(planes)
    inv = np.zeros(planes * n * n)
    st = np.zeros(planes, dtype=np.int32)
    lib().oracle_pfinv_batch(ptr(x), n, planes, ptr(pf), ptr(inv), ptr(st))
    return pf, inv, st


def physcal_samples(namelist, zqp, seed):
    d = model_dims(namelist)
    n, ns2, npj = 2 * d["ne"], 2 * d["nsite"], d["nproj"]
    b, S = d["data_qty_smp"], d["nvmc_sample"]
    out = dict(
        ele_idx=np.zeros(b * S * n, np.int64), ele_cfg=np.zeros(b * S * ns2, np.int64),
        ele_num=np.zeros(b * S * ns2, np.int64), proj_cnt=np.zeros(b * S * npj, np.int64),
        counter=np.zeros(b * 6, np.int64), draws=np.zeros(b, np.int64),
        next624=np.zeros(b * 624, np.uint32), energies=np.zeros(2 * b))
    err = err_buf()
    rc = lib().oracle_physcal_samples(
        namelist.encode(), zqp.encode(), ctypes.c_longlong(seed), *(ptr(out[k]) for k in (
            "ele_idx", "ele_cfg", "ele_num", "proj_cnt", "counter", "draws", "next624", "energies")),
        err, 1024)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    return d, out


def green_dims(namelist):
    dims = (ctypes.c_int * 5)()
    err = err_buf()
    if lib().oracle_green_dims(namelist.encode(), dims, err, 1024) != 0:
        raise RuntimeError(err.value.decode())
    return dict(zip(["one", "ex", "two", "blocks", "idx_start"], list(dims)))


def physcal_green(namelist, zqp, seed, walkers=1, out_dir=""):
    """PhysCal blocks on `walkers` chains: energies [blocks][4] (Etot, Etot2, Sztot,
    Sztot2) and the one-body, TwoBodyGEx and TwoBodyG Green functions per block."""
    g = green_dims(namelist)
    b = g["blocks"]
    out = dict(energy=np.zeros((b, 4)), one=np.zeros((b, g["one"])), ex=np.zeros((b, g["ex"])),
               two=np.zeros((b, g["two"])))
    err = err_buf()
    rc = lib().oracle_physcal_green(namelist.encode(), zqp.encode(), ctypes.c_longlong(seed), walkers,
                                    *(ptr(out[k]) for k in ("energy", "one", "ex", "two")),
                                    out_dir.encode(), err, 1024)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    return g, out


def read_physcal_expected(directory, index):
    """Numbers of the native C PhysCal files of one data block."""
    def nums(name, skip):
        path = os.path.join(directory, f"zvo_{name}_{index:03d}.dat")
        rows = [line.split() for line in open(path) if line.strip()]
        return np.array([[float(v) for v in r[skip:]] for r in rows])
    out = nums("out", 0)[0]
    return dict(energy=np.array([out[0], out[2], out[4], out[5]]), one=nums("cisajs", 4)[:, 0],
                two=nums("cisajscktalt", 8)[:, 0], ex=nums("cisajscktaltex", 0)[0, 0::2])


def step1_operands(namelist, cg=1, store=0, seed=1):
    d = model_dims(namelist)
    size = 1 + d["npara"]
    e, ho, oo, o = np.zeros(1), np.zeros(size), np.zeros(2 * size), np.zeros(size)
    err = err_buf()
    rc = lib().oracle_step1_operands(namelist.encode(), cg, store, ctypes.c_longlong(seed), ptr(e),
                                     ptr(ho), ptr(oo), ptr(o), size, err, 1024)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    return dict(energy=e, ho=ho, oo=oo, o=o)


class fixed_exp_mode:
    """Context in which the oracle's local-energy projection ratios use fixed_exp (the exp
    the device's C-order mode computes) instead of the platform libm's exp."""

    def __enter__(self):
        lib().oracle_set_fixed_exp(1)
        return self

    def __exit__(self, *exc):
        lib().oracle_set_fixed_exp(0)
        return False


def fixed_exp(x):
    f = lib().oracle_fixed_exp
    f.restype, f.argtypes = ctypes.c_double, [ctypes.c_double]
    return f(float(x))


def run_opt(namelist, out_dir, walkers=1, nsteps=0, seed=-1, initial_def=""):
    err = err_buf()
    rc = lib().oracle_run_opt(namelist.encode(), initial_def.encode(), out_dir.encode(), walkers,
                              nsteps, ctypes.c_longlong(seed), err, 1024)
    if rc != 0:
        raise RuntimeError(err.value.decode())


def cg_fixed(mean, diag, samples, g, inv_w, shift, tol, max_iter, diag_scale=False, want_apply=False):
    n = len(mean)
    ns = samples.size // n
    x = np.zeros(n)
    z = np.zeros(n) if want_apply else None
    st = lib().oracle_cg_fixed(n, ns, ptr(np.ascontiguousarray(mean)), ptr(np.ascontiguousarray(diag)),
                               ptr(np.ascontiguousarray(samples)), ptr(np.ascontiguousarray(g)),
                               ctypes.c_double(inv_w), ctypes.c_double(shift), ctypes.c_double(tol),
                               max_iter, int(diag_scale), ptr(x), ptr(z) if z is not None else None)
    return st, x, z


def hexline(line):
    import struct
    return np.array([struct.unpack(">d", bytes.fromhex(v))[0] for v in line.split()])


def opt_step1_walkers(namelist, walkers, seed=-1, initial_def=""):
    d = model_dims(namelist)
    n, S, npj, size = 2 * d["ne"], d["nvmc_sample"], d["nproj"], 1 + d["npara"]
    W = walkers
    out = dict(ele_idx=np.zeros(W * S * n, np.int64), proj_cnt=np.zeros(W * S * npj, np.int64),
               counter=np.zeros(W * 6, np.int64), draws=np.zeros(W, np.int64), energy=np.zeros(5),
               ho=np.zeros(size), oo=np.zeros(2 * size), ostore=np.zeros(W * S * size))
    err = err_buf()
    rc = lib().oracle_opt_step1_walkers(namelist.encode(), initial_def.encode(), W, ctypes.c_longlong(seed),
                                        *(ptr(out[k]) for k in ("ele_idx", "proj_cnt", "counter", "draws",
                                                                "energy", "ho", "oo", "ostore")), err, 1024)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    out["ostore"] = out["ostore"].reshape(W * S, size)
    return d, out


def trace_chain(namelist, walker, blocks, max_ops, seed=-1, initial_def=""):
    """One FP64 oracle chain with its long-double shadow (oracle_trace_chain): returns
    (idx0[n], ops[k][7], cands[k][n], rec[k][8])."""
    d = model_dims(namelist)
    n = 2 * d["ne"]
    idx0 = np.zeros(n, np.int64)
    ops = np.zeros((max_ops, 7), np.int32)
    cands = np.zeros((max_ops, n), np.int64)
    rec = np.zeros((max_ops, 8))
    k = ctypes.c_int(0)
    err = err_buf()
    rc = lib().oracle_trace_chain(namelist.encode(), initial_def.encode(), ctypes.c_longlong(seed), walker, blocks,
                                  max_ops, ptr(idx0), ptr(ops), ptr(cands), ptr(rec), ctypes.byref(k), err, 1024)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    k = k.value
    return idx0, ops[:k], cands[:k], rec[:k]


def qp_weights(namelist):
    out = np.zeros(model_dims(namelist)["nqp"])
    err = err_buf()
    if lib().oracle_qp_weights(namelist.encode(), ptr(out), err, 1024) != 0:
        raise RuntimeError(err.value.decode())
    return out


def stage_replay(namelist, params, idx0, ops, idx_seq, nqp, n):
    """Teacher-forced replay of the stage operations; returns (out[nops][nqp], inv[nqp][n][n])."""
    params = np.ascontiguousarray(params, dtype=np.float64)
    idx0 = np.ascontiguousarray(idx0, dtype=np.int64)
    ops = np.ascontiguousarray(ops, dtype=np.int32).reshape(-1, 7)
    idx_seq = np.ascontiguousarray(idx_seq, dtype=np.int64)
    out = np.zeros((len(ops), nqp))
    inv = np.zeros(nqp * n * n)
    err = err_buf()
    rc = lib().oracle_stage_replay(namelist.encode(), ptr(params), len(params), ptr(idx0), len(ops), ptr(ops),
                                   ptr(idx_seq), ptr(out), ptr(inv), err, 1024)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    return out, inv.reshape(nqp, n, n)


def cholesky_solve(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64).copy()
    b = np.ascontiguousarray(b, dtype=np.float64).copy()
    info = lib().oracle_cholesky_solve(ptr(a), ptr(b), len(b))
    return info, b


def green_identity(namelist, zqp, seed=1):
    out = np.zeros(3)
    err = err_buf()
    if lib().oracle_green_identity(namelist.encode(), zqp.encode(), ctypes.c_longlong(seed), ptr(out), err, 1024) != 0:
        raise RuntimeError(err.value.decode())
    return out
