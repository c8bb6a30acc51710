"""Python binding of the mvmc-b200 C ABI (include/mvmc_b200.h) through ctypes.

The library is built in-tree (`make -C mvmc-rs_b200`, or `__graft_entry__.build()`).
There is no CPU fallback: loading fails loudly when the shared library is missing, and
every compute call raises when the CUDA path reports an error.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libmvmc_b200.so")
_LIB = None

EXPORTS = [
    "mvmc_b200_pfinv_batch", "mvmc_b200_pfinv_batch_mixed", "mvmc_b200_pfinv_batch_device",
    "mvmc_b200_default_options", "mvmc_b200_create", "mvmc_b200_destroy", "mvmc_b200_dims",
    "mvmc_b200_get_parameters", "mvmc_b200_set_parameters", "mvmc_b200_sample",
    "mvmc_b200_get_samples", "mvmc_b200_measure", "mvmc_b200_get_o_store",
    "mvmc_b200_get_local_energies", "mvmc_b200_sr_cg", "mvmc_b200_status", "mvmc_b200_run_opt",
    "mvmc_b200_last_error", "mvmc_b200_cg_solve", "mvmc_b200_stream", "mvmc_b200_transfer_bytes",
    "mvmc_b200_sampler_timers", "mvmc_b200_cg_solve_noalloc", "mvmc_b200_refresh_stats",
    "mvmc_b200_get_log_amplitudes", "mvmc_b200_stage_create", "mvmc_b200_stage_destroy",
    "mvmc_b200_stage_begin", "mvmc_b200_stage_propose_hop", "mvmc_b200_stage_accept_hop",
    "mvmc_b200_stage_propose_exchange", "mvmc_b200_stage_accept_exchange", "mvmc_b200_stage_recompute",
    "mvmc_b200_stage_state", "mvmc_b200_gram", "mvmc_b200_cholesky_solve",
    "mvmc_b200_measure_sums", "mvmc_b200_sr_gather", "mvmc_b200_sr_local_product", "mvmc_b200_sr_apply",
    "mvmc_b200_sr_config", "mvmc_b200_physcal_create", "mvmc_b200_green_dims", "mvmc_b200_measure_green",
    "mvmc_b200_run_physcal", "mvmc_b200_pfinv_batch_complex", "mvmc_b200_pfinv_batch_complex_device",
    "mvmc_b200_gram_tc", "mvmc_b200_sr_local_product_device",
]


class Options(ctypes.Structure):
    _fields_ = [("walkers", ctypes.c_int), ("precision", ctypes.c_int),
                ("refresh_sweeps", ctypes.c_int), ("saved_per_walker", ctypes.c_int),
                ("seed", ctypes.c_longlong), ("device", ctypes.c_int), ("sr_precision", ctypes.c_int),
                ("refresh_guard", ctypes.c_double), ("c_order", ctypes.c_int), ("sr_gram", ctypes.c_int),
                ("measure_resident", ctypes.c_int)]


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"mvmc_b200: CUDA library not built ({LIB_PATH}); run make -C mvmc-rs_b200")
        _LIB = ctypes.CDLL(LIB_PATH)
        _LIB.mvmc_b200_last_error.restype = ctypes.c_char_p
        _LIB.mvmc_b200_stream.restype = ctypes.c_void_p
    return _LIB


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _check(rc, what):
    if rc < 0:
        msg = lib().mvmc_b200_last_error()
        raise RuntimeError(f"{what} failed with status {rc}: {msg.decode() if msg else ''}")
    return rc


def pfinv_batch(x_colmajor, n, planes):
    """Batched Pfaffian and inverse of column-major skew planes (true X^-1 returned)."""
    x = np.ascontiguousarray(x_colmajor, dtype=np.float64)
    pf = np.zeros(planes)
    inv = np.zeros(planes * n * n)
    st = np.zeros(planes, dtype=np.int32)
    _check(lib().mvmc_b200_pfinv_batch(_ptr(x), n, planes, _ptr(pf), _ptr(inv), _ptr(st)), "pfinv_batch")
    return pf, inv, st


def pfinv_batch_complex(x_colmajor, n, planes):
    """Complex skew planes (column-major, complex128): Pf (complex) and the true X⁻¹."""
    x = np.ascontiguousarray(x_colmajor, dtype=np.complex128)
    pf = np.zeros(planes, dtype=np.complex128)
    inv = np.zeros(x.size, dtype=np.complex128)
    st = np.zeros(planes, dtype=np.int32)
    _check(lib().mvmc_b200_pfinv_batch_complex(_ptr(x), n, planes, _ptr(pf), _ptr(inv), _ptr(st)),
           "pfinv_batch_complex")
    return pf, inv, st


def pfinv_batch_mixed(x, sizes, precision=64):
    x = np.ascontiguousarray(x, dtype=np.float64)
    sizes = np.ascontiguousarray(sizes, dtype=np.int32)
    planes = len(sizes)
    pf = np.zeros(planes)
    inv = np.zeros(x.size)
    st = np.zeros(planes, dtype=np.int32)
    _check(lib().mvmc_b200_pfinv_batch_mixed(_ptr(x), _ptr(sizes), planes, precision, _ptr(pf),
                                             _ptr(inv), _ptr(st)), "pfinv_batch_mixed")
    return pf, inv, st


def cg_solve(samples, mean, diag, g, inv_w, shift, tol, max_iter, diag_scale=False):
    """SR-CG on fixed operands; samples is [ns][na]."""
    samples = np.ascontiguousarray(samples, dtype=np.float64)
    na = len(mean)
    ns = samples.size // na
    x = np.zeros(na)
    st = ctypes.c_longlong()
    _check(lib().mvmc_b200_cg_solve(_ptr(samples), ctypes.c_longlong(ns), na,
                                    _ptr(np.ascontiguousarray(mean, dtype=np.float64)),
                                    _ptr(np.ascontiguousarray(diag, dtype=np.float64)),
                                    _ptr(np.ascontiguousarray(g, dtype=np.float64)),
                                    ctypes.c_double(inv_w), ctypes.c_double(shift), ctypes.c_double(tol),
                                    max_iter, int(diag_scale), _ptr(x), ctypes.byref(st)), "cg_solve")
    return st.value, x


def cg_solve_noalloc(samples_ptr, ns, na, mean_ptr, diag_ptr, g_ptr, inv_w, shift, tol, max_iter,
                     diag_scale, x_ptr, result_ptr, stream=0):
    """SR-CG on device buffers (integer device addresses) with no device allocation by the
    library; result_ptr receives {delta, status, iterations}. Returns the C status code."""
    vp = ctypes.c_void_p
    return _check(lib().mvmc_b200_cg_solve_noalloc(
        vp(samples_ptr), ctypes.c_longlong(ns), na, vp(mean_ptr), vp(diag_ptr), vp(g_ptr),
        ctypes.c_double(inv_w), ctypes.c_double(shift), ctypes.c_double(tol), max_iter, int(diag_scale),
        vp(x_ptr), vp(result_ptr), vp(stream)), "cg_solve_noalloc")


def gram(store):
    """out = Σ_s store[s] store[s]ᵀ for store of shape [samples, n] (device kernel)."""
    store = np.ascontiguousarray(store, dtype=np.float64)
    samples, n = store.shape
    out = np.zeros((n, n))
    _check(lib().mvmc_b200_gram(_ptr(store), n, ctypes.c_longlong(samples), _ptr(out)), "gram")
    return out


def gram_tc(samples, precision=16):
    """Σ_s x_s x_sᵀ (FP32) of samples [ns, na] on the tensor cores: BF16 (16) or TF32 (32)
    inputs, FP32 accumulation. Raises when a bounded device wait expired."""
    samples = np.ascontiguousarray(samples, dtype=np.float64)
    ns, na = samples.shape
    out = np.zeros((na, na), dtype=np.float32)
    rc = _check(lib().mvmc_b200_gram_tc(_ptr(samples), ctypes.c_longlong(ns), na, precision, _ptr(out)), "gram_tc")
    if rc != 0:
        raise RuntimeError("gram_tc: a bounded device wait expired")
    return out


def cholesky_solve(s, rhs):
    """Solve S x = rhs (S symmetric positive definite) on the device; returns (status, x)
    with status 1 for a failed factorisation."""
    s = np.ascontiguousarray(s, dtype=np.float64)
    x = np.ascontiguousarray(rhs, dtype=np.float64).copy()
    rc = _check(lib().mvmc_b200_cholesky_solve(_ptr(s), _ptr(x), len(x)), "cholesky_solve")
    return rc, x


def default_options(**kw):
    o = Options()
    lib().mvmc_b200_default_options(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class Engine:
    """Walker-ensemble engine: sample → measure → SR-CG on the device."""

    def __init__(self, namelist, initial_def="", physcal_zqp=None, **options):
        """physcal_zqp: a zqp_opt.dat path selects the PhysCal form (fixed parameters,
        Green functions); otherwise initial_def optionally seeds the optimisation."""
        self.opt = default_options(**options)
        self.ctx = ctypes.c_void_p()
        if physcal_zqp:
            _check(lib().mvmc_b200_physcal_create(namelist.encode(), physcal_zqp.encode(),
                                                  ctypes.byref(self.opt), ctypes.byref(self.ctx)), "physcal_create")
        else:
            _check(lib().mvmc_b200_create(namelist.encode(), (initial_def or "").encode(),
                                          ctypes.byref(self.opt), ctypes.byref(self.ctx)), "create")
        g = (ctypes.c_int * 5)()
        _check(lib().mvmc_b200_green_dims(self.ctx, g), "green_dims")
        self.green_dims = dict(zip(["one", "ex", "two", "blocks", "idx_start"], list(g)))
        d = (ctypes.c_int * 8)()
        _check(lib().mvmc_b200_dims(self.ctx, d), "dims")
        keys = ["nsite", "ne", "nqp", "nproj", "npara", "saved", "walkers", "n_orb"]
        self.dims = dict(zip(keys, list(d)))

    def close(self):
        if self.ctx:
            lib().mvmc_b200_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def sr_size(self):
        return 1 + self.dims["npara"]

    def parameters(self):
        p = np.zeros(self.dims["npara"])
        _check(lib().mvmc_b200_get_parameters(self.ctx, _ptr(p), len(p)), "get_parameters")
        return p

    def set_parameters(self, p):
        p = np.ascontiguousarray(p, dtype=np.float64)
        _check(lib().mvmc_b200_set_parameters(self.ctx, _ptr(p), len(p)), "set_parameters")

    def sample(self):
        _check(lib().mvmc_b200_sample(self.ctx), "sample")

    def samples(self):
        d = self.dims
        W, S, n, ns2 = d["walkers"], d["saved"], 2 * d["ne"], 2 * d["nsite"]
        out = dict(ele_idx=np.zeros(W * S * n, np.int64), ele_cfg=np.zeros(W * S * ns2, np.int64),
                   ele_num=np.zeros(W * S * ns2, np.int64),
                   proj_cnt=np.zeros(W * S * d["nproj"], np.int64),
                   counter=np.zeros(W * 6, np.int64), draws=np.zeros(W, np.int64))
        _check(lib().mvmc_b200_get_samples(self.ctx, *(_ptr(out[k]) for k in (
            "ele_idx", "ele_cfg", "ele_num", "proj_cnt", "counter", "draws"))), "get_samples")
        return out

    def measure(self):
        e = np.zeros(5)
        ho = np.zeros(self.sr_size)
        oo = np.zeros(2 * self.sr_size)
        _check(lib().mvmc_b200_measure(self.ctx, _ptr(e), _ptr(ho), _ptr(oo)), "measure")
        return e, ho, oo

    def measure_green(self):
        """PhysCal measurement: energy[5] (Wc, <E>, <E^2>, <Sz>, <Sz^2>) and the one-body,
        TwoBodyGEx and TwoBodyG Green functions."""
        g = self.green_dims
        e = np.zeros(5)
        one, ex, two = np.zeros(g["one"]), np.zeros(g["ex"]), np.zeros(g["two"])
        _check(lib().mvmc_b200_measure_green(self.ctx, _ptr(e), _ptr(one), _ptr(ex), _ptr(two)), "measure_green")
        return e, one, ex, two

    def o_store(self):
        d = self.dims
        out = np.zeros(d["walkers"] * d["saved"] * self.sr_size)
        _check(lib().mvmc_b200_get_o_store(self.ctx, _ptr(out), ctypes.c_longlong(out.size)), "o_store")
        return out.reshape(d["walkers"] * d["saved"], self.sr_size)

    def local_energies(self):
        d = self.dims
        out = np.zeros(d["walkers"] * d["saved"])
        _check(lib().mvmc_b200_get_local_energies(self.ctx, _ptr(out), ctypes.c_longlong(out.size)),
               "local_energies")
        return out

    def log_amplitudes(self):
        """ln|Psi(x)| of every saved sample from the last measurement."""
        d = self.dims
        out = np.zeros(d["walkers"] * d["saved"])
        _check(lib().mvmc_b200_get_log_amplitudes(self.ctx, _ptr(out), ctypes.c_longlong(out.size)),
               "log_amplitudes")
        return out

    def measure_sums(self):
        """Sums of the last measurement before the weight average (Wc first)."""
        out = np.zeros(5 + 3 * self.sr_size)
        _check(lib().mvmc_b200_measure_sums(self.ctx, _ptr(out)), "measure_sums")
        return out

    def sr_gather(self, mapping):
        m = np.ascontiguousarray(mapping, dtype=np.int32)
        _check(lib().mvmc_b200_sr_gather(self.ctx, _ptr(m), len(m)), "sr_gather")

    def sr_local_product(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        z = np.zeros_like(v)
        _check(lib().mvmc_b200_sr_local_product(self.ctx, _ptr(v), _ptr(z)), "sr_local_product")
        return z

    def sr_local_product_device(self, v, z, stream):
        """z = Σ_s O_s (O_s·v) on device buffers (CUDA float64 tensors of n_active values, or
        integer device addresses), ordered on `stream` (an integer cudaStream_t handle)."""
        vp = ctypes.c_void_p
        addr = lambda t: t.data_ptr() if hasattr(t, "data_ptr") else int(t)
        _check(lib().mvmc_b200_sr_local_product_device(self.ctx, vp(addr(v)), vp(addr(z)), vp(stream)),
               "sr_local_product_device")

    def sr_apply(self, mapping, x):
        m = np.ascontiguousarray(mapping, dtype=np.int32)
        x = np.ascontiguousarray(x, dtype=np.float64)
        _check(lib().mvmc_b200_sr_apply(self.ctx, _ptr(m), len(m), _ptr(x)), "sr_apply")

    def sr_config(self):
        cfg = np.zeros(10)
        flags = np.zeros(2 * self.dims["npara"], dtype=np.int32)
        _check(lib().mvmc_b200_sr_config(self.ctx, _ptr(cfg), _ptr(flags)), "sr_config")
        keys = ["nsrcg", "red_cut", "step_dt", "sta_del", "cg_tol", "cg_max_iter", "diag_scale", "cg_fallback",
                "cg_abort", "npara"]
        return dict(zip(keys, cfg.tolist())), flags

    def sr_cg(self):
        info = np.zeros(9)
        rc = _check(lib().mvmc_b200_sr_cg(self.ctx, _ptr(info)), "sr_cg")
        return rc, info

    def stream(self):
        """The engine's cudaStream_t as an integer handle."""
        return lib().mvmc_b200_stream(self.ctx)

    def transfer_bytes(self):
        h, d = ctypes.c_longlong(), ctypes.c_longlong()
        _check(lib().mvmc_b200_transfer_bytes(self.ctx, ctypes.byref(h), ctypes.byref(d)), "transfer_bytes")
        return h.value, d.value

    def refresh_stats(self):
        """{drift_max, drift_mean, scheduled refreshes / walker, guard refreshes / walker}."""
        st = np.zeros(4)
        _check(lib().mvmc_b200_refresh_stats(self.ctx, _ptr(st)), "refresh_stats")
        return dict(drift_max=st[0], drift_mean=st[1], refreshes=st[2], guard_refreshes=st[3])

    def refresh_drift(self):
        st = self.refresh_stats()
        return st["drift_max"], st["drift_mean"]

    def sampler_timers(self):
        c = np.zeros(8)
        _check(lib().mvmc_b200_sampler_timers(self.ctx, _ptr(c)), "sampler_timers")
        keys = ["candidate", "ratio", "metropolis", "update", "refresh", "total"]
        return dict(zip(keys, c[:6].tolist()))

    def status(self):
        s = ctypes.c_uint()
        _check(lib().mvmc_b200_status(self.ctx, ctypes.byref(s)), "status")
        return s.value


def run_opt(namelist, out_dir, initial_def="", nsteps=0, **options):
    opt = default_options(**options)
    _check(lib().mvmc_b200_run_opt(namelist.encode(), (initial_def or "").encode(), out_dir.encode(),
                                   ctypes.byref(opt), nsteps), "run_opt")


def run_physcal(namelist, zqp_opt, out_dir, **options):
    """PhysCal run writing zvo_out_NNN / zvo_var_NNN / zvo_cisajs* files into out_dir."""
    opt = default_options(**options)
    _check(lib().mvmc_b200_run_physcal(namelist.encode(), zqp_opt.encode(), out_dir.encode(), ctypes.byref(opt)),
           "run_physcal")


class Stage:
    """One walker's device Pfaffian stage (RealPfStage) over an Engine's model."""

    def __init__(self, engine):
        self.engine = engine
        self.h = ctypes.c_void_p()
        _check(lib().mvmc_b200_stage_create(engine.ctx, ctypes.byref(self.h)), "stage_create")
        d = engine.dims
        self.nqp, self.n, self.ne = d["nqp"], 2 * d["ne"], d["ne"]

    def close(self):
        if self.h:
            lib().mvmc_b200_stage_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _idx(ele_idx):
        return np.ascontiguousarray(ele_idx, dtype=np.int64)

    def begin(self, ele_idx):
        pf = np.zeros(self.nqp)
        idx = self._idx(ele_idx)
        return _check(lib().mvmc_b200_stage_begin(self.h, _ptr(idx), _ptr(pf)), "stage_begin"), pf

    def recompute(self, ele_idx):
        pf = np.zeros(self.nqp)
        idx = self._idx(ele_idx)
        return _check(lib().mvmc_b200_stage_recompute(self.h, _ptr(idx), _ptr(pf)), "stage_recompute"), pf

    def propose_hop(self, ele_idx, ma, spin):
        pf = np.zeros(self.nqp)
        idx = self._idx(ele_idx)
        _check(lib().mvmc_b200_stage_propose_hop(self.h, _ptr(idx), ma, spin, _ptr(pf)), "stage_propose_hop")
        return pf

    def accept_hop(self, ele_idx, ma, spin, pf_new=None):
        idx = self._idx(ele_idx)
        p = None if pf_new is None else np.ascontiguousarray(pf_new, dtype=np.float64)
        _check(lib().mvmc_b200_stage_accept_hop(self.h, _ptr(idx), ma, spin, _ptr(p)), "stage_accept_hop")

    def propose_exchange(self, ele_idx, ma, sa, mb, sb):
        pf = np.zeros(self.nqp)
        idx = self._idx(ele_idx)
        _check(lib().mvmc_b200_stage_propose_exchange(self.h, _ptr(idx), ma, sa, mb, sb, _ptr(pf)),
               "stage_propose_exchange")
        return pf

    def accept_exchange(self, ele_idx, ma, sa, mb, sb, ra_old, rb_old):
        idx = self._idx(ele_idx)
        _check(lib().mvmc_b200_stage_accept_exchange(self.h, _ptr(idx), ma, sa, mb, sb, ra_old, rb_old),
               "stage_accept_exchange")

    def state(self):
        pf = np.zeros(self.nqp)
        inv = np.zeros(self.nqp * self.n * self.n)
        _check(lib().mvmc_b200_stage_state(self.h, _ptr(pf), _ptr(inv)), "stage_state")
        return pf, inv.reshape(self.nqp, self.n, self.n)
