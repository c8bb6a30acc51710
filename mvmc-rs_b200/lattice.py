"""Expert-mode input generator for Hubbard models on chains and square lattices.

Writes the definition files the real sz-conserved optimiser reads (namelist.def,
modpara.def, locspn.def, trans.def, coulombintra.def, gutzwilleridx.def, jastrowidx.def,
orbitalidx.def, qptransidx.def) in the Expert-mode layout of mVMC (five header lines,
the count on line 2, optimisation flags after the index block), plus an initial.def
whose parameters are drawn uniform[-0.05, 0.05] from a seeded generator.

Model conventions:
  * Transfer lines "i s j s t" encode the term -t c†_{i s} c_{j s}; both directions are
    listed. Nearest neighbours carry t, next-nearest (square lattice) carry t'.
  * Pair orbitals f_ij are indexed by (sublattice of i, displacement j - i) with a
    configurable sublattice size; full translation symmetry is a 1×1 sublattice.
  * Jastrow factors are indexed by displacement classes identified under inversion
    (d ~ -d), the distance-resolved Jastrow of the reference's examples.
  * Momentum projection uses the translations by the sublattice vectors with weight 1;
    spin projection uses NSPGaussLeg Gauss–Legendre points (NSPStot 0).
"""
import os

import numpy as np

HEADER = "======================\n"


def _def_file(path, label, count, body, complex_type=None):
    with open(path, "w") as f:
        f.write(HEADER)
        f.write(f"{label} {count}\n")
        f.write(f"ComplexType {complex_type}\n" if complex_type is not None else HEADER)
        f.write(HEADER)
        f.write(HEADER)
        f.write(body)


class Lattice:
    def __init__(self, lx, ly=1):
        self.lx, self.ly = lx, ly
        self.n = lx * ly

    def site(self, x, y):
        return (x % self.lx) + self.lx * (y % self.ly)

    def coord(self, i):
        return i % self.lx, i // self.lx

    def disp(self, i, j):
        (xi, yi), (xj, yj) = self.coord(i), self.coord(j)
        return (xj - xi) % self.lx, (yj - yi) % self.ly

    def neighbours(self, i, t, tp):
        x, y = self.coord(i)
        out = [(self.site(x + 1, y), t), (self.site(x - 1, y), t)]
        if self.ly > 1:
            out += [(self.site(x, y + 1), t), (self.site(x, y - 1), t)]
            if tp != 0.0:
                out += [(self.site(x + dx, y + dy), tp) for dx in (1, -1) for dy in (1, -1)]
        return out


def write_inputs(out_dir, lx, ly=1, t=1.0, tp=0.0, U=4.0, n_up=None, sub=(1, 1), nmp=1, shifts=None,
                 nsp_gauss_leg=1, warmup=10, interval=1, samples=10, steps=10, ex_path=1,
                 seed=12345, step_dt=0.02, red_cut=1e-8, sta_del=0.02, param_seed=2024,
                 cg_max_iter=200, cg_tol=1e-6, cg_abort=0, nsrcg=1, calc_mode=0, green=None, data_qty=1,
                 V=0.0, J_hund=0.0):
    """Write a complete input set; returns (namelist path, initial.def path, dims).

    V and J_hund add nearest-neighbour CoulombInter (V n_i n_j) and Hund
    (−J (n_i↑n_j↑ + n_i↓n_j↓)) terms on every bond.
    calc_mode=1 writes a PhysCal set (NVMCCalMode 1, NDataQtySmp data_qty) whose fixed
    parameters are initial.def; green="corr" adds the correlation lists: every same-spin
    one-body term c†_{i s} c_{j s} (2·Ns² terms) and every density-density term
    n_{i s} n_{j t} = c†_{i s} c_{i s} c†_{j t} c_{j t} (4·Ns² terms)."""
    os.makedirs(out_dir, exist_ok=True)
    lat = Lattice(lx, ly)
    ns = lat.n
    n_up = ns // 2 if n_up is None else n_up
    files = dict(ModPara="modpara.def", LocSpin="locspn.def", Trans="trans.def",
                 CoulombIntra="coulombintra.def", Gutzwiller="gutzwilleridx.def",
                 Jastrow="jastrowidx.def", Orbital="orbitalidx.def", TransSym="qptransidx.def")
    if V != 0.0:
        files["CoulombInter"] = "coulombinter.def"
    if J_hund != 0.0:
        files["Hund"] = "hund.def"
    if green == "corr":
        files.update(OneBodyG="greenone.def", TwoBodyG="greentwo.def")
    elif green is not None:
        raise ValueError(f"unknown Green list {green!r}")
    with open(os.path.join(out_dir, "namelist.def"), "w") as f:
        for k, v in files.items():
            f.write(f"{k:>16s}  {v}\n")
    mod = dict(NVMCCalMode=calc_mode, Nsite=ns, Ncond=2 * n_up, **{"2Sz": 0}, NSPGaussLeg=nsp_gauss_leg,
               NSPStot=0, NMPTrans=nmp, NSROptItrStep=steps, NSROptItrSmp=max(1, steps // 10),
               DSROptRedCut=red_cut, DSROptStaDel=sta_del, DSROptStepDt=step_dt, NVMCWarmUp=warmup,
               NVMCInterval=interval, NVMCSample=samples, NExUpdatePath=ex_path, RndSeed=seed,
               NSplitSize=1, NStore=1, NSRCG=nsrcg, NSROptCGMaxIter=cg_max_iter, DSROptCGTol=cg_tol,
               NSRCGAbortOnFail=cg_abort, NDataIdxStart=0, NDataQtySmp=data_qty)
    with open(os.path.join(out_dir, "modpara.def"), "w") as f:
        f.write("--------------------\nModel_Parameters   0\n--------------------\n"
                "VMC_Cal_Parameters\n--------------------\nCDataFileHead  zvo\n"
                "CParaFileHead  zqp\n--------------------\n")
        for k, v in mod.items():
            f.write(f"{k:<14s} {v}\n")
    if green == "corr":
        _def_file(os.path.join(out_dir, "greenone.def"), "NCisAjs", 2 * ns * ns,
                  "".join(f"{i:5d} {s:5d} {j:5d} {s:5d}\n" for s in (0, 1) for i in range(ns) for j in range(ns)))
        _def_file(os.path.join(out_dir, "greentwo.def"), "NCisAjsCktAltDC", 4 * ns * ns,
                  "".join(f"{i:5d} {s:5d} {i:5d} {s:5d} {j:5d} {t:5d} {j:5d} {t:5d}\n"
                          for i in range(ns) for j in range(ns) for s in (0, 1) for t in (0, 1)))
    _def_file(os.path.join(out_dir, "locspn.def"), "NlocalSpin", 0,
              "".join(f"{i:5d} 0\n" for i in range(ns)))
    lines = []
    for i in range(ns):
        for j, amp in lat.neighbours(i, t, tp):
            for s in (0, 1):
                lines.append(f"{i:5d} {s:5d} {j:5d} {s:5d} {amp: .15f} {0.0: .15f}\n")
    _def_file(os.path.join(out_dir, "trans.def"), "NTransfer", len(lines), "".join(lines))
    bonds = sorted({(min(i, j), max(i, j)) for i in range(ns) for j, _ in lat.neighbours(i, t, 0.0) if i != j})
    if V != 0.0:
        _def_file(os.path.join(out_dir, "coulombinter.def"), "NCoulombInter", len(bonds),
                  "".join(f"{i:5d} {j:5d} {V: .15f}\n" for i, j in bonds))
    if J_hund != 0.0:
        _def_file(os.path.join(out_dir, "hund.def"), "NHund", len(bonds),
                  "".join(f"{i:5d} {j:5d} {J_hund: .15f}\n" for i, j in bonds))
    _def_file(os.path.join(out_dir, "coulombintra.def"), "NCoulombIntra", ns,
              "".join(f"{i:5d} {U: .15f}\n" for i in range(ns)))
    _def_file(os.path.join(out_dir, "gutzwilleridx.def"), "NGutzwillerIdx", 1,
              "".join(f"{i:5d} 0\n" for i in range(ns)) + "    0 1\n", complex_type=0)
    # Jastrow: displacement classes under inversion
    cls = {}
    jl = []
    for i in range(ns):
        for j in range(ns):
            if i == j:
                continue
            dx, dy = lat.disp(i, j)
            key = min((dx, dy), ((-dx) % lx, (-dy) % ly))
            if key not in cls:
                cls[key] = len(cls)
            jl.append(f"{i:5d} {j:5d} {cls[key]:5d}\n")
    nj = len(cls)
    _def_file(os.path.join(out_dir, "jastrowidx.def"), "NJastrowIdx", nj,
              "".join(jl) + "".join(f"{k:5d} 1\n" for k in range(nj)), complex_type=0)
    # Orbitals: (sublattice of i, displacement)
    sx, sy = sub
    nsub = sx * sy
    ol = []
    for i in range(ns):
        xi, yi = lat.coord(i)
        s_idx = (xi % sx) + sx * (yi % sy)
        for j in range(ns):
            dx, dy = lat.disp(i, j)
            idx = s_idx * ns + dx + lx * dy
            ol.append(f"{i:5d} {j:5d} {idx:5d}\n")
    no = nsub * ns
    _def_file(os.path.join(out_dir, "orbitalidx.def"), "NOrbitalIdx", no,
              "".join(ol) + "".join(f"{k:5d} 1\n" for k in range(no)), complex_type=0)
    # Momentum projection: translations by sublattice offsets
    if shifts is None:
        shifts = [(dx, dy) for dy in range(sy) for dx in range(sx)][:nmp]
    shifts = list(shifts)[:nmp]
    if len(shifts) < nmp:
        raise ValueError("NMPTrans exceeds the sublattice translations")
    ql = [f"{k} 1.00000\n" for k in range(nmp)]
    for k, (dx, dy) in enumerate(shifts):
        for i in range(ns):
            x, y = lat.coord(i)
            ql.append(f"{k:5d} {i:5d} {lat.site(x + dx, y + dy):5d} 1\n")
    _def_file(os.path.join(out_dir, "qptransidx.def"), "NQPTrans", nmp, "".join(ql))
    npara = 1 + nj + no
    rng = np.random.default_rng(param_seed)
    p = rng.uniform(-0.05, 0.05, size=npara)
    with open(os.path.join(out_dir, "initial.def"), "w") as f:
        f.write("0.0 0.0 0.0 0.0 0.0 0.0\n")
        for v in p:
            f.write(f"{v:.18e} 0.0 0.0\n")
    dims = dict(nsite=ns, ne=n_up, n=2 * n_up, nqp=nsp_gauss_leg * nmp, n_jast=nj, n_orb=no, npara=npara)
    return os.path.join(out_dir, "namelist.def"), os.path.join(out_dir, "initial.def"), dims


# The workloads of the benchmark (sizes as in the north-star configurations).
CONFIGS = {
    # 1D Hubbard chain L=16, U=4, half filling, translation-symmetric f (16), G (1), J (8).
    "chain16": dict(lx=16, ly=1, U=4.0, sub=(1, 1), nmp=1, nsp_gauss_leg=1, interval=16, samples=1,
                    warmup=4, steps=10, seed=12345),
    # 2D 8×8, U=4, half filling, two-sublattice f (128), NQP = 4 translations × 2 spin points.
    "square8": dict(lx=8, ly=8, U=4.0, sub=(2, 1), nmp=4, shifts=[(0, 0), (1, 0), (0, 1), (1, 1)],
                    nsp_gauss_leg=2, interval=64, samples=1,
                    warmup=4, steps=10, seed=12345),
    # 2D 16×16, t'=-0.2, U=6, 1/8 hole doping (112+112), full translation symmetry (256).
    "square16": dict(lx=16, ly=16, U=6.0, tp=-0.2, n_up=112, sub=(1, 1), nmp=1, nsp_gauss_leg=1,
                     interval=1, samples=1, warmup=4, steps=10, seed=12345),
    # As square16 with 4×4-sublattice f (4096).
    "square16_sr": dict(lx=16, ly=16, U=6.0, tp=-0.2, n_up=112, sub=(4, 4), nmp=1, nsp_gauss_leg=1,
                        interval=1, samples=1, warmup=4, steps=50, seed=12345),
    # PhysCal on the square8 model: fixed parameters, energy plus the one-body and the
    # density-density Green functions of every site pair (8192 + 16384 terms).
    "physcal8": dict(lx=8, ly=8, U=4.0, sub=(2, 1), nmp=4, shifts=[(0, 0), (1, 0), (0, 1), (1, 1)],
                     nsp_gauss_leg=2, interval=1, samples=1, warmup=4, steps=10, seed=12345, calc_mode=1,
                     green="corr"),
}
