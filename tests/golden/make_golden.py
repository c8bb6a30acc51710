"""Collect the reference's golden vectors for the VMC hot path into tests/golden/.

The reference (AtelierArith/mvmc-rs) pins its CPU path with outputs of the native
C mVMC 1.4.0 program and of the C SFMT library, checked in as data under
`tests/fixtures/` and inside `crates/sfmt19937/tests/golden_vs_c.rs`. This script
copies the subset that covers the real sz-conserved path (inputs, C outputs) and
turns the SFMT table into JSON. It only reads the reference tree; run it where the
reference is mounted:

    python tests/golden/make_golden.py /path/to/mvmc-rs
"""
import json
import os
import re
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def copy_tree(src, dst, names=None):
    os.makedirs(dst, exist_ok=True)
    for name in sorted(os.listdir(src)):
        if names is not None and name not in names:
            continue
        path = os.path.join(src, name)
        if os.path.isfile(path):
            shutil.copyfile(path, os.path.join(dst, name))


def sfmt_table(ref):
    text = open(os.path.join(ref, "crates/sfmt19937/tests/golden_vs_c.rs")).read()
    block = text[text.index("GOLDEN_FIRST8_U32"):]
    block = block[: block.index("];")]
    out = {}
    for seed, words in re.findall(r"\(\s*([0-9_]+|u32::MAX),\s*\[([^\]]*)\]", block):
        s = 0xFFFFFFFF if seed == "u32::MAX" else int(seed.replace("_", ""))
        out[str(s)] = [int(w.replace("_", ""), 16) for w in re.findall(r"0x[0-9a-f_]+", words)]
    return out


def main(ref):
    fx = os.path.join(ref, "tests/fixtures")
    with open(os.path.join(HERE, "sfmt_first8.json"), "w") as f:
        json.dump(sfmt_table(ref), f, indent=1)

    # Native C sampler trajectory at fixed parameters (every saved configuration).
    src = os.path.join(fx, "native_c_physcal_181/hubbard_chain_real")
    dst = os.path.join(HERE, "physcal_hubbard_chain_real")
    copy_tree(os.path.join(src, "inputs"), os.path.join(dst, "inputs"))
    shutil.copyfile(os.path.join(src, "zqp_opt.dat"), os.path.join(dst, "zqp_opt.dat"))
    copy_tree(os.path.join(src, "native-state"), os.path.join(dst, "native-state"))
    physcal = {f"zvo_{kind}_{idx:03d}.dat" for idx in (7, 8)
               for kind in ("out", "var", "cisajs", "cisajscktalt", "cisajscktaltex")}
    copy_tree(os.path.join(src, "expected"), os.path.join(dst, "expected"), names=physcal)
    # The same inputs run as 2 and 4 MPI ranks (chains seeded RndSeed + rank): only the
    # C outputs differ.
    for ranks in (2, 4):
        other = src + f"_mpi{ranks}"
        for name in sorted(os.listdir(os.path.join(src, "inputs"))):
            a = open(os.path.join(src, "inputs", name), "rb").read()
            b = open(os.path.join(other, "inputs", name), "rb").read()
            assert a == b, (other, name)
        copy_tree(os.path.join(other, "expected"), os.path.join(dst, f"expected_mpi{ranks}"), names=physcal)

    # Native C step-1 SR operands (energy, HO, <O>, <O^2>, last O) for the Hubbard chain.
    src = os.path.join(fx, "c_order_sr_operands")
    dst = os.path.join(HERE, "sr_operands_hubbard")
    copy_tree(os.path.join(src, "inputs/hubbard"), os.path.join(dst, "inputs"))
    shutil.copyfile(os.path.join(src, "hubbard-cg-store0.txt"), os.path.join(dst, "hubbard-cg-store0.txt"))

    # Skew-symmetric test matrices (identities Pf^2 = det, inverse residual).
    src = os.path.join(fx, "pfapack")
    copy_tree(src, os.path.join(HERE, "pfapack"),
              names={f for f in os.listdir(src) if f.startswith("real_n") and
                     int(f.split("_")[1][1:]) <= 64})

    # Complex skew test matrices (identities of the complex Pfaffian + inverse).
    copy_tree(src, os.path.join(HERE, "pfapack_complex"),
              names={f for f in os.listdir(src) if f.startswith("complex_n") and
                     int(f.split("_")[1][1:]) <= 128})

    # C StochasticOptCG iterates on fixed operands (tol 0, shift 1e-5).
    copy_tree(os.path.join(fx, "sr_cg/c_refresh"), os.path.join(HERE, "sr_cg"),
              names={"real.txt", "real_diag_scale.txt"})


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
