"""Host-driven Metropolis-like chains for the stage replay tests: random hops and
exchanges on a fixed configuration, each proposal followed by an accept half of the time,
and a recompute every few moves. The candidate configuration (move applied) is passed with
every call, as the reference's sampler does around its stage calls."""
import numpy as np

PROPOSE_HOP, ACCEPT_HOP, PROPOSE_EX, ACCEPT_EX, RECOMPUTE = 0, 1, 2, 3, 4


def random_configuration(rng, ns, ne):
    up = rng.choice(ns, ne, replace=False)
    dn = rng.choice(ns, ne, replace=False)
    return np.concatenate([up, dn]).astype(np.int64)


def random_sequence(rng, idx0, ns, ne, moves, ex_frac=0.3, recompute_every=16):
    idx = np.array(idx0, dtype=np.int64)
    ops, seq = [], []
    for k in range(moves):
        up, dn = set(idx[:ne].tolist()), set(idx[ne:].tolist())
        if rng.random() < ex_frac:
            ca = [m for m in range(ne) if int(idx[m]) not in dn]
            cb = [m for m in range(ne) if int(idx[ne + m]) not in up]
            if ca and cb:
                ma, mb = int(rng.choice(ca)), int(rng.choice(cb))
                ra, rb = int(idx[ma]), int(idx[ne + mb])
                cand = idx.copy()
                cand[ma], cand[ne + mb] = rb, ra
                ops.append([PROPOSE_EX, ma, 0, mb, 1, 0, 0])
                seq.append(cand)
                if rng.random() < 0.5:
                    ops.append([ACCEPT_EX, ma, 0, mb, 1, ra, rb])
                    seq.append(cand)
                    idx = cand
        else:
            s = int(rng.integers(2))
            ma = int(rng.integers(ne))
            occ = up if s == 0 else dn
            free = [r for r in range(ns) if r not in occ]
            rj = int(rng.choice(free))
            cand = idx.copy()
            cand[ma + s * ne] = rj
            ops.append([PROPOSE_HOP, ma, s, 0, 0, 0, 0])
            seq.append(cand)
            if rng.random() < 0.5:
                ops.append([ACCEPT_HOP, ma, s, 0, 0, 0, 0])
                seq.append(cand)
                idx = cand
        if (k + 1) % recompute_every == 0:
            ops.append([RECOMPUTE, 0, 0, 0, 0, 0, 0])
            seq.append(idx.copy())
    return np.array(ops, dtype=np.int32), np.array(seq, dtype=np.int64), idx
