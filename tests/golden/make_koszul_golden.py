#!/usr/bin/env python3
"""Generate the golden fixtures for the synthetic Koszul block-Wiedemann path.

Run in a container that holds the reference checkout (it imports the
reference's explicit sparse-matrix oracle):

    python tests/golden/make_koszul_golden.py --reference <reference checkout>

The operator d is assembled as an explicit scipy CSR matrix by the
reference's own ``differential()`` (tests/deformation_reference.py:75-89 of
the reference) with ``mu[i] = M_i`` (dim_out x dim_in), source subsets
``combinations(range(r), k)`` and target subsets ``combinations(range(r),
k-1)``.  The square operator is ``S = D d^T d`` and the sequence is
``a_i = X^T S^i Y``.  The seeded inputs follow the counter-based stream that
the engine and the oracle both implement (splitmix64 finaliser over
``seed ^ tag`` and the element index, multiply-shift onto ``[lo, p)``);
this script restates it in numpy so the fixtures pin all three.

Outputs ``tests/golden/koszul_golden.npz``.
"""
import argparse
import hashlib
import itertools
import sys
from pathlib import Path

import numpy as np

MASK = (1 << 64) - 1

# (name, r, k, dim_in, dim_out, p, nb, m, nlen, seed)
CASES = [
    ("tiny", 6, 3, 3, 4, 101, 4, 4, 20, 7),
    ("ragged", 7, 4, 5, 3, 32003, 8, 8, 16, 11),
    ("wide32", 6, 2, 4, 6, 32003, 32, 32, 6, 5),
    # Lambda^4(F^10) (x) R_q, dim R_q = 16, dim R_(q+1) = 24,
    # p = 32003, m = n = 8, 2N/8 + 16 sequence entries with N = 3360.
    ("config1", 10, 4, 16, 24, 32003, 8, 8, 2 * 3360 // 8 + 16, 1),
]

TAG_MAPS, TAG_DIAG, TAG_X, TAG_Y = 1, 2, 3, 4


def mix64(z):
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
    return z ^ (z >> 31)


def seeded_residues(seed, tag, count, p, lo):
    """Vectorised counter-based stream (numpy uint64 arithmetic wraps mod 2^64)."""
    base = mix64((seed ^ ((0xD1B54A32D192ED03 * (tag + 1)) & MASK)) & MASK)
    with np.errstate(over="ignore"):
        idx = np.arange(1, count + 1, dtype=np.uint64)
        z = np.uint64(base) + idx * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    span = p - lo
    # (z * span) >> 64 without 128-bit integers: split z into 32-bit halves.
    hi = (z >> np.uint64(32)).astype(object)
    lo32 = (z & np.uint64(0xFFFFFFFF)).astype(object)
    val = (hi * span + ((lo32 * span) >> 32)) >> 32
    return (np.asarray(val, dtype=np.int64) + lo).astype(np.int64)


def build(case, differential):
    name, r, k, ci, co, p, nb, m, nlen, seed = case
    src = list(itertools.combinations(range(r), k))
    tgt = list(itertools.combinations(range(r), k - 1))
    n_src, n_tgt = len(src) * ci, len(tgt) * co
    maps = seeded_residues(seed, TAG_MAPS, r * co * ci, p, 0).reshape(r, co, ci)
    diag = seeded_residues(seed, TAG_DIAG, n_src, p, 1)
    X = seeded_residues(seed, TAG_X, n_src * m, p, 0).reshape(n_src, m)
    Y = seeded_residues(seed, TAG_Y, n_src * nb, p, 0).reshape(n_src, nb)
    # The reference's explicit differential: rows target*n + beta, columns source*g + alpha.
    d = differential(maps, src, tgt, ci, co, p)
    assert d.shape == (n_tgt, n_src)
    dt = d.T.tocsr()
    seq = np.zeros((nlen, m, nb), dtype=np.int64)
    cur = Y.copy()
    seq[0] = (X.T @ cur) % p
    first_apply = None
    for i in range(1, nlen):
        z = (d @ cur) % p
        w = (dt @ z) % p
        cur = (diag[:, None] * w) % p
        if first_apply is None:
            first_apply = cur.copy()
            first_forward = z.copy()
        seq[i] = (X.T @ cur) % p
    out = {
        f"{name}/shape": np.array([r, k, ci, co, p, nb, m, nlen, seed], dtype=np.int64),
        f"{name}/maps_head": maps.reshape(-1)[:16].astype(np.uint32),
        f"{name}/diag_head": diag[:16].astype(np.uint32),
        f"{name}/x_head": X.reshape(-1)[:16].astype(np.uint32),
        f"{name}/y_head": Y.reshape(-1)[:16].astype(np.uint32),
        f"{name}/seq": seq.astype(np.uint32),
        f"{name}/y_final_sha256": np.frombuffer(
            hashlib.sha256(cur.astype("<u4").tobytes()).digest(), dtype=np.uint8),
        f"{name}/d_nnz": np.array([d.nnz], dtype=np.int64),
    }
    if n_src * nb <= 4096:
        out[f"{name}/apply1"] = first_apply.astype(np.uint32)
        out[f"{name}/forward1"] = first_forward.astype(np.uint32)
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--reference", type=Path, required=True,
                    help="reference checkout (provides tests/deformation_reference.py)")
    ap.add_argument("--out", type=Path, default=Path(__file__).with_name("koszul_golden.npz"))
    args = ap.parse_args()
    sys.path.insert(0, str(args.reference / "tests"))
    from deformation_reference import differential  # the reference's explicit oracle
    arrays = {}
    for case in CASES:
        arrays.update(build(case, differential))
        print("built", case[0])
    np.savez_compressed(args.out, **arrays)
    print("wrote", args.out)


if __name__ == "__main__":
    main()
