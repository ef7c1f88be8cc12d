"""Helpers shared by the paper-mode GPU tests: explicit S from the engine, a
minimal-polynomial generator for kernel recovery, and deformation input files."""
import json

import numpy as np

from prym_green_ancillary_b200.engine import APPLY_SQUARE


def square_matrix(eng, p):
    """Explicit S (cols x cols) from the engine's square applied to unit vectors."""
    n = eng.info["cols"]
    cols = []
    for c0 in range(0, n, 4):
        block = np.zeros((n, 4), dtype=np.uint32)
        for j in range(4):
            if c0 + j < n:
                block[c0 + j, j] = 1
        out = eng.apply(APPLY_SQUARE, block).astype(np.int64)
        for j in range(4):
            if c0 + j < n:
                cols.append(out[:, j])
    return np.stack(cols, axis=1) % p


def minimal_polynomial(S, p, seed=3):
    """Monic minimal polynomial of a random vector under S (exact, Python ints)."""
    n = S.shape[0]
    v = np.random.default_rng(seed).integers(0, p, n).astype(object)
    krylov = [v]
    Sobj = S.astype(object)
    basis, pivots = [], []   # reduced echelon rows with combination coefficients
    for d in range(n + 1):
        w = krylov[-1]
        comb = [0] * (d + 1)
        comb[d] = 1
        w = list(w)
        for (row, rcomb), pc in zip(basis, pivots):
            f = w[pc] % p
            if f:
                w = [(a - f * b) % p for a, b in zip(w, row)]
                for i, c in enumerate(rcomb):
                    comb[i] = (comb[i] - f * c) % p
        nz = next((i for i, a in enumerate(w) if a % p), None)
        if nz is None:
            return [c % p for c in comb]    # sum comb[i] S^i v = 0, comb[d] = 1
        inv = pow(int(w[nz]), -1, p)
        basis.append(([a * inv % p for a in w], [c * inv % p for c in comb]))
        pivots.append(nz)
        krylov.append(np.array([int(x) for x in Sobj.dot(np.array(krylov[-1], dtype=object)) % p], dtype=object))
    raise AssertionError("no minimal polynomial found")


def kernel_generator(S, p):
    """x^(e-1) q(x) for mu(x) = x^e q(x): D = S^(e-1) q(S) V lies in ker S (mu itself when S is invertible)."""
    mu = minimal_polynomial(S, p)
    e = next(i for i, c in enumerate(mu) if c)
    return [0] * (e - 1) + mu[e:] if e >= 1 else mu


def write_generator(path, coeffs, p):
    """One 4 x 4 scalar matrix per line, some entries written as negative representatives."""
    with open(path, "w") as f:
        for c in coeffs:
            m = np.zeros((4, 4), dtype=np.int64)
            np.fill_diagonal(m, c % p)
            row = [int(x) if (i % 5) else int(x) - p if x else 0 for i, x in enumerate(m.reshape(-1))]
            f.write(" ".join(str(x) for x in row) + "\n")


def write_dense_block(path, rows, p, seed, nested=True):
    """A seeded rows x 2 dense block JSON (values as nested rows, as the pipeline writes matrices)."""
    vals = np.random.default_rng(seed).integers(0, p, (rows, 2))
    values = vals.tolist() if nested else vals.reshape(-1).tolist()
    with open(path, "w") as f:
        json.dump({"format": "dense-block", "rows": int(rows), "columns": 2, "prime": int(p), "values": values}, f)
    return vals


def write_drop_columns(path, indices):
    with open(path, "w") as f:
        json.dump({"indices": [int(i) for i in indices]}, f)
