"""Row-sampled oracle for large synthetic Koszul operators (test infrastructure).

``S Y`` at a few source subsets needs only their neighbourhoods:
    W[S] = D_S sum_{i in S} (-1)^pos(i,S) M_i^T Z[S \\ i],
    Z[T] = sum_{i' not in T} (-1)^pos(i',T u i') M_i' Y[T u i'],
so a full-size application (BASELINE configs 2 and 5) is checked exactly at
sampled rows without running the whole operator on the CPU.  Same conventions
as koszul_oracle.c (the reference's differential(),
tests/deformation_reference.py:75-89).
"""
from math import comb

import numpy as np


def lex_rank(s, r):
    k = len(s)
    return comb(r, k) - 1 - sum(comb(r - 1 - v, k - pos) for pos, v in enumerate(s))


def lex_unrank(rank, r, k):
    out, start = [], 0
    for pos in range(k):
        rem = k - pos - 1
        for v in range(start, r):
            c = comb(r - v - 1, rem)
            if rank < c:
                out.append(v)
                start = v + 1
                break
            rank -= c
    return tuple(out)


def needed_sources(sample_ranks, r, k):
    """All source subsets whose Y blocks the sampled outputs read."""
    need = set()
    for s_rank in sample_ranks:
        S = lex_unrank(s_rank, r, k)
        for i in S:
            T = tuple(v for v in S if v != i)
            for j in range(r):
                if j not in T:
                    need.add(lex_rank(tuple(sorted(T + (j,))), r))
    return sorted(need)


def apply_rows(r, k, ci, co, p, maps, diag_of, y_of, sample_ranks):
    """Blocks (S Y)[S] for the sampled source ranks.

    maps: (r, co, ci) int array; diag_of(S_rank) -> (ci,) residues;
    y_of(S_rank) -> (ci, nb) residues.  Returns {S_rank: (ci, nb) uint32}.
    """
    maps = np.asarray(maps, dtype=np.int64).reshape(r, co, ci)
    out = {}
    zcache = {}
    for s_rank in sample_ranks:
        S = lex_unrank(s_rank, r, k)
        acc = None
        for pos, i in enumerate(S):
            T = tuple(v for v in S if v != i)
            if T not in zcache:
                z = None
                for j in range(r):
                    if j in T:
                        continue
                    Sj = tuple(sorted(T + (j,)))
                    sgn = -1 if Sj.index(j) % 2 else 1
                    term = sgn * (maps[j] @ np.asarray(y_of(lex_rank(Sj, r)), dtype=np.int64))
                    z = term if z is None else z + term
                zcache[T] = z % p
            sgn = -1 if pos % 2 else 1
            term = sgn * (maps[i].T @ zcache[T])
            acc = term if acc is None else acc + term
        d = np.asarray(diag_of(s_rank), dtype=np.int64)[:, None]
        out[s_rank] = ((acc % p) * d % p).astype(np.uint32)
    return out
