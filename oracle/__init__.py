"""CPU oracle for the block-Wiedemann engine (test infrastructure only).

Loaded by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline and
reference arms, never by the product package.  ``load()`` builds the shared
library with ``make -C oracle`` when it is missing.
"""
import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_LIB = None

U32P = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")


def build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def load():
    global _LIB
    if _LIB is not None:
        return _LIB
    path = HERE / "_build" / "libkoszul_oracle.so"
    if not path.exists():
        build()
    lib = ctypes.CDLL(str(path))
    c_int, c_u32, c_u64, c_i64 = ctypes.c_int, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int64
    lib.orc_binom.restype = c_u64
    lib.orc_binom.argtypes = [c_int, c_int]
    lib.orc_seeded_residue.restype = c_u32
    lib.orc_seeded_residue.argtypes = [c_u64, c_u32, c_u64, c_u32, c_u32]
    lib.orc_fill_seeded.restype = None
    lib.orc_fill_seeded.argtypes = [c_u64, c_u32, c_u32, c_u32, U32P, c_u64]
    shape = [c_int, c_int, c_int, c_int, c_u32, c_int]
    lib.orc_koszul_forward.argtypes = shape + [U32P, U32P, U32P]
    lib.orc_koszul_transpose.argtypes = shape + [U32P, U32P, U32P]
    lib.orc_koszul_forward_range.argtypes = shape + [U32P, U32P, U32P, c_i64, c_i64]
    lib.orc_koszul_transpose_range.argtypes = shape + [U32P, U32P, U32P, c_i64, c_i64]
    lib.orc_koszul_apply.argtypes = shape + [U32P, U32P, U32P, U32P]
    lib.orc_project.argtypes = [c_i64, c_int, c_int, c_u32, U32P, U32P, U32P]
    lib.orc_koszul_sequence.argtypes = shape + [c_int, U32P, U32P, U32P, U32P, c_i64, U32P, U32P]
    lib.orc_num_threads.restype = c_int
    _LIB = lib
    return lib


TAG_MAPS, TAG_DIAG, TAG_X, TAG_Y = 1, 2, 3, 4


class KoszulShape:
    """Shape of a synthetic Koszul operator d: Lambda^k(F^r)(x)R_q -> Lambda^(k-1)(F^r)(x)R_(q+1)."""

    def __init__(self, r, k, dim_in, dim_out, prime, nb, m=None):
        self.r, self.k, self.ci, self.co, self.p, self.nb = r, k, dim_in, dim_out, prime, nb
        self.m = nb if m is None else m
        lib = load()
        self.n_src = lib.orc_binom(r, k) * dim_in
        self.n_tgt = lib.orc_binom(r, k - 1) * dim_out

    @property
    def args(self):
        return (self.r, self.k, self.ci, self.co, self.p, self.nb)


def seeded(seed, tag, count, p, lo=0):
    out = np.empty(count, dtype=np.uint32)
    load().orc_fill_seeded(seed, tag, p, lo, out, count)
    return out


def seeded_problem(shape, seed):
    """Maps, diagonal, X and Y of the seeded synthetic problem."""
    maps = seeded(seed, TAG_MAPS, shape.r * shape.co * shape.ci, shape.p)
    diag = seeded(seed, TAG_DIAG, shape.n_src, shape.p, 1)
    X = seeded(seed, TAG_X, shape.n_src * shape.m, shape.p).reshape(shape.n_src, shape.m)
    Y = seeded(seed, TAG_Y, shape.n_src * shape.nb, shape.p).reshape(shape.n_src, shape.nb)
    return maps, diag, X, Y


def forward(shape, maps, Y):
    Z = np.empty((shape.n_tgt, shape.nb), dtype=np.uint32)
    load().orc_koszul_forward(*shape.args, maps, np.ascontiguousarray(Y), Z)
    return Z


def transpose(shape, maps, Z):
    W = np.empty((shape.n_src, shape.nb), dtype=np.uint32)
    load().orc_koszul_transpose(*shape.args, maps, np.ascontiguousarray(Z), W)
    return W


def apply(shape, maps, diag, Y):
    out = np.empty((shape.n_src, shape.nb), dtype=np.uint32)
    load().orc_koszul_apply(*shape.args, maps, diag, np.ascontiguousarray(Y), out)
    return out


def project(p, X, Y):
    rows, m = X.shape
    nb = Y.shape[1]
    P = np.empty((m, nb), dtype=np.uint32)
    load().orc_project(rows, m, nb, p, np.ascontiguousarray(X), np.ascontiguousarray(Y), P)
    return P


def sequence(shape, maps, diag, X, Y0, nlen):
    seq = np.empty((nlen, shape.m, shape.nb), dtype=np.uint32)
    yf = np.empty((shape.n_src, shape.nb), dtype=np.uint32)
    load().orc_koszul_sequence(*shape.args, shape.m, maps, diag, np.ascontiguousarray(X),
                               np.ascontiguousarray(Y0), nlen, seq, yf)
    return seq, yf


def num_threads():
    return load().orc_num_threads()


def set_threads(n):
    os.environ["OMP_NUM_THREADS"] = str(n)
