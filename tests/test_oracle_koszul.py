"""The synthetic-Koszul CPU oracle against the golden fixtures.

The fixtures come from the reference's explicit ``differential()`` matrices
(tests/deformation_reference.py:75-89 of the reference), see
tests/golden/make_koszul_golden.py.
"""
import hashlib
from pathlib import Path

import numpy as np
import pytest

import oracle

GOLDEN = np.load(Path(__file__).parent / "golden" / "koszul_golden.npz")
CASES = sorted({k.split("/")[0] for k in GOLDEN.files})


def _case(name):
    r, k, ci, co, p, nb, m, nlen, seed = (int(v) for v in GOLDEN[f"{name}/shape"])
    return oracle.KoszulShape(r, k, ci, co, p, nb, m), nlen, seed


@pytest.mark.parametrize("name", CASES)
def test_seeded_streams_match_golden(name):
    shape, _, seed = _case(name)
    maps, diag, X, Y = oracle.seeded_problem(shape, seed)
    np.testing.assert_array_equal(maps[:16], GOLDEN[f"{name}/maps_head"])
    np.testing.assert_array_equal(diag[:16], GOLDEN[f"{name}/diag_head"])
    np.testing.assert_array_equal(X.reshape(-1)[:16], GOLDEN[f"{name}/x_head"])
    np.testing.assert_array_equal(Y.reshape(-1)[:16], GOLDEN[f"{name}/y_head"])
    assert diag.min() >= 1 and diag.max() < shape.p


@pytest.mark.parametrize("name", CASES)
def test_sequence_matches_explicit_matrices(name):
    shape, nlen, seed = _case(name)
    maps, diag, X, Y = oracle.seeded_problem(shape, seed)
    seq, yf = oracle.sequence(shape, maps, diag, X, Y, nlen)
    np.testing.assert_array_equal(seq, GOLDEN[f"{name}/seq"])
    digest = hashlib.sha256(yf.astype("<u4").tobytes()).digest()
    assert digest == GOLDEN[f"{name}/y_final_sha256"].tobytes()


@pytest.mark.parametrize("name", [n for n in CASES if f"{n}/apply1" in GOLDEN.files])
def test_single_applications(name):
    shape, _, seed = _case(name)
    maps, diag, X, Y = oracle.seeded_problem(shape, seed)
    np.testing.assert_array_equal(oracle.forward(shape, maps, Y), GOLDEN[f"{name}/forward1"])
    np.testing.assert_array_equal(oracle.apply(shape, maps, diag, Y), GOLDEN[f"{name}/apply1"])


def test_transpose_identity():
    """<d y, z> == <y, d^T z> on random blocks (size-independent property)."""
    shape = oracle.KoszulShape(9, 4, 5, 7, 32003, 4)
    rng = np.random.default_rng(3)
    maps = rng.integers(0, shape.p, shape.r * shape.co * shape.ci, dtype=np.uint32)
    y = rng.integers(0, shape.p, (shape.n_src, 4), dtype=np.uint32)
    z = rng.integers(0, shape.p, (shape.n_tgt, 4), dtype=np.uint32)
    dy = oracle.forward(shape, maps, y).astype(object)
    dtz = oracle.transpose(shape, maps, z).astype(object)
    left = int((dy * z.astype(object)).sum()) % shape.p
    right = int((y.astype(object) * dtz).sum()) % shape.p
    assert left == right
