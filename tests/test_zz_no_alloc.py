"""The allocation-free projection entry point (bw_project_noalloc).

Some callers cannot allocate device memory (their allocator owns all of HBM,
or they must not trigger cudaMalloc's device-wide synchronisation); this entry
point keeps its cross-CTA scratch in a fixed array inside the library.  Its
result must equal the projection the engine computes with scratch it
allocates itself (the first moment a_0 = X^T Y written by
bw_koszul_seq_start), on two calls in a row, since every call shares and
reuses the same array.

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import oracle
from prym_green_ancillary_b200 import KoszulEngine, seeded_fill_device, seeded_fill_host
from prym_green_ancillary_b200 import TAG_DIAG, TAG_MAPS, TAG_X, TAG_Y
from prym_green_ancillary_b200.engine import EngineError, _check, load

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _noalloc(x, w, p, out):
    rows, m = x.shape
    n = w.shape[1]
    _check(load().bw_project_noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(w.data_ptr()), rows, m, n, p,
                                     ctypes.c_void_p(out.data_ptr()), 0, None))


@pytest.mark.parametrize("dims", [
    # r, k, dim_in, dim_out, p, n, m
    (19, 9, 20, 28, 32003, 16, 16),   # BASELINE config 2 (1,847,560 rows)
    (8, 3, 6, 5, 32003, 8, 32),
    (6, 3, 3, 4, 101, 4, 4),
])
def test_noalloc_projection_matches_engine_projection(dims):
    r, k, ci, co, p, n, m = dims
    shape = oracle.KoszulShape(r, k, ci, co, p, n, m)
    dev = torch.device("cuda", 0)
    maps = seeded_fill_host(r * co * ci, 31, TAG_MAPS, p)
    diag = torch.empty(shape.n_src, dtype=torch.int32, device=dev)
    x = torch.empty((shape.n_src, m), dtype=torch.int32, device=dev)
    y = torch.empty((shape.n_src, n), dtype=torch.int32, device=dev)
    seeded_fill_device(diag, 31, TAG_DIAG, p, 1)
    seeded_fill_device(x, 31, TAG_X, p)
    seeded_fill_device(y, 31, TAG_Y, p)
    with KoszulEngine(r, k, ci, co, p, n, m, maps=maps, diag=diag) as eng:
        seq = torch.zeros((1, m, n), dtype=torch.int32, device=dev)
        eng.seq_start(x, y, seq)
        eng.seq_finish()
        torch.cuda.synchronize()
        want = seq[0].cpu().numpy()
    for call in range(2):
        out = torch.full((m, n), -1, dtype=torch.int32, device=dev)
        _noalloc(x, y, p, out)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy(), want, err_msg=f"call {call}")


def test_noalloc_rejects_sizes_beyond_its_scratch():
    dev = torch.device("cuda", 0)
    x = torch.zeros((64, 64), dtype=torch.int32, device=dev)
    out = torch.zeros((64, 64), dtype=torch.int32, device=dev)
    with pytest.raises(EngineError, match="m and n must be 4, 8, 16 or 32"):
        _noalloc(x, x, 32003, out)
