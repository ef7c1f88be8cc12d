"""The allocation-free projection entry point (bw_project_noalloc).

Some callers cannot allocate device memory (their allocator owns all of HBM,
or they must not trigger cudaMalloc's device-wide synchronisation); this entry
point keeps its cross-CTA scratch in a fixed array inside the library.  Its
result must equal the projection the engine computes with scratch it
allocates itself (the first moment a_0 = X^T Y written by
bw_koszul_seq_start), on two calls in a row, since every call shares and
reuses the same array.

The result is also checked against an exact float64 projection, the second
call is checked to allocate no device memory, and sizes beyond the fixed
scratch are rejected with status 1.

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
    np.testing.assert_array_equal(want, _exact_projection(x, y, p))
    outs = [torch.full((m, n), -1, dtype=torch.int32, device=dev) for _ in range(2)]
    torch.cuda.synchronize()
    for call in range(2):
        if call == 1:
            free_before = torch.cuda.mem_get_info(dev)[0]
        _noalloc(x, y, p, outs[call])
        torch.cuda.synchronize()
        if call == 1:   # the second call allocates nothing on the device
            assert torch.cuda.mem_get_info(dev)[0] == free_before
        np.testing.assert_array_equal(outs[call].cpu().numpy(), want, err_msg=f"call {call}")


def _exact_projection(x, w, p):
    """X^T W mod p in float64 on the GPU: residues below 2^15, products below
    2^30, chunks of 2^21 rows sum below 2^53, so every partial sum is exact."""
    acc = torch.zeros((x.shape[1], w.shape[1]), dtype=torch.float64, device=x.device)
    for s in range(0, x.shape[0], 1 << 21):
        part = x[s:s + (1 << 21)].to(torch.float64).T @ w[s:s + (1 << 21)].to(torch.float64)
        acc = torch.remainder(acc + torch.remainder(part, p), p)
    return acc.to(torch.int64).cpu().numpy().astype(np.int32)


@pytest.mark.parametrize("case", ["width", "even prime", "prime too large", "misaligned W"])
def test_noalloc_rejects_arguments_beyond_its_limits(case):
    dev = torch.device("cuda", 0)
    x = torch.zeros((64, 64), dtype=torch.int32, device=dev)
    w = torch.zeros((65, 16), dtype=torch.int32, device=dev)
    out = torch.zeros((64, 64), dtype=torch.int32, device=dev)
    args = {"width": (x, x, 32003, "m and n must be 4, 8, 16 or 32"),
            "even prime": (x[:, :16], w[:64], 32002, "prime must be odd"),
            "prime too large": (x[:, :16], w[:64], 32771, "below 2\\^15"),
            "misaligned W": (x[:, :16], w.view(-1)[1:1 + 64 * 16].view(64, 16), 32003, "16-byte aligned")}[case]
    with pytest.raises(EngineError, match=args[3]) as err:
        _noalloc(args[0], args[1], args[2], out)
    assert err.value.status == 1
