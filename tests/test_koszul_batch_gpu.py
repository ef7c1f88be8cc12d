"""Batched sectors (bw_koszul_batch_*): sectors of uneven shapes, block widths
and forms advance together; every sector's sequence and final block equal the
oracle's for that sector alone.  Bit-exact."""
import numpy as np
import pytest

import oracle
from prym_green_ancillary_b200 import KoszulBatch

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SECTORS = [
    # r, k, dim_in, dim_out, p, nb, m, form, seed
    (7, 3, 5, 6, 32003, 8, 8, "int8", 11),
    (8, 4, 6, 7, 32003, 16, 16, "int8", 12),
    (6, 2, 4, 5, 32003, 32, 32, "int8", 13),
    (7, 4, 3, 9, 32749, 4, 8, "int8", 14),
    (8, 3, 6, 5, 32003, 16, 16, "plain", 15),
    (5, 5, 2, 3, 101, 8, 4, "plain", 16),    # k = r: one source subset
]


def _problems():
    out = []
    for r, k, ci, co, p, nb, m, form, seed in SECTORS:
        shape = oracle.KoszulShape(r, k, ci, co, p, nb, m)
        maps, diag, X, Y = oracle.seeded_problem(shape, seed)
        out.append((shape, form, maps, diag, X, Y))
    return out


def _run_batch(batch, problems, nlen, dev):
    xs = [torch.from_numpy(X.view(np.int32)).to(dev) for _, _, _, _, X, _ in problems]
    ys = [torch.from_numpy(Y.view(np.int32)).to(dev) for _, _, _, _, _, Y in problems]
    seqs = [torch.zeros((nlen, sh.m, sh.nb), dtype=torch.int32, device=dev) for sh, *_ in problems]
    finals = [torch.empty_like(y) for y in ys]
    batch.seq_start(xs, ys, seqs)
    batch.seq_step(nlen - 1)
    assert batch.seq_finish(finals) == nlen
    torch.cuda.synchronize()
    return ([s.cpu().numpy().view(np.uint32) for s in seqs], [f.cpu().numpy().view(np.uint32) for f in finals])


def test_batch_matches_each_sector_alone():
    dev = torch.device("cuda", 0)
    problems = _problems()
    nlen = 41   # 40 steps: two graphs of 16 batch steps plus 8 direct steps
    sectors = [dict(r=sh.r, k=sh.k, dim_in=sh.ci, dim_out=sh.co, prime=sh.p, block_width=sh.nb, proj_width=sh.m,
                    maps=maps, diag=diag, form=form) for sh, form, maps, diag, _, _ in problems]
    with KoszulBatch(sectors) as batch:
        assert [e.n_src for e in batch.engines] == [sh.n_src for sh, *_ in problems]
        for attempt in range(2):   # a second session on the same batch rebuilds its graphs
            seqs, finals = _run_batch(batch, problems, nlen, dev)
            for i, (sh, form, maps, diag, X, Y) in enumerate(problems):
                want, yf = oracle.sequence(sh, maps, diag, X, Y, nlen)
                np.testing.assert_array_equal(seqs[i], want, err_msg=f"sector {i} ({form}), session {attempt}")
                np.testing.assert_array_equal(finals[i], yf, err_msg=f"sector {i} final block")
        assert batch.launch_count > 0


def test_batch_refuses_bad_sector():
    from prym_green_ancillary_b200 import EngineError
    sh, form, maps, diag, _, _ = _problems()[0]
    good = dict(r=sh.r, k=sh.k, dim_in=sh.ci, dim_out=sh.co, prime=sh.p, block_width=sh.nb, maps=maps, diag=diag)
    bad = dict(good, block_width=12)
    with pytest.raises(EngineError, match="sector 1"):
        KoszulBatch([good, bad])
