"""The batched workload's own sector shapes (24 sectors, r in {19, 20, 21},
k in {8, 9, 10}, dim R_q in 12..40, block widths 8/16/32, p = 32003), each
with the seeded maps, diagonal, X and Y the bench draws for it.

* One batched step: every sector's S Y0 equals the row oracle at sampled
  source subsets, and its first two moments X^T Y0, X^T S Y0 equal an exact
  projection.
* Seventeen batched steps (one captured graph of 16 plus one direct step):
  every sector's sequence and final block equal those of the sector run alone.

Bit-exact throughout.
"""
import numpy as np
import pytest

from bench import config3_sectors
from oracle import koszul_rows
from prym_green_ancillary_b200 import (KoszulBatch, KoszulEngine, seeded_fill_device, seeded_fill_host, TAG_DIAG,
                                       TAG_MAPS, TAG_X, TAG_Y)

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _projection(x, w, p):
    """Exact X^T W mod p in float64 (products below 2^30, chunks of 2^21 rows below 2^53)."""
    acc = torch.zeros((x.shape[1], w.shape[1]), dtype=torch.float64, device=x.device)
    for s in range(0, x.shape[0], 1 << 21):
        part = x[s:s + (1 << 21)].to(torch.float64).T @ w[s:s + (1 << 21)].to(torch.float64)
        acc = torch.remainder(acc + torch.remainder(part, p), p)
    return acc.to(torch.int64).cpu().numpy().astype(np.uint32)


def _problem(sec, dev):
    seed = sec["seed"]
    maps = seeded_fill_host(sec["r"] * sec["co"] * sec["ci"], seed, TAG_MAPS, sec["p"])
    diag = torch.empty(sec["n_src"], dtype=torch.int32, device=dev)
    x = torch.empty((sec["n_src"], sec["m"]), dtype=torch.int32, device=dev)
    y = torch.empty((sec["n_src"], sec["n"]), dtype=torch.int32, device=dev)
    seeded_fill_device(diag, seed, TAG_DIAG, sec["p"], 1)
    seeded_fill_device(x, seed, TAG_X, sec["p"])
    seeded_fill_device(y, seed, TAG_Y, sec["p"])
    return maps, diag, x, y


def _spec(sec, maps, diag, form):
    return dict(r=sec["r"], k=sec["k"], dim_in=sec["ci"], dim_out=sec["co"], prime=sec["p"], block_width=sec["n"],
                proj_width=sec["m"], maps=maps, diag=diag, form=form)


def _check_rows(sec, maps, diag, y, out, count, seed):
    r, k, ci, co, p, nb = sec["r"], sec["k"], sec["ci"], sec["co"], sec["p"], sec["n"]
    n_s = sec["n_src"] // ci
    rng = np.random.default_rng(seed)
    sample = sorted(set(int(v) for v in rng.integers(0, n_s, count)) | {0, n_s - 1})
    need = koszul_rows.needed_sources(sample, r, k)
    yb = y.view(n_s, ci, nb).index_select(0, torch.tensor(need, device=y.device)).cpu().numpy().view(np.uint32)
    sidx = torch.tensor(sample, device=y.device)
    db = diag.view(n_s, ci).index_select(0, sidx).cpu().numpy().view(np.uint32)
    got = out.view(n_s, ci, nb).index_select(0, sidx).cpu().numpy().view(np.uint32)
    where = {s: j for j, s in enumerate(need)}
    dwhere = {s: j for j, s in enumerate(sample)}
    want = koszul_rows.apply_rows(r, k, ci, co, p, maps.reshape(r, co, ci), lambda s: db[dwhere[s]],
                                  lambda s: yb[where[s]], sample)
    for j, s in enumerate(sample):
        np.testing.assert_array_equal(got[j], want[s], err_msg=f"source subset {s}")


def test_config3_shapes_one_batched_step_and_graph_session():
    dev = torch.device("cuda", 0)
    secs = config3_sectors()
    assert len(secs) == 24
    problems = [_problem(sec, dev) for sec in secs]
    steps = 17
    specs = [_spec(sec, maps, diag, "int8") for sec, (maps, diag, _, _) in zip(secs, problems)]
    with KoszulBatch(specs) as batch:
        xs = [pr[2] for pr in problems]
        ys = [pr[3] for pr in problems]
        # one batched step
        seqs = [torch.zeros((2, s["m"], s["n"]), dtype=torch.int32, device=dev) for s in secs]
        finals = [torch.empty_like(y) for y in ys]
        batch.seq_start(xs, ys, seqs)
        batch.seq_step(1)
        assert batch.seq_finish(finals) == 2
        torch.cuda.synchronize()
        for i, (sec, (maps, diag, x, y)) in enumerate(zip(secs, problems)):
            shape = (sec["r"], sec["k"], sec["ci"], sec["co"], sec["n"])
            _check_rows(sec, maps, diag, y, finals[i], 12, 100 + i)
            got = seqs[i].cpu().numpy().view(np.uint32)
            np.testing.assert_array_equal(got[0], _projection(x, y, sec["p"]), err_msg=f"sector {i} {shape} a_0")
            np.testing.assert_array_equal(got[1], _projection(x, finals[i], sec["p"]),
                                          err_msg=f"sector {i} {shape} a_1")
        # a 17-step session: one 16-step graph of the whole batch plus one direct step
        seqs = [torch.zeros((steps + 1, s["m"], s["n"]), dtype=torch.int32, device=dev) for s in secs]
        finals = [torch.empty_like(y) for y in ys]
        batch.seq_start(xs, ys, seqs)
        batch.seq_step(steps)
        assert batch.seq_finish(finals) == steps + 1
        torch.cuda.synchronize()
        batch_seqs = [s.cpu().numpy() for s in seqs]
        batch_finals = finals
    for i, (sec, (maps, diag, x, y)) in enumerate(zip(secs, problems)):
        with KoszulEngine(sec["r"], sec["k"], sec["ci"], sec["co"], sec["p"], sec["n"], sec["m"], maps=maps,
                          diag=diag, form="int8") as eng:
            seq = torch.zeros((steps + 1, sec["m"], sec["n"]), dtype=torch.int32, device=dev)
            fin = torch.empty_like(y)
            eng.seq_start(x, y, seq)
            eng.seq_step(steps)
            eng.seq_finish(fin)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(batch_seqs[i], seq.cpu().numpy(), err_msg=f"sector {i} sequence")
            assert torch.equal(batch_finals[i], fin), f"sector {i} final block"
