"""Parity of the CUDA Koszul engine with the CPU oracle and the golden fixtures.

Bit-exact throughout (integer arithmetic mod p).  Small shapes are compared
with the full oracle; BASELINE-sized operators (config 2 and config 5) are
checked at sampled rows with the row oracle, and multi-step sequences through
the sequence session are checked against repeated applications plus an exact
int64 projection.
"""
import hashlib
from pathlib import Path

import numpy as np
import pytest

import oracle
from oracle import koszul_rows
from prym_green_ancillary_b200 import KoszulEngine, seeded_fill_device, seeded_fill_host
from prym_green_ancillary_b200 import TAG_DIAG, TAG_MAPS, TAG_X, TAG_Y

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

GOLDEN = np.load(Path(__file__).parent / "golden" / "koszul_golden.npz")
CASES = sorted({k.split("/")[0] for k in GOLDEN.files})
FORMS = ["plain", "int8"]
# The INT8 form's stage producers (the set-up autotuner picks one per shape;
# BW_I8_PRODUCER restricts the choice): cp.async warps alone (8 or 16 of them,
# BW_I8_PRODUCER_WARPS), or TMA gathers beside them.  The plain form's two
# tile heights (4 or 8 output rows a thread; timed at set-up, BW_PLAIN_TILE
# forces one).
PRODUCER_FORMS = ["plain:tile4", "plain:tile8", "int8:cpasync8", "int8:cpasync16", "int8:hybrid"]


@pytest.fixture
def producer_form(request, monkeypatch):
    form, _, producer = request.param.partition(":")
    for var in ("BW_I8_PRODUCER", "BW_I8_PRODUCER_WARPS", "BW_PLAIN_TILE"):
        monkeypatch.delenv(var, raising=False)
    if form == "int8":
        if producer.startswith("cpasync"):
            monkeypatch.setenv("BW_I8_PRODUCER", "cpasync")
            monkeypatch.setenv("BW_I8_PRODUCER_WARPS", producer[len("cpasync"):])
        else:
            monkeypatch.setenv("BW_I8_PRODUCER", producer)
    else:
        monkeypatch.setenv("BW_PLAIN_TILE", producer[len("tile"):])
    return form, producer


def _supported(form, nb):
    """Both forms take every block width of the ABI (4, 8, 16, 32); the INT8-limb
    form runs widths 4 and 8 as 16 with zero columns."""
    assert nb in (4, 8, 16, 32)


def _golden_case(name):
    r, k, ci, co, p, nb, m, nlen, seed = (int(v) for v in GOLDEN[f"{name}/shape"])
    return oracle.KoszulShape(r, k, ci, co, p, nb, m), nlen, seed


def _engine(shape, maps, diag, form):
    return KoszulEngine(shape.r, shape.k, shape.ci, shape.co, shape.p, shape.nb, shape.m,
                        maps=maps, diag=diag, form=form)


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("name", CASES)
def test_sequence_matches_golden(name, form):
    shape, nlen, seed = _golden_case(name)
    _supported(form, shape.nb)
    maps, diag, X, Y = oracle.seeded_problem(shape, seed)
    with _engine(shape, maps, diag, form) as eng:
        seq, yf = eng.sequence_host(X, Y, nlen)
    np.testing.assert_array_equal(seq, GOLDEN[f"{name}/seq"])
    assert hashlib.sha256(yf.astype("<u4").tobytes()).digest() == GOLDEN[f"{name}/y_final_sha256"].tobytes()


SHAPES = [
    # r, k, ci, co, p, nb, m
    (6, 3, 3, 4, 101, 4, 4),
    (7, 1, 5, 3, 32003, 8, 4),      # k = 1: the target space is Lambda^0 (one empty subset)
    (6, 6, 4, 5, 32003, 4, 8),      # k = r: one source subset
    (8, 4, 5, 7, 32003, 16, 16),    # ragged dims (not multiples of 4)
    (9, 4, 20, 28, 32003, 16, 16),  # config-2 map sizes, fewer generators
    (7, 3, 32, 40, 32749, 32, 32),  # config-5 map sizes, largest 15-bit prime
    (10, 5, 1, 1, 3, 8, 8),         # smallest dims and prime
]


@pytest.mark.parametrize("producer_form", PRODUCER_FORMS, indirect=True)
@pytest.mark.parametrize("dims", SHAPES)
def test_operators_match_oracle(dims, producer_form):
    form, producer = producer_form
    shape = oracle.KoszulShape(*dims)
    _supported(form, shape.nb)
    maps, diag, X, Y = oracle.seeded_problem(shape, 99)
    rng = np.random.default_rng(5)
    Z = rng.integers(0, shape.p, (shape.n_tgt, shape.nb), dtype=np.uint32)
    dev = torch.device("cuda", 0)
    with _engine(shape, maps, diag, form) as eng:
        if form == "int8":
            assert ("hybrid" in eng.plan) == (producer == "hybrid"), eng.plan
            if producer.startswith("cpasync"):
                assert "%s producer warps" % producer[len("cpasync"):] in eng.plan, eng.plan
        else:
            assert eng.plan.startswith("plain: %s output rows" % producer[len("tile"):]), eng.plan
        y = torch.from_numpy(Y.view(np.int32)).to(dev)
        z = torch.from_numpy(Z.view(np.int32)).to(dev)
        out_z = torch.empty((shape.n_tgt, shape.nb), dtype=torch.int32, device=dev)
        out_w = torch.empty((shape.n_src, shape.nb), dtype=torch.int32, device=dev)
        out_s = torch.empty_like(out_w)
        eng.forward(y, out_z)
        eng.transpose(z, out_w, scale_by_diag=False)
        eng.apply(y, out_s)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out_z.cpu().numpy().view(np.uint32), oracle.forward(shape, maps, Y))
        np.testing.assert_array_equal(out_w.cpu().numpy().view(np.uint32), oracle.transpose(shape, maps, Z))
        np.testing.assert_array_equal(out_s.cpu().numpy().view(np.uint32), oracle.apply(shape, maps, diag, Y))
        eng.transpose(z, out_w, scale_by_diag=True)
        torch.cuda.synchronize()
        tz = oracle.transpose(shape, maps, Z).astype(np.uint64)
        np.testing.assert_array_equal(out_w.cpu().numpy().view(np.uint32),
                                      (tz * diag[:, None] % shape.p).astype(np.uint32))


def test_device_seeded_fill_matches_host():
    dev = torch.device("cuda", 0)
    for tag, lo, n in ((TAG_MAPS, 0, 1000), (TAG_DIAG, 1, 4097), (TAG_Y, 0, 1 << 20)):
        t = torch.empty(n, dtype=torch.int32, device=dev)
        seeded_fill_device(t, 77, tag, 32003, lo)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(t.cpu().numpy().view(np.uint32), seeded_fill_host(n, 77, tag, 32003, lo))


def _device_problem(shape, seed, dev):
    maps = seeded_fill_host(shape.r * shape.co * shape.ci, seed, TAG_MAPS, shape.p)
    diag = torch.empty(shape.n_src, dtype=torch.int32, device=dev)
    x = torch.empty((shape.n_src, shape.m), dtype=torch.int32, device=dev)
    y = torch.empty((shape.n_src, shape.nb), dtype=torch.int32, device=dev)
    seeded_fill_device(diag, seed, TAG_DIAG, shape.p, 1)
    seeded_fill_device(x, seed, TAG_X, shape.p)
    seeded_fill_device(y, seed, TAG_Y, shape.p)
    return maps, diag, x, y


def _check_sampled_rows(shape, maps, diag, y, out, count, seed):
    rng = np.random.default_rng(seed)
    n_s = shape.n_src // shape.ci
    sample = sorted(set(int(v) for v in rng.integers(0, n_s, count)) | {0, n_s - 1})
    need = koszul_rows.needed_sources(sample, shape.r, shape.k)
    idx = torch.tensor(need, dtype=torch.long, device=y.device)
    yb = y.view(n_s, shape.ci, shape.nb).index_select(0, idx).cpu().numpy().view(np.uint32)
    where = {s: j for j, s in enumerate(need)}
    sidx = torch.tensor(sample, dtype=torch.long, device=y.device)
    db = diag.view(n_s, shape.ci).index_select(0, sidx).cpu().numpy().view(np.uint32)
    dwhere = {s: j for j, s in enumerate(sample)}
    got = out.view(n_s, shape.ci, shape.nb).index_select(0, sidx).cpu().numpy().view(np.uint32)
    want = koszul_rows.apply_rows(shape.r, shape.k, shape.ci, shape.co, shape.p,
                                  maps.reshape(shape.r, shape.co, shape.ci),
                                  lambda s: db[dwhere[s]], lambda s: yb[where[s]], sample)
    for j, s in enumerate(sample):
        np.testing.assert_array_equal(got[j], want[s], err_msg=f"source subset {s}")


def _projection(x, w, p):
    """Exact X^T W mod p on the GPU in float64: residues are below 2^15, so a
    product is below 2^30 and a chunk of 2^21 rows sums below 2^51 < 2^53."""
    acc = torch.zeros((x.shape[1], w.shape[1]), dtype=torch.float64, device=x.device)
    for s in range(0, x.shape[0], 1 << 21):
        part = x[s:s + (1 << 21)].to(torch.float64).T @ w[s:s + (1 << 21)].to(torch.float64)
        acc = torch.remainder(acc + torch.remainder(part, p), p)
    return acc.to(torch.int64).cpu().numpy().astype(np.uint32)


@pytest.mark.parametrize("producer_form", PRODUCER_FORMS, indirect=True)
@pytest.mark.parametrize("cfg", [
    # r = 19, k = 9, dim 20 -> 28, p = 32003, block 16 x 16 (N = 1,847,560)
    ("config2", 19, 9, 20, 28, 32003, 16, 16, 3),
    # r = 23, k = 11, dim 32 -> 40, block 32 x 32 (N = 43,266,496)
    ("config5", 23, 11, 32, 40, 32003, 32, 32, 1),
])
def test_full_size_apply_and_session(cfg, producer_form):
    form, producer = producer_form
    name, r, k, ci, co, p, nb, m, steps = cfg
    shape = oracle.KoszulShape(r, k, ci, co, p, nb, m)
    dev = torch.device("cuda", 0)
    maps, diag, x, y = _device_problem(shape, 2024, dev)
    with _engine(shape, maps, diag, form) as eng:
        out = torch.empty_like(y)
        eng.apply(y, out)
        torch.cuda.synchronize()
        _check_sampled_rows(shape, maps, diag, y, out, 48, 1)
        # sequence session == repeated applications + exact projection
        seq = torch.zeros((steps + 1, m, nb), dtype=torch.int32, device=dev)
        eng.seq_start(x, y, seq)
        eng.seq_step(steps)
        y_end = torch.empty_like(y)
        assert eng.seq_finish(y_end) == steps + 1
        torch.cuda.synchronize()
        cur = y.clone()
        want = [_projection(x, cur, p)]
        for _ in range(steps):
            nxt = torch.empty_like(cur)
            eng.apply(cur, nxt)
            cur = nxt
            want.append(_projection(x, cur, p))
        torch.cuda.synchronize()
        np.testing.assert_array_equal(seq.cpu().numpy().view(np.uint32), np.stack(want))
        assert torch.equal(y_end, cur)


@pytest.mark.parametrize("form", FORMS)
def test_session_graph_path_matches_direct(form):
    """Long sessions use captured graphs of 16 steps; compare with a direct run."""
    shape = oracle.KoszulShape(8, 3, 6, 5, 32003, 16, 16)
    maps, diag, X, Y = oracle.seeded_problem(shape, 3)
    nlen = 41   # 40 steps: two graph replays of 16 plus 8 direct steps
    want, yf_want = oracle.sequence(shape, maps, diag, X, Y, nlen)
    with _engine(shape, maps, diag, form) as eng:
        seq, yf = eng.sequence_host(X, Y, nlen)
        np.testing.assert_array_equal(seq, want)
        np.testing.assert_array_equal(yf, yf_want)
        # a second session on the same context (graphs are rebuilt)
        seq2, _ = eng.sequence_host(X, Y, nlen)
        np.testing.assert_array_equal(seq2, want)


@pytest.mark.parametrize("form", FORMS)
def test_contexts_of_different_shapes_coexist(form):
    """Per-kernel launch limits are process-wide: a context created after a
    larger one must not break the larger one's launches."""
    big = oracle.KoszulShape(6, 3, 40, 48, 32003, 32, 32)
    small = oracle.KoszulShape(7, 3, 5, 6, 32003, 16, 16)
    dev = torch.device("cuda", 0)
    engines = []
    for shape in (big, small):
        maps, diag, X, Y = oracle.seeded_problem(shape, 21)
        engines.append((shape, maps, diag, Y, _engine(shape, maps, diag, form)))
    try:
        for shape, maps, diag, Y, eng in engines:   # the large context runs after the small one was created
            y = torch.from_numpy(Y.view(np.int32)).to(dev)
            out = torch.empty_like(y)
            eng.apply(y, out)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), oracle.apply(shape, maps, diag, Y))
    finally:
        for *_, eng in engines:
            eng.close()


def test_int8_form_refuses_dims_beyond_its_accumulators():
    """The INT8 form keeps two double-buffered accumulators of 2 N TMEM columns
    (N = 2 x dim rounded up to 16): dims above 64 would need more than the 512
    columns an SM has, so such contexts are refused with status 3."""
    from prym_green_ancillary_b200 import EngineError
    shape = oracle.KoszulShape(3, 2, 65, 4, 32003, 16, 16)
    maps, diag, X, Y = oracle.seeded_problem(shape, 5)
    with pytest.raises(EngineError) as err:
        _engine(shape, maps, diag, "int8")
    assert err.value.status == 3 and "at most 64" in str(err.value)
