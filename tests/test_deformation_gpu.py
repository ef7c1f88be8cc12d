"""Deformation variants of the eliminated operator on the GPU.

* augmented   F = [F0 | -b]: the base sector's columns plus two dense columns;
* replacement F = F0 without two base columns, plus the two dense columns
  (cuda/cuprym_deformation.cu:2554-3066 of the reference).

F and F^t equal the explicit matrices built from the reference's exact g12
blocks (tests/golden/cyclic_g12_golden.npz).  bin/cuprym_deformation and the
reference's cuprym_deformation (built from its sources by oracle/build_ref.sh)
write the same decompressed WDM text and sidecar, and
bin/cuprym_deformation_kernel_vectors recovers the same candidates as the
reference's recovery program.  Refusals match the reference binary's.
"""
import json
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from paper_helpers import kernel_generator, square_matrix, write_dense_block, write_drop_columns, write_generator
from prym_green_ancillary_b200 import CyclicEngine, read_text
from prym_green_ancillary_b200.engine import APPLY_FORWARD, APPLY_TRANSPOSE

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
G = np.load(GOLDEN / "cyclic_g12_golden.npz")
BIN = ROOT / "prym_green_ancillary_b200" / "bin"
REF = ROOT / "oracle" / "_ref" / "bin"
REF_DATA = ROOT / "oracle" / "_ref" / "data"
RECIPE = ["-v", "4", "--seed", "1", "--rowmix-rounds", "2", "--rowmix-seed", "10001"]


def _inputs(tmp_path, instance, sector, op, seed):
    """Dense block (and drop columns for replacement) sized for this sector."""
    with CyclicEngine(instance, sector, device=-1) as host:
        rows, base = host.info["rows"], host.info["cols"]
        p = host.info["prime"]
    dense_path = tmp_path / f"dense_{op}_{sector}.json"
    dense = write_dense_block(dense_path, rows, p, seed)
    drop_path, drop = None, None
    if op == "replacement":
        rng = np.random.default_rng(seed + 1)
        drop = sorted(int(v) for v in rng.choice(base, 2, replace=False))
        drop_path = tmp_path / f"drop_{sector}.json"
        write_drop_columns(drop_path, drop[::-1])   # unsorted on disk: the loader sorts
    return p, rows, base, dense, dense_path, drop, drop_path


def _explicit(F0, dense, op, drop, p):
    if op == "augmented":
        return np.concatenate([F0, -dense], axis=1) % p
    keep = [c for c in range(F0.shape[1]) if c not in drop]
    return np.concatenate([F0[:, keep], dense], axis=1) % p


@pytest.mark.parametrize("generic", [False, True], ids=["subset", "generic"])
@pytest.mark.parametrize("op", ["augmented", "replacement"])
@pytest.mark.parametrize("p, sector", [(661, 0), (661, 1), (661, 4), (109, 0), (109, 2)])
def test_operator_matches_explicit_matrix(op, p, sector, generic, tmp_path, monkeypatch):
    if generic:
        monkeypatch.setenv("BW_CYCLIC_GENERIC", "1")
    else:
        monkeypatch.delenv("BW_CYCLIC_GENERIC", raising=False)
    inst = GOLDEN / f"g12_p{p}.json"
    _, rows, base, dense, dense_path, drop, drop_path = _inputs(tmp_path, inst, sector, op, 10 * sector + p)
    F0 = G[f"p{p}/sector{sector}/F"].astype(np.int64)
    assert F0.shape == (rows, base)
    F = _explicit(F0, dense.astype(np.int64), op, drop, p)
    rng = np.random.default_rng(sector + 7)
    with CyclicEngine(inst, sector, op=op, dense_file=dense_path, drop_columns=drop_path) as eng:
        assert eng.gather_path.startswith("generic" if generic else "subset")
        assert eng.info["cols"] == F.shape[1]
        X = rng.integers(0, p, (F.shape[1], 4)).astype(np.uint32)
        U = rng.integers(0, p, (rows, 4)).astype(np.uint32)
        np.testing.assert_array_equal(eng.apply(APPLY_FORWARD, X), (F @ X.astype(np.int64)) % p)
        np.testing.assert_array_equal(eng.apply(APPLY_TRANSPOSE, U), (F.T @ U.astype(np.int64)) % p)
        # folded target preconditioner == round by round, and S symmetric, on the deformation operator too
        eng.validate(4)


def _run(cmd):
    return subprocess.run([str(c) for c in cmd], capture_output=True, text=True, timeout=1800)


def _sequence_outputs(tmp_path, instance, sector, op, dense_path, drop_path):
    """Runs ours and the reference's cuprym_deformation; returns {name: (wdm path, text, sidecar)}."""
    outs = {}
    for name, exe in (("ours", BIN / "cuprym_deformation"), ("ref", REF / "cuprym_deformation")):
        out_dir = tmp_path / f"o_{name}"
        cmd = [exe, instance, "--operator", op, "--sector", sector, "--out", out_dir, "--device", 0, *RECIPE,
               "--dense-file", dense_path]
        if drop_path:
            cmd += ["--drop-columns", drop_path]
        res = _run(cmd)
        assert res.returncode == 0, f"{name}: {res.stdout[-1500:]}\n{res.stderr[-1500:]}"
        stem = f"{op}-sector{sector:02d}-v4-rowmix-r2-s10001"
        wdm = out_dir / f"{stem}.wdm.zst"
        side = out_dir / f"{stem}.rowmix.json"
        outs[name] = (wdm, read_text(wdm), side.read_text().replace(f"o_{name}", "o_X"))
    return outs


def _need_reference(name):
    if not (REF / name).exists():
        pytest.skip("reference binaries not built (oracle/build_ref.sh)")


@pytest.mark.parametrize("op", ["augmented", "replacement"])
@pytest.mark.parametrize("sector", [0, 3])
def test_g12_deformation_outputs_identical_to_reference(op, sector, tmp_path):
    _need_reference("cuprym_deformation")
    inst = GOLDEN / "g12_p661.json"
    *_, dense_path, _, drop_path = _inputs(tmp_path, inst, sector, op, 101 + sector)
    outs = _sequence_outputs(tmp_path, inst, sector, op, dense_path, drop_path)
    assert outs["ours"][2] == outs["ref"][2], "rowmix sidecar differs from the reference's"
    assert outs["ours"][1] == outs["ref"][1], "WDM text differs from the reference's"


def test_g20_augmented_outputs_identical_to_reference(tmp_path):
    _need_reference("cuprym_deformation")
    inst = REF_DATA / "g20.json"
    if not inst.exists():
        pytest.skip("paper inputs not staged (oracle/build_ref.sh)")
    *_, dense_path, _, drop_path = _inputs(tmp_path, inst, 1, "augmented", 2020)
    outs = _sequence_outputs(tmp_path, inst, 1, "augmented", dense_path, drop_path)
    assert outs["ours"][2] == outs["ref"][2]
    assert outs["ours"][1] == outs["ref"][1]


def test_deformation_eliminated_operator_matches_cyclic(tmp_path):
    """cuprym_deformation --operator eliminated writes what cuprym_cyclic writes."""
    inst = GOLDEN / "g12_p661.json"
    texts = []
    for exe in ("cuprym_deformation", "cuprym_cyclic"):
        out = tmp_path / exe
        res = _run([BIN / exe, inst, "--operator", "eliminated", "--sector", 2, "--out", out, *RECIPE])
        assert res.returncode == 0, res.stderr
        texts.append(read_text(out / "eliminated-sector02-v4-rowmix-r2-s10001.wdm.zst"))
    assert texts[0] == texts[1]


@pytest.mark.parametrize("op", ["augmented", "replacement"])
@pytest.mark.parametrize("sector", [0, 1])
def test_deformation_recovery_matches_reference(op, sector, tmp_path):
    """The recovery program on each deformation variant: the same null-vector
    files and report as the reference's cuprym_deformation_kernel_vectors, from
    the same sequence files and the same generator."""
    _need_reference("cuprym_deformation_kernel_vectors")
    p = 661
    inst = GOLDEN / "g12_p661.json"
    *_, dense_path, _, drop_path = _inputs(tmp_path, inst, sector, op, 303 + sector)
    drop_args = ["--drop-columns", drop_path] if drop_path else []
    seq_dir = tmp_path / "seq"
    res = _run([BIN / "cuprym_deformation", inst, "--operator", op, "--sector", sector, "--out", seq_dir,
                *RECIPE, "--dense-file", dense_path, *drop_args])
    assert res.returncode == 0, res.stderr
    with CyclicEngine(inst, sector, op=op, dense_file=dense_path, drop_columns=drop_path) as eng:
        S = square_matrix(eng, p)
    gen = kernel_generator(S, p)
    stem = f"{op}-sector{sector:02d}-v4-rowmix-r2-s10001"
    outs = {}
    for name, exe in (("ours", BIN / "cuprym_deformation_kernel_vectors"),
                      (("ref", REF / "cuprym_deformation_kernel_vectors"))):
        d = tmp_path / f"r_{name}"
        d.mkdir()
        for suffix in (".wdm.zst", ".rowmix.json"):
            shutil.copy(seq_dir / (stem + suffix), d / (stem + suffix))
        write_generator(d / (stem + "_generators.txt"), gen, p)
        wdm = d / (stem + ".wdm.zst")
        res = _run([exe, inst, "-f", wdm, "--operator", op, "--sector", sector, "-d", 0,
                    "--dense-file", dense_path, *drop_args])
        outs[name] = (res.returncode, res.stderr, wdm)
    (rc_o, err_o, w_o), (rc_r, err_r, w_r) = outs["ours"], outs["ref"]
    assert rc_o == rc_r, (err_o, err_r)
    if rc_r != 0:
        assert err_r.strip().split("error: ", 1)[-1] in err_o
        return
    for suffix in ("_nullvectors_1.txt", "_nullvectors_2.txt"):
        assert Path(str(w_o) + suffix).read_bytes() == Path(str(w_r) + suffix).read_bytes(), suffix
    ra = json.loads(Path(str(w_o) + "_nullvectors_report.json").read_text())
    rb = json.loads(Path(str(w_r) + "_nullvectors_report.json").read_text())
    for key in ("runtime_ms", "instance", "wdm_file", "generators_file"):
        ra.pop(key)
        rb.pop(key)
    assert ra == rb


def test_deformation_refusals_match_reference(tmp_path):
    _need_reference("cuprym_deformation")
    inst = GOLDEN / "g12_p661.json"
    *_, dense_path, _, drop_path = _inputs(tmp_path, inst, 0, "replacement", 77)
    bad_dims = tmp_path / "bad_dims.json"
    write_dense_block(bad_dims, 5, 661, 1)
    bad_prime = tmp_path / "bad_prime.json"
    bad_prime.write_text(json.dumps({"rows": 1, "columns": 2, "prime": 109, "values": [1, 2]}))
    cases = [
        ["--operator", "augmented"],                                               # no dense file
        ["--operator", "replacement", "--dense-file", dense_path],                 # no drop columns
        ["--operator", "augmented", "--dense-file", dense_path, "--drop-columns", drop_path],
        ["--operator", "augmented", "--dense-file", bad_dims],
        ["--operator", "augmented", "--dense-file", bad_prime],
        ["--operator", "sideways"],
    ]
    for i, extra in enumerate(cases):
        got = {}
        for name, exe in (("ours", BIN / "cuprym_deformation"), ("ref", REF / "cuprym_deformation")):
            res = _run([exe, inst, "--sector", 0, "--out", tmp_path / f"c{i}_{name}", *RECIPE, *extra])
            got[name] = (res.returncode, res.stderr.strip().splitlines()[-1] if res.stderr.strip() else "")
        assert got["ours"] == got["ref"], (extra, got)
