"""Paper-mode host assembly on the CPU (host-only contexts, no device calls).

Sector shapes are checked against the reference's explicit-matrix oracle
(tests/golden/cyclic_g12_golden.npz, from tests/deformation_reference.py of the
reference) and the instance's own sector_columns / sector_rows metadata.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from prym_green_ancillary_b200 import CyclicEngine, EngineError

GOLDEN = Path(__file__).parent / "golden"
G = np.load(GOLDEN / "cyclic_g12_golden.npz")


@pytest.mark.parametrize("p", [661, 109])
@pytest.mark.parametrize("sector", range(6))
def test_sector_shapes_match_explicit_matrices(p, sector):
    F = G[f"p{p}/sector{sector}/F"]
    with CyclicEngine(GOLDEN / f"g12_p{p}.json", sector, device=-1) as eng:
        assert (eng.info["rows"], eng.info["cols"]) == F.shape
        assert eng.info["prime"] == p and eng.info["genus"] == 12 and eng.info["order"] == 6
        assert eng.info["default_nlen"] == 2 * F.shape[1] // 4 + 50


def test_sidecar_text(tmp_path):
    with CyclicEngine(GOLDEN / "g12_p661.json", 0, device=-1) as eng:
        wdm = eng.output_path(tmp_path / "out")
        assert wdm.endswith("eliminated-sector00-v4-rowmix-r2-s10001.wdm.zst")
        eng.write_sidecar(wdm)
        side = Path(wdm[: -len(".wdm.zst")] + ".rowmix.json")
        doc = json.loads(side.read_text())
        assert doc["type"] == "prym_cyclic_rowmix_sidecar" and doc["algorithm_version"] == "paired-sl2-target-v1"
        assert doc["rows"] == eng.info["rows"] and doc["columns"] == eng.info["cols"]
        assert doc["rowmix"]["realized_seed"] == eng.info["rowmix_realized_seed"]
        assert doc["rowmix"]["hash_fnv1a64"] == "0x%016x" % eng.info["rowmix_hash"]
        assert doc["rowmix"]["pair_count_per_round"] == [eng.info["rows"] // 2] * 2
        # refusing to overwrite (cuda/cuprym_cyclic.cu:1323-1334)
        with pytest.raises(EngineError, match="refusing to reuse existing rowmix sidecar"):
            from prym_green_ancillary_b200.engine import load, _check
            _check(load().bw_cyclic_check_outputs_absent(wdm.encode()))


def test_host_only_context_refuses_device_work():
    with CyclicEngine(GOLDEN / "g12_p661.json", 1, device=-1) as eng:
        with pytest.raises(EngineError, match="host-only"):
            eng.generate()


@pytest.mark.parametrize("kw, msg", [
    (dict(op="sideways"), "--operator must be one of: eliminated, augmented, replacement."),
    (dict(op="augmented"), "deformation operators require --dense-file"),
    (dict(num_v=8), "exactly 4 block vectors"),
    (dict(sector=6), "--sector must be in 0..5"),
])
def test_paper_recipe_refusals(kw, msg):
    args = dict(sector=0)
    args.update(kw)
    with pytest.raises(EngineError, match=msg):
        CyclicEngine(GOLDEN / "g12_p661.json", device=-1, **args)


def test_tampered_instance_is_rejected(tmp_path):
    doc = json.loads((GOLDEN / "g12_p661.json").read_text())
    e = doc["third_section_elimination"]
    flat = e["right_inverse_A0_by_A1"]
    first = flat[0] if isinstance(flat[0], list) else flat
    first[0] = (first[0] + 1) % doc["modulus"]
    bad = tmp_path / "bad.json"
    bad.write_text(json.dumps(doc))
    with pytest.raises(EngineError, match="mu_w\\*R=I failed"):
        CyclicEngine(bad, 0, device=-1)


# ----- deformation inputs (host-only contexts; the reference's refusals)

def _dense(tmp_path, n_rows, p=661, over=None):
    from paper_helpers import write_dense_block
    path = tmp_path / "dense.json"
    write_dense_block(path, n_rows, p, 5)
    if over:
        doc = json.loads(path.read_text())
        doc.update(over)
        path.write_text(json.dumps(doc))
    return path


def _shape(sector=0):
    with CyclicEngine(GOLDEN / "g12_p661.json", sector, device=-1) as eng:
        return eng.info["rows"], eng.info["cols"]


def test_deformation_operator_columns(tmp_path):
    rows, base = _shape()
    dense = _dense(tmp_path, rows)
    with CyclicEngine(GOLDEN / "g12_p661.json", 0, op="augmented", dense_file=dense, device=-1) as eng:
        assert (eng.info["rows"], eng.info["cols"]) == (rows, base + 2)
        assert eng.info["default_nlen"] == 2 * (base + 2) // 4 + 50
    drop = tmp_path / "drop.json"
    drop.write_text(json.dumps({"indices": [base - 1, 3]}))
    with CyclicEngine(GOLDEN / "g12_p661.json", 0, op="replacement", dense_file=dense, drop_columns=drop,
                      device=-1) as eng:
        assert eng.info["cols"] == base


@pytest.mark.parametrize("over, drop, msg", [
    (dict(prime=109), None, "dense block prime does not match instance modulus"),
    (dict(columns=3), None, "values has"),
    (dict(rows=5), None, "values has"),
    (dict(values=[700, 1]), None, "values has"),
    (None, [1], "drop-column file has the wrong number of indices"),
    (None, [4, 4], "drop-column indices must be distinct"),
    (None, [0, 10 ** 6], "drop-column index is outside the base column range"),
])
def test_deformation_input_refusals(tmp_path, over, drop, msg):
    rows, _ = _shape()
    dense = _dense(tmp_path, rows, over=over)
    kw = dict(op="augmented")
    if drop is not None:
        path = tmp_path / "drop.json"
        path.write_text(json.dumps({"indices": drop}))
        kw = dict(op="replacement", drop_columns=path)
    with pytest.raises(EngineError, match=msg):
        CyclicEngine(GOLDEN / "g12_p661.json", 0, dense_file=dense, device=-1, **kw)


def test_dense_values_must_be_reduced(tmp_path):
    rows, _ = _shape()
    vals = [[1, 2]] * (rows - 1) + [[661, 0]]
    path = tmp_path / "dense.json"
    path.write_text(json.dumps({"rows": rows, "columns": 2, "prime": 661, "values": vals}))
    with pytest.raises(EngineError, match="not reduced modulo the instance modulus"):
        CyclicEngine(GOLDEN / "g12_p661.json", 0, op="augmented", dense_file=path, device=-1)


def test_drop_columns_only_for_replacement(tmp_path):
    rows, _ = _shape()
    dense = _dense(tmp_path, rows)
    drop = tmp_path / "drop.json"
    drop.write_text(json.dumps({"indices": [0, 1]}))
    with pytest.raises(EngineError, match="only meaningful for replacement"):
        CyclicEngine(GOLDEN / "g12_p661.json", 0, op="augmented", dense_file=dense, drop_columns=drop, device=-1)
    with pytest.raises(EngineError, match="replacement operator requires --drop-columns"):
        CyclicEngine(GOLDEN / "g12_p661.json", 0, op="replacement", dense_file=dense, device=-1)


def test_dense_dimensions_must_match_sector(tmp_path):
    rows, _ = _shape()
    dense = _dense(tmp_path, rows - 1)
    with pytest.raises(EngineError, match="dense block dimensions do not match the eliminated target sector"):
        CyclicEngine(GOLDEN / "g12_p661.json", 0, op="augmented", dense_file=dense, device=-1)
