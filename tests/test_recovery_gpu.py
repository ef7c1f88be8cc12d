"""Kernel-vector recovery (bin/cuprym_cyclic_kernel_vectors) against the reference binary.

A generator file is built from the minimal polynomial of S (exact linear
algebra mod p on the g12 sector, in this test): for mu(x) = x^e q(x) the
scalar generator G(x) = x^(e-1) q(x) I gives D = S^(e-1) q(S) V in ker S,
the same kind of polynomial the bcw solver exports.  Both executables read
the same WDM, sidecar and generator files; their null-vector files must be
byte-identical and their reports equal up to run time and paths.
"""
import json
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from prym_green_ancillary_b200 import CyclicEngine
from prym_green_ancillary_b200.engine import APPLY_SQUARE

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
OUR_SEQ = ROOT / "prym_green_ancillary_b200" / "bin" / "cuprym_cyclic"
OUR_REC = ROOT / "prym_green_ancillary_b200" / "bin" / "cuprym_cyclic_kernel_vectors"
REF_REC = ROOT / "oracle" / "_ref" / "bin" / "cuprym_cyclic_kernel_vectors"
RECIPE = ["--operator", "eliminated", "-v", "4", "--seed", "1", "--rowmix-rounds", "2", "--rowmix-seed", "10001"]
STEM = "eliminated-sector{:02d}-v4-rowmix-r2-s10001"


def _square_matrix(eng, p):
    n = eng.info["cols"]
    cols = []
    for c0 in range(0, n, 4):
        block = np.zeros((n, 4), dtype=np.uint32)
        for j in range(4):
            if c0 + j < n:
                block[c0 + j, j] = 1
        out = eng.apply(APPLY_SQUARE, block).astype(np.int64)
        for j in range(4):
            if c0 + j < n:
                cols.append(out[:, j])
    return np.stack(cols, axis=1) % p


def _minimal_polynomial(S, p, seed=3):
    """Monic minimal polynomial of a random vector under S (exact, Python ints)."""
    n = S.shape[0]
    v = np.random.default_rng(seed).integers(0, p, n).astype(object)
    krylov = [v]
    Sobj = S.astype(object)
    basis, pivots = [], []   # reduced echelon rows with combination coefficients
    for d in range(n + 1):
        w = krylov[-1]
        # reduce w against the basis, tracking the combination of Krylov vectors
        comb = [0] * (d + 1)
        comb[d] = 1
        w = list(w)
        for (row, rcomb), pc in zip(basis, pivots):
            f = w[pc] % p
            if f:
                w = [(a - f * b) % p for a, b in zip(w, row)]
                for i, c in enumerate(rcomb):
                    comb[i] = (comb[i] - f * c) % p
        nz = next((i for i, a in enumerate(w) if a % p), None)
        if nz is None:
            return [c % p for c in comb]    # sum comb[i] S^i v = 0, comb[d] = 1
        inv = pow(int(w[nz]), -1, p)
        basis.append(([a * inv % p for a in w], [c * inv % p for c in comb]))
        pivots.append(nz)
        krylov.append(np.array([int(x) for x in Sobj.dot(np.array(krylov[-1], dtype=object)) % p], dtype=object))
    raise AssertionError("no minimal polynomial found")


def _write_generator(path, coeffs, p):
    with open(path, "w") as f:
        for c in coeffs:
            m = np.zeros((4, 4), dtype=np.int64)
            np.fill_diagonal(m, c % p)
            # exported generator entries may be negative: write some as c - p
            row = [int(x) if (i % 5) else int(x) - p if x else 0 for i, x in enumerate(m.reshape(-1))]
            f.write(" ".join(str(x) for x in row) + "\n")


def _run(cmd):
    return subprocess.run(cmd, capture_output=True, text=True, timeout=1200)


@pytest.mark.parametrize("sector", [0, 1])
def test_recovery_matches_reference_binary(sector, tmp_path):
    if not REF_REC.exists():
        pytest.skip("reference binary not built (oracle/build_ref.sh)")
    p = 661
    inst = GOLDEN / "g12_p661.json"
    seq_dir = tmp_path / "seq"
    res = _run([str(OUR_SEQ), str(inst), "--sector", str(sector), "--out", str(seq_dir), *RECIPE])
    assert res.returncode == 0, res.stderr
    with CyclicEngine(inst, sector) as eng:
        S = _square_matrix(eng, p)
    mu = _minimal_polynomial(S, p)
    e = next(i for i, c in enumerate(mu) if c)
    # x^(e-1) q(x) for mu = x^e q(x); mu itself when S is invertible (then D = mu(S) V = 0)
    gen = [0] * (e - 1) + mu[e:] if e >= 1 else mu
    stem = STEM.format(sector)
    outs = {}
    for name, exe in (("ours", OUR_REC), ("ref", REF_REC)):
        d = tmp_path / f"r_{name}"
        d.mkdir()
        for suffix in (".wdm.zst", ".rowmix.json"):
            shutil.copy(seq_dir / (stem + suffix), d / (stem + suffix))
        _write_generator(d / (stem + "_generators.txt"), gen, p)
        wdm = d / (stem + ".wdm.zst")
        res = _run([str(exe), str(inst), "-f", str(wdm), "--operator", "eliminated", "--sector", str(sector),
                    "-d", "0"])
        outs[name] = (res.returncode, res.stderr, d, wdm)
    (rc_o, err_o, d_o, w_o), (rc_r, err_r, d_r, w_r) = outs["ours"], outs["ref"]
    assert rc_o == rc_r, (err_o, err_r)
    if rc_r != 0:
        # the same refusal (for an invertible S every candidate is zero)
        msg_r = err_r.strip().split("error: ", 1)[-1]
        assert msg_r in err_o
        return
    for suffix in ("_nullvectors_1.txt", "_nullvectors_2.txt"):
        a = (Path(str(w_o) + suffix)).read_bytes()
        b = (Path(str(w_r) + suffix)).read_bytes()
        assert a == b, f"{suffix} differs from the reference's"
    ra = json.loads(Path(str(w_o) + "_nullvectors_report.json").read_text())
    rb = json.loads(Path(str(w_r) + "_nullvectors_report.json").read_text())
    for key in ("runtime_ms", "instance", "wdm_file", "generators_file"):
        ra.pop(key)
        rb.pop(key)
    assert ra == rb
    if sector == 0:
        assert ra["candidate_rank"] >= 1 and sum(ra["product_nonzeros"]) == 0
