#!/usr/bin/env python3
"""Generate the paper-mode golden fixtures from the reference's own code.

    python tests/golden/make_cyclic_golden.py --reference <reference checkout>

* ``g12_p661.json`` / ``g12_p109.json``: genus-12 instances made by the
  reference's ``scripts.prepare_deformation.build_instance`` (the instance its
  GPU integration test builds, tests/check_cuda.py:74, and its CPU unit test,
  tests/test_deformation_reference.py:10).
* ``cyclic_g12_golden.npz``: for each prime and sector, the explicit
  eliminated operator block F_c assembled by the reference's exact
  sparse-matrix oracle (tests/deformation_reference.py:75-165, ``assemble``),
  its rank (``check``), and the sector shapes.
"""
import argparse
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def main():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--reference", type=Path, required=True)
    args = ap.parse_args()
    sys.path.insert(0, str(args.reference))
    sys.path.insert(0, str(args.reference / "tests"))
    from scripts.prepare_deformation import build_instance
    from deformation_reference import assemble, check

    arrays = {}
    for p in (661, 109):
        fixture = build_instance(12, p)
        (HERE / f"g12_p{p}.json").write_text(json.dumps(fixture, separators=(",", ":")) + "\n")
        matrices, rows, cols = assemble(fixture)
        f0 = matrices[0]
        r = fixture["cyclic"]["order"]
        result = check(fixture)
        for c in range(r):
            ri = np.flatnonzero(rows == c)
            ci = np.flatnonzero(cols == c)
            block = f0[ri][:, ci].toarray() % p
            arrays[f"p{p}/sector{c}/F"] = block.astype(np.uint32)
            arrays[f"p{p}/sector{c}/rank"] = np.array([result["sector_profiles"][c]["rank"]], dtype=np.int64)
        arrays[f"p{p}/order"] = np.array([r], dtype=np.int64)
        print("p", p, [(c["rows"], c["columns"], c["rank"]) for c in result["sector_profiles"]])
    np.savez_compressed(HERE / "cyclic_g12_golden.npz", **arrays)


if __name__ == "__main__":
    main()
