"""The C-ABI library loads on a CPU-only machine and exports every declared symbol.

No compute call is made here (there is no GPU); argument validation runs
before any CUDA call, so the error convention is checked too.
"""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from prym_green_ancillary_b200 import engine

ROOT = Path(__file__).resolve().parents[1]
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_symbols():
    names = set()
    for h in HEADERS:
        text = h.read_text()
        names |= set(re.findall(r"^BW_API\s+[\w\s\*]+?\b(bw_\w+)\s*\(", text, flags=re.M))
    return sorted(names)


def test_headers_declare_symbols():
    assert len(declared_symbols()) >= 10


@pytest.mark.parametrize("name", declared_symbols())
def test_symbol_exported(name):
    lib = ctypes.CDLL(str(engine.LIB_PATH))
    assert hasattr(lib, name), f"{name} declared in include/ but not exported"


def test_binding_covers_header():
    missing = [n for n in declared_symbols() if n not in engine.SIGNATURES]
    assert not missing, f"engine.py has no signature for {missing}"


def test_abi_version():
    assert engine.load().bw_abi_version() == 2


def test_seeded_host_matches_oracle():
    import oracle
    for tag, lo in ((1, 0), (2, 1), (4, 0)):
        got = engine.seeded_fill_host(1000, 12345, tag, 32003, lo)
        np.testing.assert_array_equal(got, oracle.seeded(12345, tag, 1000, 32003, lo))


@pytest.mark.parametrize("kw, msg", [
    (dict(prime=32001), "not prime"),
    (dict(prime=65537), "below 2^15"),
    (dict(block_width=12), "4, 8, 16 or 32"),
    (dict(r=40), "r must be"),
    (dict(k=0), "k must be"),
])
def test_invalid_arguments_fail_loudly(kw, msg):
    args = dict(r=6, k=3, dim_in=3, dim_out=4, prime=101, block_width=4)
    args.update(kw)
    maps = np.ones(args["r"] * args["dim_in"] * args["dim_out"], dtype=np.uint32)
    diag = np.ones(1000, dtype=np.uint32)
    with pytest.raises(engine.EngineError) as err:
        engine.KoszulEngine(maps=maps, diag=diag, **args)
    assert msg in str(err.value)
