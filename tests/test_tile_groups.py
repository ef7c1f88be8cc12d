"""Grouped tiles of the INT8 gather-GEMM (csrc/tile_groups.hpp), on the CPU.

The header is plain C++; a small harness compiled here enumerates the output
blocks of d (the complements of the (k-1)-subsets: the generators a block of
d is incident to) and of d^T (the k-subsets) in rank order, groups them and
checks that the tiles are a partition of the blocks, that every block's
generators lie in its tile's union, and that the unions are the small ones the
grouping is for: at the bench's config-2 and config-5 shapes every tile but
the last is full and the mean union is within 1.3 of the blocks' own generator count
(against r for tiles of consecutive blocks).
"""
import json
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "prym_green_ancillary_b200" / "csrc" / "tile_groups.hpp"

HARNESS = r"""
#include "tile_groups.hpp"
#include <cstdio>
#include <cstdlib>
using namespace bw;
static void subsets(int r, int c, bool complement, std::vector<uint32_t>& out) {
    std::vector<int> a(c);
    for (int i = 0; i < c; ++i) a[i] = i;
    for (;;) {
        uint32_t m = 0;
        for (int v : a) m |= 1u << v;
        out.push_back(complement ? (~m & ((1u << r) - 1)) : m);
        int i = c - 1;
        while (i >= 0 && a[i] == r - c + i) --i;
        if (i < 0) break;
        ++a[i];
        for (int j = i + 1; j < c; ++j) a[j] = a[j - 1] + 1;
    }
}
int main(int argc, char** argv) {
    const int r = atoi(argv[1]), k = atoi(argv[2]), bt = atoi(argv[3]), dir = atoi(argv[4]);
    std::vector<uint32_t> m;
    if (dir == 0) subsets(r, k - 1, true, m); else subsets(r, k, false, m);
    const TileGroups G = group_tiles(m, r, bt);
    std::vector<int> seen(m.size(), 0);
    long long bad_union = 0, bad_list = 0, full = 0;
    for (uint64_t t = 0; t < G.n_tiles(); ++t) {
        uint32_t u = 0, want = 0;
        for (int g = 0; g < G.ngen[t]; ++g) {
            if (g > 0 && G.gens[t * 32 + g] <= G.gens[t * 32 + g - 1]) ++bad_list;
            u |= 1u << G.gens[t * 32 + g];
        }
        int cnt = 0;
        for (int q = 0; q < bt; ++q) {
            const int b = G.blk[t * bt + q];
            if (b < 0) continue;
            ++cnt;
            if (b >= (int)m.size()) { ++bad_union; continue; }
            ++seen[b];
            want |= m[b];
        }
        if (u != want) ++bad_union;   // the list is exactly the union of the tile's blocks
        if (cnt == bt) ++full;
    }
    long long missing = 0, twice = 0;
    for (int v : seen) { missing += v == 0; twice += v > 1; }
    printf("{\"blocks\": %zu, \"tiles\": %llu, \"full\": %lld, \"mean_union\": %.4f, \"bad_union\": %lld, "
           "\"bad_list\": %lld, \"missing\": %lld, \"twice\": %lld}\n", m.size(), (unsigned long long)G.n_tiles(),
           full, G.mean_union(), bad_union, bad_list, missing, twice);
    return 0;
}
"""


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    d = tmp_path_factory.mktemp("tile_groups")
    src = d / "harness.cpp"
    src.write_text(HARNESS)
    exe = d / "harness"
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", str(HEADER.parent), str(src), "-o", str(exe)], check=True)
    return exe


def _run(exe, r, k, bt, direction):
    out = subprocess.run([str(exe), str(r), str(k), str(bt), str(direction)], check=True, capture_output=True,
                         text=True, timeout=120).stdout
    return json.loads(out)


@pytest.mark.parametrize("r, k", [(6, 3), (7, 1), (6, 6), (8, 4), (10, 5), (9, 4), (12, 6)])
@pytest.mark.parametrize("bt", [4, 8])
@pytest.mark.parametrize("direction", [0, 1], ids=["d", "dT"])
def test_small_shapes_are_partitions(harness, r, k, bt, direction):
    res = _run(harness, r, k, bt, direction)
    assert res["missing"] == 0 and res["twice"] == 0
    assert res["bad_union"] == 0 and res["bad_list"] == 0
    assert res["tiles"] >= -(-res["blocks"] // bt)


@pytest.mark.parametrize("r, k, bt", [(19, 9, 8), (23, 11, 4)], ids=["config2", "config5"])
@pytest.mark.parametrize("direction", [0, 1], ids=["d", "dT"])
def test_bench_shapes_group_into_full_tiles_with_small_unions(harness, r, k, bt, direction):
    res = _run(harness, r, k, bt, direction)
    assert res["missing"] == 0 and res["twice"] == 0 and res["bad_union"] == 0 and res["bad_list"] == 0
    assert res["tiles"] == -(-res["blocks"] // bt)   # as many tiles as consecutive blocks would take
    assert res["full"] >= res["tiles"] - 1
    own = r - k + 1 if direction == 0 else k
    assert own <= res["mean_union"] <= own + 1.3, res
