"""The INT8 epilogue's modular arithmetic (csrc/bw_common.cuh), on the CPU.

The header's helpers are host-and-device inline functions; a harness compiled
here with the host compiler checks them against exact 64-bit arithmetic:

* reduce_balanced_fast(x) is the balanced residue for every |x| <= 2^31 - 2p
  (random values, the range ends, multiples of p and their neighbours);
* the epilogue's chain (ll + 255 (lh + hl) + c2 hh, then times the diagonal
  entry, one Barrett step each) gives the balanced residue of the exact
  value, at the extreme accumulator sizes of 1024 K rows of int8 limbs;
* neg_bytes4 negates every byte in [-127, 127] of a packed word.
"""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "prym_green_ancillary_b200" / "csrc"
CUDA_INCLUDE = Path("/usr/local/cuda/include")

HARNESS = r"""
#include "bw_common.cuh"
#include <cstdio>
#include <random>
using namespace bw;
static int64_t bal(int64_t x, int64_t p) { int64_t r = ((x % p) + p) % p; return r > (p - 1) / 2 ? r - p : r; }
int main() {
    const uint32_t primes[] = {3, 5, 7, 251, 257, 1093, 32003, 32749};   // 32749: the largest 15-bit prime
    std::mt19937_64 g(7);
    long long bad_fast = 0, bad_chain = 0, bad_neg = 0, checked = 0;
    for (uint32_t pu : primes) {
        const Mod m = make_mod(pu);
        const int64_t p = pu, lim = (int64_t{1} << 31) - 2 * p;
        auto check = [&](int64_t x) {
            if (x < -lim || x > lim) return;   // outside the stated range
            ++checked;
            if (reduce_balanced_fast(static_cast<int32_t>(x), m) != bal(x, p)) ++bad_fast;
        };
        for (int64_t x : {-lim, -lim + 1, lim - 1, lim, int64_t{0}, int64_t{1}, int64_t{-1}, p, -p, p - 1, 1 - p,
                          int64_t{(p - 1) / 2}, -int64_t{(p - 1) / 2}, int64_t{(p + 1) / 2}, -int64_t{(p + 1) / 2}})
            check(x);
        for (int64_t k = -3; k <= 3; ++k)
            for (int64_t d = -2; d <= 2; ++d) check((lim / p - k) * p + d);
        std::uniform_int_distribution<int64_t> any(-lim, lim);
        for (int i = 0; i < 200000; ++i) check(any(g));
        // the epilogue chain at the accumulators' extreme sizes
        const int64_t c2 = bal(255 * 255, p);
        const int64_t LL = 1024LL * 127 * 127, LH = 2LL * 1024 * 127 * 64, HH = 1024LL * 64 * 64;
        std::uniform_int_distribution<int64_t> ll_d(-LL, LL), lh_d(-LH, LH), hh_d(-HH, HH), dg_d(-(p - 1) / 2, (p - 1) / 2);
        for (int i = 0; i < 200000; ++i) {
            const int64_t ll = i < 8 ? ((i & 1) ? LL : -LL) : ll_d(g);
            const int64_t lh = i < 8 ? ((i & 2) ? LH : -LH) : lh_d(g);
            const int64_t hh = i < 8 ? ((i & 4) ? HH : -HH) : hh_d(g);
            const int64_t dg = i < 4 ? ((i & 1) ? (p - 1) / 2 : -(p - 1) / 2) : dg_d(g);
            const int32_t t = static_cast<int32_t>(ll) + 255 * reduce_partial(static_cast<int32_t>(lh), m) +
                              static_cast<int32_t>(c2) * reduce_partial(static_cast<int32_t>(hh), m);
            const int32_t plain = reduce_balanced_fast(t, m);
            const int32_t scaled = reduce_balanced_fast(reduce_partial(t, m) * static_cast<int32_t>(dg), m);
            const int64_t exact = ll + 255 * lh + 65025 * hh;
            if (plain != bal(exact, p) || scaled != bal(bal(exact, p) * dg, p)) ++bad_chain;
        }
    }
    for (int a = -127; a <= 127; ++a)
        for (int b = -127; b <= 127; ++b) {
            const uint32_t w = static_cast<uint8_t>(a) | static_cast<uint32_t>(static_cast<uint8_t>(b)) << 8 |
                               static_cast<uint32_t>(static_cast<uint8_t>(-a)) << 16 |
                               static_cast<uint32_t>(static_cast<uint8_t>(b / 2)) << 24;
            const uint32_t n = neg_bytes4(w);
            for (int q = 0; q < 4; ++q)
                if (static_cast<int8_t>(n >> (8 * q)) != -static_cast<int8_t>(w >> (8 * q))) ++bad_neg;
        }
    std::printf("%lld %lld %lld %lld\n", checked, bad_fast, bad_chain, bad_neg);
    return 0;
}
"""


def test_epilogue_arithmetic_is_exact(tmp_path):
    cxx = shutil.which("g++")
    if cxx is None or not (CUDA_INCLUDE / "cuda_runtime.h").exists():
        pytest.skip("needs g++ and the CUDA headers")
    src = tmp_path / "mod.cpp"
    src.write_text(HARNESS)
    exe = tmp_path / "mod"
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", str(CSRC), "-I", str(CUDA_INCLUDE), str(src), "-o", str(exe)],
                   check=True)
    checked, bad_fast, bad_chain, bad_neg = (int(v) for v in
                                             subprocess.run([str(exe)], check=True, capture_output=True, text=True,
                                                            timeout=120).stdout.split())
    assert checked > 1_000_000
    assert (bad_fast, bad_chain, bad_neg) == (0, 0, 0)
