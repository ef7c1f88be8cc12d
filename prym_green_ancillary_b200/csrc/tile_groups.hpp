// Grouped tiles for the INT8 gather-GEMM (host code, no CUDA).
//
// A tile of the gather-GEMM is BT output blocks; its K dimension runs over the
// generators that any of its blocks is incident to.  In rank order the blocks
// of a tile share few generators: a k-subset block of d^T touches its own k
// generators, and eight consecutive k-subsets together touch nearly all r.
// The rows of every other generator are zero-filled copies and zero MMA rows.
//
// Grouping instead puts together blocks whose generator sets (all of one size
// c: k for d^T, r - k + 1 for d) lie inside one common set U of c + 1
// generators, then c + 2, so the tile's K covers |U| generators instead of r.
// Every c-subset of U is a block, so a U holds c + e candidates for e = 1.  A
// greedy pass over all U in increasing mask order takes BT unused candidates at
// a time.  The blocks left after both passes are grouped in runs of BT
// consecutive blocks.  Any partition is exact: a tile's output is its blocks'
// own sums, whatever the K order.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <vector>

namespace bw {

struct TileGroups {
    int bt = 0;
    std::vector<int32_t> blk;    // [n_tiles * bt]: output block at each tile position, -1 when empty
    std::vector<uint8_t> gens;   // [n_tiles * 32]: the tile's union of generators, ascending
    std::vector<uint8_t> ngen;   // [n_tiles]: size of the union
    uint64_t n_tiles() const { return ngen.size(); }
    double mean_union() const {
        double s = 0;
        for (uint8_t v : ngen) s += v;
        return ngen.empty() ? 0.0 : s / static_cast<double>(ngen.size());
    }
};

// present[b] = bit i set when output block b is incident to generator i
// (i < r <= 31).  Blocks with equal masks are allowed (the later ones are
// grouped with the leftovers).
inline TileGroups group_tiles(const std::vector<uint32_t>& present, int r, int bt) {
    if (r < 1 || r > 31 || bt < 1 || bt > 32) throw std::invalid_argument("group_tiles: r or bt out of range");
    const uint64_t n_blk = present.size();
    uint64_t C[33][33] = {};
    for (int n = 0; n <= 32; ++n) {
        C[n][0] = 1;
        for (int j = 1; j <= n; ++j) C[n][j] = C[n - 1][j - 1] + C[n - 1][j];
    }
    int c = -1;
    bool uniform = n_blk > 0;
    for (uint64_t b = 0; b < n_blk; ++b) {
        if (present[b] >> r) throw std::invalid_argument("group_tiles: generator index above r");
        const int pc = __builtin_popcount(present[b]);
        if (c < 0) c = pc;
        else if (pc != c) uniform = false;
    }
    // colex rank of a c-subset: sum over its j-th smallest element p of C(p, j + 1)
    auto colex = [&](uint32_t m) {
        uint64_t rk = 0;
        for (int j = 1; m; ++j, m &= m - 1) rk += C[__builtin_ctz(m)][j];
        return rk;
    };
    std::vector<uint8_t> used(n_blk, 0);
    TileGroups G;
    G.bt = bt;
    auto emit = [&](const int32_t* members, int cnt) {
        uint32_t u = 0;
        for (int q = 0; q < cnt; ++q) {
            u |= present[members[q]];
            used[members[q]] = 1;
        }
        for (int q = 0; q < bt; ++q) G.blk.push_back(q < cnt ? members[q] : -1);
        uint8_t list[32] = {};
        int n = 0;
        for (int i = 0; i < r; ++i)
            if ((u >> i) & 1u) list[n++] = static_cast<uint8_t>(i);
        G.gens.insert(G.gens.end(), list, list + 32);
        G.ngen.push_back(static_cast<uint8_t>(n));
    };
    if (uniform && c >= 1 && c < r) {
        std::vector<int32_t> of_rank(C[r][c], -1);
        for (uint64_t b = 0; b < n_blk; ++b) {
            int32_t& slot = of_rank[colex(present[b])];
            if (slot < 0) slot = static_cast<int32_t>(b);
        }
        std::vector<int32_t> cand;
        for (int e = 1; e <= 2 && c + e <= r; ++e) {
            for (uint32_t U = (1u << (c + e)) - 1; U < (1u << r);) {
                cand.clear();
                for (uint32_t x = U; x; x &= x - 1) {
                    const uint32_t bx = x & (~x + 1u);
                    if (e == 1) {
                        const int32_t b = of_rank[colex(U ^ bx)];
                        if (b >= 0 && !used[b]) cand.push_back(b);
                    } else {
                        for (uint32_t y = x & (x - 1); y; y &= y - 1) {
                            const int32_t b = of_rank[colex(U ^ bx ^ (y & (~y + 1u)))];
                            if (b >= 0 && !used[b]) cand.push_back(b);
                        }
                    }
                }
                for (size_t q = 0; q + bt <= cand.size(); q += bt) emit(cand.data() + q, bt);
                // next mask with the same number of bits (Gosper)
                const uint32_t t = U | (U - 1);
                U = (t + 1) | (((~t & (t + 1)) - 1) >> (__builtin_ctz(U) + 1));
            }
        }
    }
    int32_t run[32];
    int n = 0;
    for (uint64_t b = 0; b < n_blk; ++b) {
        if (used[b]) continue;
        run[n++] = static_cast<int32_t>(b);
        if (n == bt) {
            emit(run, n);
            n = 0;
        }
    }
    if (n > 0) emit(run, n);
    return G;
}

}  // namespace bw
