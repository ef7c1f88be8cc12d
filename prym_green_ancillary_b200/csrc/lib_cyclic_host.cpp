// Host-side assembly of the eliminated cyclic operator (see cyclic_host.hpp).
#include "cyclic_host.hpp"

#include "json_lite.hpp"

#include <algorithm>
#include <cctype>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <limits>
#include <map>
#include <sstream>
#include <stdexcept>
#include <thread>

namespace bw {
namespace cyclic {

namespace {

constexpr uint64_t kFnvOffset = 14695981039346656037ULL;
constexpr uint64_t kFnvPrime = 1099511628211ULL;

uint64_t binom64(size_t n, size_t k) {
    if (k > n) return 0;
    k = std::min(k, n - k);
    unsigned __int128 out = 1;
    for (size_t i = 0; i < k; ++i) {
        out = out * (n - i) / (i + 1);
        if (out > std::numeric_limits<uint64_t>::max()) throw std::runtime_error("binomial coefficient overflows u64");
    }
    return static_cast<uint64_t>(out);
}

uint32_t sub_mod(size_t a, size_t b, size_t r) { return static_cast<uint32_t>((a + r - (b % r)) % r); }

uint32_t checked_u32(size_t v, const std::string& label) {
    if (v > std::numeric_limits<uint32_t>::max()) throw std::runtime_error(label + " does not fit in uint32_t");
    return static_cast<uint32_t>(v);
}

std::string read_file(const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("failed to open " + path);
    std::ostringstream ss;
    ss << in.rdbuf();
    return ss.str();
}

std::vector<uint16_t> weight_array(const json::Value& obj, const std::string& key, size_t r) {
    std::vector<int64_t> raw = obj.at(key).ints(key);
    std::vector<uint16_t> out;
    out.reserve(raw.size());
    for (int64_t v : raw) {
        if (v < 0 || static_cast<uint64_t>(v) >= r || v > 65535)
            throw std::runtime_error("weight " + std::to_string(v) + " in " + key + " is outside 0..r-1");
        out.push_back(static_cast<uint16_t>(v));
    }
    return out;
}

std::vector<uint32_t> mod_array(const json::Value& obj, const std::string& key, size_t expected, uint32_t modulus) {
    std::vector<int64_t> raw = obj.at(key).ints(key);
    if (expected != 0 && raw.size() != expected)
        throw std::runtime_error(key + " has " + std::to_string(raw.size()) + " entries; expected " +
                                 std::to_string(expected));
    std::vector<uint32_t> out;
    out.reserve(raw.size());
    for (int64_t v : raw) {
        if (v < 0 || static_cast<uint64_t>(v) >= modulus)
            throw std::runtime_error(key + " entry is not reduced modulo the instance modulus");
        out.push_back(static_cast<uint32_t>(v));
    }
    return out;
}

std::vector<uint64_t> u64_array(const json::Value& obj, const std::string& key) {
    std::vector<int64_t> raw = obj.at(key).ints(key);
    std::vector<uint64_t> out(raw.size());
    for (size_t i = 0; i < raw.size(); ++i) {
        if (raw[i] < 0) throw std::runtime_error(key + " has a negative entry");
        out[i] = static_cast<uint64_t>(raw[i]);
    }
    return out;
}

// mu_w R = I and mu_w B = 0 (cuda/cuprym_cyclic.cu:423-481).
void validate_elimination(const Instance& inst) {
    if (!inst.has_elimination) return;
    if (inst.w_index >= inst.n) throw std::runtime_error("elimination w_V_index is outside V");
    if (inst.w_weight != inst.weight_v[inst.w_index])
        throw std::runtime_error("elimination w_weight does not match V weight");
    if (inst.right_inverse.size() != inst.genus * inst.n)
        throw std::runtime_error("elimination right inverse has wrong shape");
    const size_t kd = inst.kernel_dim();
    if (kd == 0) throw std::runtime_error("elimination kernel basis is empty");
    if (inst.kernel_basis.size() != inst.genus * kd) throw std::runtime_error("elimination kernel basis has wrong shape");
    const uint64_t p = inst.modulus;
    for (size_t beta = 0; beta < inst.n; ++beta) {
        for (size_t gamma = 0; gamma < inst.n; ++gamma) {
            uint64_t acc = 0;
            for (size_t a = 0; a < inst.genus; ++a)
                acc = (acc + static_cast<uint64_t>(inst.mu_at(inst.w_index, beta, a)) *
                                 inst.right_inverse[a * inst.n + gamma]) % p;
            if (acc != (beta == gamma ? 1u : 0u))
                throw std::runtime_error("elimination right inverse check mu_w*R=I failed");
        }
        for (size_t k = 0; k < kd; ++k) {
            uint64_t acc = 0;
            for (size_t a = 0; a < inst.genus; ++a)
                acc = (acc + static_cast<uint64_t>(inst.mu_at(inst.w_index, beta, a)) *
                                 inst.kernel_basis[a * kd + k]) % p;
            if (acc != 0) throw std::runtime_error("elimination kernel check mu_w*B=0 failed");
        }
    }
}

uint64_t fnv_u8(uint64_t h, uint8_t v) { return (h ^ v) * kFnvPrime; }
uint64_t fnv_u64(uint64_t h, uint64_t v) {
    for (int b = 0; b < 8; ++b) h = fnv_u8(h, static_cast<uint8_t>((v >> (8 * b)) & 0xffu));
    return h;
}
uint64_t fnv_str(uint64_t h, const std::string& s) {
    for (unsigned char c : s) h = fnv_u8(h, c);
    return h;
}

// C(n, k) for n, k < 64 (0 when k > n; saturates at 2^64 - 1, never reached by
// the subset counts that pass the u32 checks).
struct BinomTable {
    uint64_t c[64][64];
    BinomTable() {
        for (int n = 0; n < 64; ++n)
            for (int k = 0; k < 64; ++k) {
                if (k == 0) c[n][k] = 1;
                else if (n == 0) c[n][k] = 0;
                else {
                    const uint64_t a = c[n - 1][k - 1], b = c[n - 1][k];
                    c[n][k] = a > ~b ? ~0ULL : a + b;
                }
            }
    }
};
const BinomTable& binoms() {
    static const BinomTable t;
    return t;
}

// Lexicographic rank of a k-subset of {0..n-1} given as a bit mask:
// rank = C(n,k) - 1 - sum_pos C(n-1-s_pos, k-pos).
uint64_t lex_rank_mask(uint64_t mask, size_t n, size_t k) {
    const BinomTable& B = binoms();
    uint64_t acc = 0;
    size_t pos = 0;
    for (uint64_t m = mask; m && pos < k; m &= m - 1) {
        const size_t v = static_cast<size_t>(__builtin_ctzll(m));
        acc += B.c[n - 1 - v][k - pos++];
    }
    return B.c[n][k] - 1 - acc;
}

// The k-subset of {0..n-1} with lexicographic rank `rank` (inverse of lex_rank_mask).
void lex_unrank_into(uint64_t rank, size_t n, size_t k, std::vector<size_t>& s) {
    const BinomTable& B = binoms();
    uint64_t rev = B.c[n][k] - 1 - rank;   // co-lexicographic index of the complement order
    s.resize(k);
    size_t v = 0;
    for (size_t pos = 0; pos < k; ++pos) {
        // smallest v with C(n-1-v, k-pos) <= rev
        while (B.c[n - 1 - v][k - pos] > rev) ++v;
        s[pos] = v;
        rev -= B.c[n - 1 - v][k - pos];
        ++v;
    }
}

// Runs f(begin, end) over [0, n) in contiguous chunks on the host's cores.
template <class F>
void parallel_chunks(size_t n, F&& f) {
    const size_t hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t threads = std::min(hw, std::max<size_t>(1, n / 16384));
    if (threads <= 1) {
        f(size_t{0}, n);
        return;
    }
    std::vector<std::thread> pool;
    const size_t chunk = (n + threads - 1) / threads;
    for (size_t t = 0; t < threads; ++t) {
        const size_t b = t * chunk, e = std::min(n, b + chunk);
        if (b < e) pool.emplace_back([&f, b, e] { f(b, e); });
    }
    for (auto& th : pool) th.join();
}

}  // namespace

bool is_prime(uint32_t n) {
    if (n <= 1) return false;
    for (uint32_t i = 2; i <= n / i; ++i)
        if (n % i == 0) return false;
    return true;
}

// load_cyclic_instance (cuda/cuprym_cyclic.cu:483-609).
Instance load_instance(const std::string& path) {
    const std::string text = read_file(path);
    const json::Value root = json::parse(text);
    Instance inst;
    const uint64_t genus = root.at("genus").as_u64("genus");
    const uint64_t modulus = root.at("modulus").as_u64("modulus");
    const uint64_t r = root.at("cyclic").at("order").as_u64("cyclic.order");
    if (modulus == 0 || modulus > 65535) throw std::runtime_error("instance modulus must fit uint16_t CUDA storage");
    if (genus < 6 || genus % 2 != 0) throw std::runtime_error("cyclic Prym CUDA path expects an even genus >= 6");
    inst.genus = genus;
    inst.modulus = static_cast<uint32_t>(modulus);
    inst.r = r;
    inst.n = genus - 3;
    inst.m = genus / 2;
    if (r == 0 || inst.m > inst.n) throw std::runtime_error("invalid cyclic Prym dimensions");
    const json::Value& w = root.at("weights");
    inst.weight_v = weight_array(w, "V", r);
    inst.weight_a0 = weight_array(w, "A0", r);
    inst.weight_a1 = weight_array(w, "A1", r);
    if (inst.weight_v.size() != inst.n || inst.weight_a0.size() != inst.genus || inst.weight_a1.size() != inst.n)
        throw std::runtime_error("cyclic weight vector lengths do not match genus metadata");
    const json::Value& mu = root.at("artinian").at("mu");
    const uint64_t mu_n = mu.at("n").as_u64("mu.n"), mu_g = mu.at("g").as_u64("mu.g");
    inst.mu = mod_array(mu, "values", 0, inst.modulus);
    if (mu_n != inst.n || mu_g != inst.genus || inst.mu.size() != inst.n * inst.n * inst.genus)
        throw std::runtime_error("artinian.mu dimensions do not match cyclic genus metadata");
    if (const json::Value* k = root.find("koszul")) {
        try {
            inst.expected_sector_columns = u64_array(*k, "sector_columns");
            inst.expected_sector_rows = u64_array(*k, "sector_rows");
            inst.expected_sector_nnz = u64_array(*k, "sector_nnz");
        } catch (const std::exception&) {
            inst.expected_sector_columns.clear();
            inst.expected_sector_rows.clear();
            inst.expected_sector_nnz.clear();
        }
    }
    if (const json::Value* e = root.find("third_section_elimination")) {
        inst.has_elimination = true;
        const uint64_t wi = e->at("w_V_index").as_u64("w_V_index");
        const uint64_t ww = e->at("w_weight").as_u64("w_weight");
        if (ww >= r) throw std::runtime_error("third_section_elimination scalar metadata is invalid");
        inst.w_index = wi;
        inst.w_weight = static_cast<uint16_t>(ww);
        inst.kernel_weights = weight_array(*e, "kernel_weights", r);
        inst.right_inverse = mod_array(*e, "right_inverse_A0_by_A1", inst.genus * inst.n, inst.modulus);
        inst.kernel_basis = mod_array(*e, "kernel_basis_A0_by_3", inst.genus * inst.kernel_dim(), inst.modulus);
        inst.expected_elim_columns = u64_array(*e, "sector_columns");
        inst.expected_elim_rows = u64_array(*e, "sector_rows");
    }
    validate_elimination(inst);
    return inst;
}

size_t CharMap::max_block() const {
    size_t best = 0;
    for (size_t c = 0; c + 1 < offsets.size(); ++c) best = std::max<size_t>(best, offsets[c + 1] - offsets[c]);
    return best;
}

// build_character_map (cuda/cuprym_cyclic.cu:611-627).
CharMap build_char_map(const std::vector<uint16_t>& weights, size_t r) {
    CharMap map;
    map.offsets.resize(r + 1);
    for (size_t ch = 0; ch < r; ++ch) {
        map.offsets[ch] = checked_u32(map.indices.size(), "character offset");
        for (size_t idx = 0; idx < weights.size(); ++idx)
            if (weights[idx] == ch) map.indices.push_back(static_cast<uint16_t>(idx));
    }
    map.offsets[r] = checked_u32(map.indices.size(), "character offset");
    return map;
}

// build_common_incidences_generic (cuda/cuprym_cyclic.cu:631-727), with the
// subset ranks computed by the lexicographic ranking formula instead of a hash
// map (same ranks: the lexicographic order of itertools.combinations).
Incidence build_incidences(size_t local_n, size_t degree, size_t r, const std::vector<size_t>& original,
                           const std::vector<uint16_t>& local_weights) {
    if (local_n >= 64) throw std::runtime_error("implicit operator supports local_n < 64");
    if (degree == 0 || degree > local_n) throw std::runtime_error("source exterior degree is invalid");
    if (original.size() != local_n || local_weights.size() != local_n)
        throw std::runtime_error("local index metadata has the wrong length");
    Incidence inc;
    inc.local_n = local_n;
    inc.degree = degree;
    const size_t td = degree - 1;
    inc.row_subsets = binom64(local_n, td);
    inc.column_subsets = binom64(local_n, degree);
    inc.row_width = local_n - td;
    inc.column_width = degree;
    inc.row_subset_weights.resize(inc.row_subsets);
    inc.column_subset_weights.resize(inc.column_subsets);
    checked_u32(inc.column_subsets, "column rank");
    checked_u32(inc.row_subsets, "row rank");
    for (size_t li = 0; li < local_n; ++li) checked_u32(original[li], "incidence i");
    inc.row_i.resize(inc.row_subsets * inc.row_width);
    inc.row_col.resize(inc.row_subsets * inc.row_width);
    inc.row_neg.resize(inc.row_subsets * inc.row_width);
    inc.col_i.resize(inc.column_subsets * degree);
    inc.col_row.resize(inc.column_subsets * degree);
    inc.col_neg.resize(inc.column_subsets * degree);

    // (d-1)-subsets T in lexicographic order: for every i not in T, the column
    // subset T u {i} and the sign (-1)^(number of elements of T below i).
    // Chunks of ranks run on the host's cores; each starts from its first
    // subset (unranked) and walks to the next combination.
    parallel_chunks(inc.row_subsets, [&](size_t begin, size_t end) {
        std::vector<size_t> s;
        lex_unrank_into(begin, local_n, td, s);
        for (uint64_t rank = begin; rank < end; ++rank) {
            uint64_t mask = 0;
            size_t wsum = 0;
            for (size_t v : s) {
                mask |= 1ULL << v;
                wsum += local_weights[v];
            }
            inc.row_subset_weights[rank] = static_cast<uint16_t>(wsum % r);
            size_t position = 0, q = rank * inc.row_width;
            for (size_t li = 0; li < local_n; ++li) {
                if (mask & (1ULL << li)) {
                    ++position;
                    continue;
                }
                inc.row_i[q] = static_cast<uint32_t>(original[li]);
                inc.row_col[q] = static_cast<uint32_t>(lex_rank_mask(mask | (1ULL << li), local_n, degree));
                inc.row_neg[q] = static_cast<uint8_t>(position % 2 == 1);
                ++q;
            }
            if (td > 0 && rank + 1 < end) {   // next combination
                size_t i = td;
                while (i > 0 && s[i - 1] == local_n - td + i - 1) --i;
                ++s[i - 1];
                for (size_t j = i; j < td; ++j) s[j] = s[j - 1] + 1;
            }
        }
    });
    // d-subsets S: for every position of S, the row subset S \ {S_pos} and the sign (-1)^pos.
    parallel_chunks(inc.column_subsets, [&](size_t begin, size_t end) {
        std::vector<size_t> c;
        lex_unrank_into(begin, local_n, degree, c);
        for (uint64_t rank = begin; rank < end; ++rank) {
            uint64_t mask = 0;
            size_t wsum = 0;
            for (size_t v : c) {
                mask |= 1ULL << v;
                wsum += local_weights[v];
            }
            inc.column_subset_weights[rank] = static_cast<uint16_t>(wsum % r);
            for (size_t position = 0; position < degree; ++position) {
                const size_t li = c[position], q = rank * degree + position;
                inc.col_i[q] = static_cast<uint32_t>(original[li]);
                inc.col_row[q] = static_cast<uint32_t>(lex_rank_mask(mask & ~(1ULL << li), local_n, td));
                inc.col_neg[q] = static_cast<uint8_t>(position % 2 == 1);
            }
            if (rank + 1 < end) {
                size_t i = degree;
                while (i > 0 && c[i - 1] == local_n - degree + i - 1) --i;
                ++c[i - 1];
                for (size_t j = i; j < degree; ++j) c[j] = c[j - 1] + 1;
            }
        }
    });
    return inc;
}

// build_sector_layout_generic (cuda/cuprym_cyclic.cu:733-790).
SectorLayout build_sector_layout(const Instance& inst, const Incidence& inc, const CharMap& a0, const CharMap& a1,
                                 size_t sector) {
    SectorLayout L;
    L.sector = sector;
    L.row_offsets.resize(inc.row_subsets + 1);
    L.col_offsets.resize(inc.column_subsets + 1);
    for (size_t rr = 0; rr < inc.row_subsets; ++rr) {
        L.row_offsets[rr] = checked_u32(L.row_subset.size(), "row offset");
        const uint32_t ch = sub_mod(sector, inc.row_subset_weights[rr], inst.r);
        for (uint32_t idx = a1.offsets[ch]; idx < a1.offsets[ch + 1]; ++idx) {
            L.row_subset.push_back(static_cast<uint32_t>(rr));
            L.row_beta.push_back(a1.indices[idx]);
        }
    }
    L.row_offsets[inc.row_subsets] = checked_u32(L.row_subset.size(), "row offset");
    for (size_t cr = 0; cr < inc.column_subsets; ++cr) {
        L.col_offsets[cr] = checked_u32(L.col_subset.size(), "column offset");
        const uint32_t ch = sub_mod(sector, inc.column_subset_weights[cr], inst.r);
        for (uint32_t idx = a0.offsets[ch]; idx < a0.offsets[ch + 1]; ++idx) {
            L.col_subset.push_back(static_cast<uint32_t>(cr));
            L.col_a.push_back(a0.indices[idx]);
        }
    }
    L.col_offsets[inc.column_subsets] = checked_u32(L.col_subset.size(), "column offset");
    uint64_t nnz = 0;
    for (size_t row = 0; row < L.row_subset.size(); ++row) {
        const size_t rr = L.row_subset[row];
        const uint32_t beta = L.row_beta[row];
        for (size_t pos = 0; pos < inc.row_width; ++pos) {
            const uint32_t i = inc.row_i[rr * inc.row_width + pos];
            const uint32_t q = sub_mod(inst.weight_a1[beta], inst.weight_v[i], inst.r);
            for (uint32_t idx = a0.offsets[q]; idx < a0.offsets[q + 1]; ++idx)
                if (inst.mu_at(i, beta, a0.indices[idx]) != 0) ++nnz;
        }
    }
    L.nnz = nnz;
    return L;
}

// build_tensor_layout (cuda/cuprym_cyclic.cu:796-819).
TensorLayout build_tensor_layout(const std::vector<uint16_t>& subset_weights, const CharMap& map, size_t r,
                                 size_t sector) {
    TensorLayout L;
    L.offsets.resize(subset_weights.size() + 1);
    for (size_t s = 0; s < subset_weights.size(); ++s) {
        L.offsets[s] = checked_u32(L.subset.size(), "tensor offset");
        const uint32_t ch = sub_mod(sector, subset_weights[s], r);
        for (uint32_t idx = map.offsets[ch]; idx < map.offsets[ch + 1]; ++idx) {
            L.subset.push_back(static_cast<uint32_t>(s));
            L.index.push_back(map.indices[idx]);
        }
    }
    L.offsets[subset_weights.size()] = checked_u32(L.subset.size(), "tensor offset");
    return L;
}

// seeded_sector_value (cuda/cuprym_cyclic.cu:1143-1151).
uint64_t seeded_sector_value(uint64_t seed, size_t sector) {
    uint64_t x = seed ^ (0x9E3779B97F4A7C15ULL + (static_cast<uint64_t>(sector) << 6) + (static_cast<uint64_t>(sector) >> 2));
    x ^= x >> 30;
    x *= 0xBF58476D1CE4E5B9ULL;
    x ^= x >> 27;
    x *= 0x94D049BB133111EBULL;
    x ^= x >> 31;
    return x;
}

uint64_t splitmix64_next(uint64_t& state) {
    uint64_t z = (state += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// generate_random_vector (cuda/matrices.h:44-56): the libstdc++ uniform
// distribution over mt19937_64, drawn in the caller's order.
std::vector<uint32_t> random_vector(size_t size, uint32_t prime, std::mt19937_64& gen, bool nonzero) {
    std::vector<uint32_t> out(size);
    std::uniform_int_distribution<uint64_t> dis(nonzero ? 1 : 0, static_cast<uint64_t>(prime) - 1);
    for (size_t i = 0; i < size; ++i) out[i] = static_cast<uint32_t>(static_cast<uint16_t>(dis(gen)));
    return out;
}

namespace {
uint64_t rowmix_bounded(uint64_t& state, uint64_t bound) {
    if (bound == 0) throw std::runtime_error("rowmix bounded RNG called with zero bound");
    const uint64_t threshold = (0ULL - bound) % bound;
    while (true) {
        const uint64_t v = splitmix64_next(state);
        if (v >= threshold) return v % bound;
    }
}
uint16_t rowmix_nonzero(uint64_t& state, uint32_t prime) {
    if (prime <= 1 || prime > 65535) throw std::runtime_error("rowmix prime must be in 2..65535");
    return static_cast<uint16_t>(1 + rowmix_bounded(state, prime - 1));
}
uint64_t rowmix_realized_seed(uint64_t seed, const std::string& op, size_t sector, size_t rows, uint32_t prime) {
    uint64_t h = kFnvOffset;
    h = fnv_str(h, kRowmixAlgorithm);
    h = fnv_str(h, op);
    h = fnv_u64(h, seed);
    h = fnv_u64(h, sector);
    h = fnv_u64(h, rows);
    h = fnv_u64(h, prime);
    return seeded_sector_value(h, sector);
}
}  // namespace

// generate_rowmix_plan (cuda/cuprym_cyclic.cu:1227-1268).
RowMixPlan generate_rowmix_plan(size_t target_rows, const std::string& op, size_t sector, uint32_t prime,
                                size_t rounds, uint64_t seed) {
    RowMixPlan plan;
    plan.target_rows = target_rows;
    plan.rounds = rounds;
    plan.seed = seed;
    plan.realized_seed = rowmix_realized_seed(seed, op, sector, target_rows, prime);
    plan.round_pairs.resize(rounds);
    if (rounds == 0) return plan;
    std::vector<uint32_t> perm(target_rows);
    for (size_t i = 0; i < target_rows; ++i) perm[i] = checked_u32(i, "rowmix target coordinate");
    uint64_t state = plan.realized_seed;
    const size_t pairs = target_rows / 2;
    for (size_t round = 0; round < rounds; ++round) {
        for (size_t i = target_rows; i > 1; --i) {
            const size_t j = static_cast<size_t>(rowmix_bounded(state, i));
            std::swap(perm[i - 1], perm[j]);
        }
        auto& out = plan.round_pairs[round];
        out.reserve(pairs);
        for (size_t q = 0; q < pairs; ++q) {
            RowMixPair pr;
            pr.first = perm[2 * q];
            pr.second = perm[2 * q + 1];
            pr.a = rowmix_nonzero(state, prime);
            pr.b = rowmix_nonzero(state, prime);
            out.push_back(pr);
        }
    }
    return plan;
}

uint64_t rowmix_plan_hash(const RowMixPlan& plan) {
    uint64_t h = kFnvOffset;
    h = fnv_str(h, kRowmixAlgorithm);
    h = fnv_u64(h, plan.target_rows);
    h = fnv_u64(h, plan.rounds);
    h = fnv_u64(h, plan.seed);
    h = fnv_u64(h, plan.realized_seed);
    for (const auto& round : plan.round_pairs) {
        h = fnv_u64(h, round.size());
        for (const auto& pr : round) {
            h = fnv_u64(h, pr.first);
            h = fnv_u64(h, pr.second);
            h = fnv_u64(h, pr.a);
            h = fnv_u64(h, pr.b);
        }
    }
    return h;
}

uint64_t fnv1a64_vector_hash(const std::vector<uint32_t>& values) {
    uint64_t h = fnv_u64(kFnvOffset, values.size());
    for (uint32_t v : values) h = fnv_u64(h, v);
    return h;
}

std::string hex_u64(uint64_t v) {
    std::ostringstream out;
    out << "0x" << std::hex << std::setw(16) << std::setfill('0') << v;
    return out.str();
}

// deterministic_dense_block (cuda/cuprym_cyclic.cu:1413-1424).
std::vector<uint32_t> deterministic_block(size_t rows, size_t cols, uint32_t prime, uint64_t salt) {
    std::vector<uint32_t> out(rows * cols);
    uint64_t state = salt ^ (0xD6E8FEB86659FD93ULL + rows * 1315423911ULL + cols * 2654435761ULL);
    for (size_t i = 0; i < rows * cols; ++i) out[i] = static_cast<uint32_t>(splitmix64_next(state) % prime);
    return out;
}

namespace {
void rowmix_apply(const RowMixPlan& plan, std::vector<uint32_t>& block, size_t cols, uint32_t prime, bool transpose) {
    auto one = [&](const std::vector<RowMixPair>& round) {
        for (const auto& pr : round)
            for (size_t c = 0; c < cols; ++c) {
                uint64_t x = block[pr.first * cols + c], y = block[pr.second * cols + c];
                uint64_t a = pr.a, b = pr.b, oab = 1 + a * b;
                if (transpose) {
                    block[pr.first * cols + c] = static_cast<uint32_t>((x + b * y) % prime);
                    block[pr.second * cols + c] = static_cast<uint32_t>((a * x + oab * y) % prime);
                } else {
                    block[pr.first * cols + c] = static_cast<uint32_t>((x + a * y) % prime);
                    block[pr.second * cols + c] = static_cast<uint32_t>((b * x + oab * y) % prime);
                }
            }
    };
    if (transpose)
        for (size_t r = plan.round_pairs.size(); r > 0; --r) one(plan.round_pairs[r - 1]);
    else
        for (const auto& round : plan.round_pairs) one(round);
}
}  // namespace

uint32_t dot_mod(const std::vector<uint32_t>& a, const std::vector<uint32_t>& b, uint32_t p) {
    if (a.size() != b.size()) throw std::runtime_error("dense dot input size mismatch");
    uint64_t s = 0;
    for (size_t i = 0; i < a.size(); ++i) {
        s += static_cast<uint64_t>(a[i]) * b[i];
        if (s > (1ULL << 62)) s %= p;
    }
    return static_cast<uint32_t>(s % p);
}

void validate_rowmix_transpose_identity(const RowMixPlan& plan, size_t cols, uint32_t prime) {
    std::vector<uint32_t> x = deterministic_block(plan.target_rows, cols, prime, 0xA11CE001ULL);
    std::vector<uint32_t> y = deterministic_block(plan.target_rows, cols, prime, 0xB0B5EED2ULL);
    std::vector<uint32_t> tx = x, tty = y;
    rowmix_apply(plan, tx, cols, prime, false);
    rowmix_apply(plan, tty, cols, prime, true);
    const uint32_t left = dot_mod(tx, y, prime), right = dot_mod(x, tty, prime);
    if (left != right)
        throw std::runtime_error("rowmix transpose identity failed: <Tx,y>=" + std::to_string(left) +
                                 ", <x,T^t y>=" + std::to_string(right));
}

// P = T^t Dr T with T = T_R ... T_1 (the rounds of generate_rowmix_plan).
namespace {
// T = T_R ... T_1 of a row-mixing plan, row by row: a round pairs disjoint
// rows, so every row has at most W = 2^R entries (columns sorted), and its
// columns (the rows of T^t, rows sorted).
struct RowMixT {
    size_t n = 0, W = 1;
    std::vector<uint32_t> tc, tv;   // row k: columns and values at k * W, tn[k] of them
    std::vector<uint8_t> tn;
    std::vector<uint32_t> cptr, crow, cval;   // column i: rows crow and values cval at cptr[i]..cptr[i+1]
};

RowMixT build_rowmix_t(const RowMixPlan& plan, uint32_t prime) {
    RowMixT t;
    const size_t n = plan.target_rows;
    if (plan.rounds > 6) throw std::runtime_error("at most 6 row-mixing rounds can be folded");
    t.n = n;
    t.W = size_t(1) << plan.rounds;
    const size_t W = t.W;
    auto& tc = t.tc;
    auto& tv = t.tv;
    auto& tn = t.tn;
    tc.resize(n * W);
    tv.resize(n * W);
    tn.assign(n, 1);
    for (size_t i = 0; i < n; ++i) {
        tc[i * W] = static_cast<uint32_t>(i);
        tv[i * W] = 1;
    }
    const uint64_t p = prime;
    // out = cu * row u + cv * row v (sorted merge, zeros dropped); returns the count
    auto combine = [&](size_t u, uint64_t cu, size_t v, uint64_t cv, uint32_t* oc, uint32_t* ov) {
        size_t a = 0, b = 0, k = 0;
        const uint32_t *uc = &tc[u * W], *uv = &tv[u * W], *vc = &tc[v * W], *vv = &tv[v * W];
        while (a < tn[u] || b < tn[v]) {
            uint32_t col;
            uint64_t val = 0;
            if (b >= tn[v] || (a < tn[u] && uc[a] < vc[b])) {
                col = uc[a];
                val = cu * uv[a++] % p;
            } else if (a >= tn[u] || vc[b] < uc[a]) {
                col = vc[b];
                val = cv * vv[b++] % p;
            } else {
                col = uc[a];
                val = (cu * uv[a++] + cv * vv[b++]) % p;
            }
            if (val) {
                oc[k] = col;
                ov[k++] = static_cast<uint32_t>(val);
            }
        }
        return k;
    };
    for (const auto& round : plan.round_pairs) {
        parallel_chunks(round.size(), [&](size_t begin, size_t end) {
            std::vector<uint32_t> fc(W), fv(W), sc(W), sv(W);
            for (size_t q = begin; q < end; ++q) {
                const auto& pr = round[q];
                const uint64_t a = pr.a, b = pr.b, oab = (1 + a * b) % p;
                const size_t nf = combine(pr.first, 1, pr.second, a, fc.data(), fv.data());
                const size_t ns = combine(pr.first, b, pr.second, oab, sc.data(), sv.data());
                std::copy(fc.begin(), fc.begin() + nf, &tc[pr.first * W]);
                std::copy(fv.begin(), fv.begin() + nf, &tv[pr.first * W]);
                std::copy(sc.begin(), sc.begin() + ns, &tc[pr.second * W]);
                std::copy(sv.begin(), sv.begin() + ns, &tv[pr.second * W]);
                tn[pr.first] = static_cast<uint8_t>(nf);
                tn[pr.second] = static_cast<uint8_t>(ns);
            }
        });
    }
    // columns of T: for column i, the rows k with T[k][i] != 0
    std::vector<uint32_t> cptr(n + 1, 0);
    for (size_t k = 0; k < n; ++k)
        for (size_t e = 0; e < tn[k]; ++e) ++cptr[tc[k * W + e] + 1];
    for (size_t i = 0; i < n; ++i) cptr[i + 1] += cptr[i];
    std::vector<uint32_t> crow(cptr[n]), cval(cptr[n]);
    {
        std::vector<uint32_t> fill(cptr.begin(), cptr.end() - 1);
        for (size_t k = 0; k < n; ++k)
            for (size_t e = 0; e < tn[k]; ++e) {
                const uint32_t i = tc[k * W + e];
                crow[fill[i]] = static_cast<uint32_t>(k);
                cval[fill[i]++] = tv[k * W + e];
            }
    }
    t.cptr = std::move(cptr);
    t.crow = std::move(crow);
    t.cval = std::move(cval);
    return t;
}
}  // namespace

Csr composite_target_preconditioner(const RowMixPlan& plan, const std::vector<uint32_t>& dr, uint32_t prime) {
    const size_t n = plan.target_rows;
    if (dr.size() != n) throw std::runtime_error("row preconditioner length does not match the rowmix plan");
    const RowMixT t = build_rowmix_t(plan, prime);
    const size_t W = t.W;
    const uint64_t p = prime;
    const auto& tc = t.tc;
    const auto& tv = t.tv;
    const auto& tn = t.tn;
    const auto& cptr = t.cptr;
    const auto& crow = t.crow;
    const auto& cval = t.cval;
    // P[i][j] = sum_k T[k][i] Dr[k] T[k][j]: row i merges the rows k of column i
    const size_t PW = W * W;
    std::vector<uint32_t> pc(n * PW), pv(n * PW);
    std::vector<uint16_t> pn(n);
    parallel_chunks(n, [&](size_t begin, size_t end) {
        std::vector<std::pair<uint32_t, uint64_t>> acc;
        for (size_t i = begin; i < end; ++i) {
            acc.clear();
            for (uint32_t e = cptr[i]; e < cptr[i + 1]; ++e) {
                const size_t k = crow[e];
                const uint64_t coef = static_cast<uint64_t>(cval[e]) * dr[k] % p;
                for (size_t f = 0; f < tn[k]; ++f) acc.emplace_back(tc[k * W + f], coef * tv[k * W + f] % p);
            }
            std::sort(acc.begin(), acc.end(),
                      [](const auto& x, const auto& y) { return x.first < y.first; });
            size_t cnt = 0;
            for (size_t a = 0; a < acc.size();) {
                uint64_t sum = 0;
                const uint32_t col = acc[a].first;
                for (; a < acc.size() && acc[a].first == col; ++a) sum = (sum + acc[a].second) % p;
                if (sum) {
                    pc[i * PW + cnt] = col;
                    pv[i * PW + cnt++] = static_cast<uint32_t>(sum);
                }
            }
            pn[i] = static_cast<uint16_t>(cnt);
        }
    });
    Csr out;
    out.row_ptr.resize(n + 1);
    size_t total = 0;
    for (size_t i = 0; i < n; ++i) {
        out.row_ptr[i] = checked_u32(total, "preconditioner nnz");
        total += pn[i];
    }
    out.row_ptr[n] = checked_u32(total, "preconditioner nnz");
    out.col.resize(total);
    out.val.resize(total);
    parallel_chunks(n, [&](size_t begin, size_t end) {
        for (size_t i = begin; i < end; ++i) {
            std::copy(&pc[i * PW], &pc[i * PW] + pn[i], &out.col[out.row_ptr[i]]);
            std::copy(&pv[i * PW], &pv[i * PW] + pn[i], &out.val[out.row_ptr[i]]);
        }
    });
    return out;
}

std::string rowmix_label(size_t rounds, uint64_t seed) {
    std::ostringstream out;
    out << "rowmix-r" << rounds << "-s" << seed;
    return out.str();
}

// sector_filename (cuda/cuprym_cyclic.cu:1295-1312).
std::string sector_filename(const std::string& out_dir, const std::string& op, size_t sector, size_t num_v,
                            size_t rowmix_rounds, uint64_t rowmix_seed) {
    std::filesystem::path dir(out_dir.empty() ? "." : out_dir);
    std::filesystem::create_directories(dir);
    std::ostringstream name;
    name << op << "-sector" << std::setw(2) << std::setfill('0') << sector << "-v" << num_v;
    if (rowmix_rounds > 0) name << "-rowmix-r" << rowmix_rounds << "-s" << rowmix_seed;
    name << ".wdm.zst";
    return (dir / name.str()).string();
}

std::string rowmix_sidecar_filename(const std::string& wdm) {
    const std::string suffix = ".wdm.zst";
    if (wdm.size() >= suffix.size() && wdm.compare(wdm.size() - suffix.size(), suffix.size(), suffix) == 0)
        return wdm.substr(0, wdm.size() - suffix.size()) + ".rowmix.json";
    return wdm + ".rowmix.json";
}

void ensure_output_absent(const std::string& wdm) {
    if (std::filesystem::exists(wdm)) throw std::runtime_error("refusing to overwrite existing WDM file " + wdm);
    const std::string side = rowmix_sidecar_filename(wdm);
    if (std::filesystem::exists(side)) throw std::runtime_error("refusing to reuse existing rowmix sidecar " + side);
}

// write_rowmix_sidecar (cuda/cuprym_cyclic.cu:1336-1400): the same keys, order and text.
void write_rowmix_sidecar(const std::string& wdm, const std::string& op, size_t sector, size_t rows, size_t cols,
                          size_t num_v, uint32_t prime, uint64_t random_seed, const RowMixPlan& plan,
                          const std::vector<uint32_t>& row_precond, const std::vector<uint32_t>& col_precond,
                          const std::vector<uint32_t>& initial_block) {
    const std::string side = rowmix_sidecar_filename(wdm);
    const std::string tmp = side + ".tmp";
    std::ofstream out(tmp, std::ios::binary);
    if (!out) throw std::runtime_error("failed to open rowmix sidecar " + tmp);
    out << "{\n";
    out << "  \"type\": \"prym_cyclic_rowmix_sidecar\",\n";
    out << "  \"version\": 1,\n";
    out << "  \"algorithm_version\": \"" << kRowmixAlgorithm << "\",\n";
    out << "  \"wdm_file\": \"" << wdm << "\",\n";
    out << "  \"operator\": \"" << op << "\",\n";
    out << "  \"sector\": " << sector << ",\n";
    out << "  \"rows\": " << rows << ",\n";
    out << "  \"columns\": " << cols << ",\n";
    out << "  \"vector_count\": " << num_v << ",\n";
    out << "  \"prime\": " << prime << ",\n";
    out << "  \"numerical_seed\": " << random_seed << ",\n";
    out << "  \"rowmix\": {\n";
    out << "    \"rounds\": " << plan.rounds << ",\n";
    out << "    \"seed\": " << plan.seed << ",\n";
    out << "    \"realized_seed\": " << plan.realized_seed << ",\n";
    out << "    \"rng\": \"splitmix64-v1\",\n";
    out << "    \"target_rows\": " << plan.target_rows << ",\n";
    out << "    \"pair_count_per_round\": [";
    for (size_t i = 0; i < plan.round_pairs.size(); ++i) out << (i ? ", " : "") << plan.round_pairs[i].size();
    out << "],\n";
    out << "    \"recipe\": \"Starting from realized_seed, for each round reset permutation to the previous round's "
           "final order, run descending Fisher-Yates using splitmix64 rejection-bounded draws, pair consecutive "
           "coordinates, then draw nonzero a,b in F_p by rejection-bounded draws in 1..p-1.\",\n";
    out << "    \"hash_fnv1a64\": \"" << hex_u64(rowmix_plan_hash(plan)) << "\"\n";
    out << "  },\n";
    out << "  \"hashes\": {\n";
    out << "    \"row_preconditioner_fnv1a64\": \"" << hex_u64(fnv1a64_vector_hash(row_precond)) << "\",\n";
    out << "    \"column_preconditioner_fnv1a64\": \"" << hex_u64(fnv1a64_vector_hash(col_precond)) << "\",\n";
    out << "    \"initial_block_fnv1a64\": \"" << hex_u64(fnv1a64_vector_hash(initial_block)) << "\"\n";
    out << "  }\n";
    out << "}\n";
    out.close();
    if (!out) throw std::runtime_error("failed to write rowmix sidecar " + tmp);
    std::filesystem::rename(tmp, side);
}

// The sector assembly of run_eliminated_sector (cuda/cuprym_cyclic.cu:2155-2176)
// with the U basis and incidences of main (:2605-2657).
EliminatedSector assemble_eliminated_sector(const Instance& inst, size_t sector) {
    if (!inst.has_elimination) throw std::runtime_error("instance does not contain third_section_elimination data");
    if (sector >= inst.r) throw std::runtime_error("--sector must be in 0.." + std::to_string(inst.r - 1));
    EliminatedSector es;
    es.sector = sector;
    std::vector<size_t> u_idx;
    std::vector<uint16_t> u_w;
    for (size_t i = 0; i < inst.n; ++i) {
        if (i == inst.w_index) continue;
        u_idx.push_back(i);
        u_w.push_back(inst.weight_v[i]);
    }
    const CharMap a0 = build_char_map(inst.weight_a0, inst.r);
    const CharMap a1 = build_char_map(inst.weight_a1, inst.r);
    const CharMap km = build_char_map(inst.kernel_weights, inst.r);
    es.dm = build_incidences(u_idx.size(), inst.m, inst.r, u_idx, u_w);
    es.d2 = build_incidences(u_idx.size(), inst.m - 1, inst.r, u_idx, u_w);
    es.y_sector = sub_mod(sector, inst.w_weight, inst.r);
    es.dm_layout = build_sector_layout(inst, es.dm, a0, a1, sector);
    es.d2_layout = build_sector_layout(inst, es.d2, a0, a1, es.y_sector);
    es.z_layout = build_tensor_layout(es.dm.row_subset_weights, km, inst.r, es.y_sector);
    es.x_cols = es.dm_layout.col_subset.size();
    es.t_rows = es.dm_layout.row_subset.size();
    es.y_rows = es.d2_layout.col_subset.size();
    es.z_cols = es.z_layout.subset.size();
    es.target_rows = es.d2_layout.row_subset.size();
    es.dm_nnz = es.dm_layout.nnz;
    es.d2_nnz = es.d2_layout.nnz;
    // validate_eliminated_sector_against_fixture (cuda/cuprym_cyclic.cu:1124-1141)
    if (!inst.expected_elim_columns.empty() && sector < inst.expected_elim_columns.size() &&
        inst.expected_elim_columns[sector] != es.total_cols())
        throw std::runtime_error("eliminated sector column count does not match fixture metadata");
    if (!inst.expected_elim_rows.empty() && sector < inst.expected_elim_rows.size() &&
        inst.expected_elim_rows[sector] != es.target_rows)
        throw std::runtime_error("eliminated sector row count does not match fixture metadata");
    return es;
}

// A row order in which row-mixing partners sit next to each other.  Every
// round pairs disjoint rows, so each row has at most one partner a round; with
// two rounds the partner graph is a set of paths and cycles that alternate
// between the rounds.  Walking each path (from an end) and then each cycle
// puts both partners of a row beside it, so a row of T^t Dr T (its rows
// within two partner steps on either side) lies within seven consecutive
// positions.  Returns pos[row].
std::vector<uint32_t> rowmix_locality_order(const RowMixPlan& plan) {
    const size_t n = plan.target_rows, R = plan.rounds;
    std::vector<uint32_t> partner(n * std::max<size_t>(R, 1), UINT32_MAX);
    for (size_t r = 0; r < R; ++r)
        for (const auto& pr : plan.round_pairs[r]) {
            partner[pr.first * R + r] = pr.second;
            partner[pr.second * R + r] = pr.first;
        }
    std::vector<uint32_t> pos(n, UINT32_MAX);
    uint32_t next = 0;
    auto walk = [&](size_t v) {
        size_t cur = v;
        while (cur != SIZE_MAX) {
            pos[cur] = next++;
            size_t nb = SIZE_MAX;
            for (size_t r = 0; r < R && nb == SIZE_MAX; ++r) {
                const uint32_t w = partner[cur * R + r];
                if (w != UINT32_MAX && pos[w] == UINT32_MAX) nb = w;
            }
            cur = nb;
        }
    };
    for (size_t v = 0; v < n; ++v) {   // path ends (fewer than R partners) first
        if (pos[v] != UINT32_MAX) continue;
        size_t degree = 0;
        for (size_t r = 0; r < R; ++r) degree += partner[v * R + r] != UINT32_MAX;
        if (degree < R) walk(v);
    }
    for (size_t v = 0; v < n; ++v)   // then the cycles
        if (pos[v] == UINT32_MAX) walk(v);
    return pos;
}

// Subset-major gather tables (the device side is bw_cyclic_subset.cu).
std::string build_subset_tables(const Instance& inst, const EliminatedSector& es, const Csr& precond,
                                const std::vector<uint32_t>& u_pos, SubsetTables& out) {
    out = SubsetTables{};
    const CharMap a0 = build_char_map(inst.weight_a0, inst.r);
    const CharMap a1 = build_char_map(inst.weight_a1, inst.r);
    const CharMap km = build_char_map(inst.kernel_weights, inst.r);
    if (a0.max_block() > 2 || a1.max_block() > 2 || km.max_block() > 2) return "a character block has more than two rows";
    if (inst.n > 32) return "more than 32 generators";
    if (inst.r > 64) return "cyclic order above 64";
    if (inst.modulus >= (1u << 15)) return "prime above 2^15 (balanced residues must fit int16)";
    const Incidence& dm = es.dm;
    const Incidence& d2 = es.d2;
    const size_t n1 = dm.row_subsets, n2 = d2.row_subsets, n0 = dm.column_subsets;
    const uint64_t limit = 1ull << 26;
    if (n0 >= limit || n1 >= limit || n2 >= limit || es.total_cols() >= limit || es.target_rows >= limit)
        return "2^26 subsets or rows or more";
    if (d2.column_subsets != n1) return "inconsistent subset counts";
    if (precond.row_ptr.size() != es.target_rows + 1) return "preconditioner size does not match the sector";
    if (u_pos.size() != es.target_rows) return "u order size does not match the sector";
    out.m1.resize(n1);
    out.m2.resize(n2);
    out.m0.resize(n0);
    for (size_t s = 0; s < n1; ++s)
        out.m1[s] = es.z_layout.offsets[s] | (sub_mod(es.sector, dm.row_subset_weights[s], inst.r) << 26);
    for (size_t s = 0; s < n2; ++s)
        out.m2[s] = es.d2_layout.row_offsets[s] | (sub_mod(es.y_sector, d2.row_subset_weights[s], inst.r) << 26);
    for (size_t s = 0; s < n0; ++s)
        out.m0[s] = es.dm_layout.col_offsets[s] | (sub_mod(es.sector, dm.column_subset_weights[s], inst.r) << 26);
    // incidence words, transposed to [position][subset]
    const uint32_t n = static_cast<uint32_t>(inst.n);
    auto fill = [n](std::vector<uint32_t>& dst, size_t subsets, size_t width, const std::vector<uint32_t>& nb,
                   const std::vector<uint32_t>& idx, const std::vector<uint8_t>& neg) {
        dst.resize(subsets * width);
        parallel_chunks(subsets, [&](size_t b, size_t e) {
            for (size_t s = b; s < e; ++s)
                for (size_t pos = 0; pos < width; ++pos) {
                    const size_t q = s * width + pos;
                    // coefficient code: sign * n + generator (six bits, n <= 32)
                    dst[pos * subsets + s] = nb[q] | ((idx[q] + (neg[q] ? n : 0u)) << 26);
                }
        });
    };
    fill(out.inc_dmf, n1, dm.row_width, dm.row_col, dm.row_i, dm.row_neg);
    fill(out.inc_d2f, n2, d2.row_width, d2.row_col, d2.row_i, d2.row_neg);
    fill(out.inc_d2t, n1, d2.column_width, d2.col_row, d2.col_i, d2.col_neg);
    fill(out.inc_dmt, n0, dm.column_width, dm.col_row, dm.col_i, dm.col_neg);
    // padded preconditioner: compact row -> padded slot
    std::vector<uint32_t> slot(es.target_rows);
    for (size_t s = 0; s < n2; ++s)
        for (uint32_t q = es.d2_layout.row_offsets[s]; q < es.d2_layout.row_offsets[s + 1]; ++q)
            slot[q] = static_cast<uint32_t>(2 * s + (q - es.d2_layout.row_offsets[s]));
    std::vector<uint32_t> compact_of(2 * n2, UINT32_MAX);
    for (size_t q = 0; q < es.target_rows; ++q) compact_of[slot[q]] = static_cast<uint32_t>(q);
    const int32_t p = static_cast<int32_t>(inst.modulus), half = (p - 1) / 2;
    size_t widest = 1;
    for (size_t q = 0; q < es.target_rows; ++q)
        widest = std::max<size_t>(widest, precond.row_ptr[q + 1] - precond.row_ptr[q]);
    if (widest > 64) return "preconditioner above 64 entries a row";
    out.ell = (widest + 3) / 4 * 4;
    const size_t rows = 2 * n2;
    if (rows * out.ell >= (1ull << 32)) return "preconditioner above 2^32 slots";
    out.e_col.assign(rows * out.ell, 0u);
    out.e_val.assign(rows * out.ell, int16_t{0});
    parallel_chunks(rows, [&](size_t b, size_t e) {
        for (size_t pr = b; pr < e; ++pr) {
            const uint32_t q = compact_of[pr];
            if (q == UINT32_MAX) continue;
            size_t k = 0;
            for (uint32_t x = precond.row_ptr[q]; x < precond.row_ptr[q + 1]; ++x, ++k) {
                out.e_col[k * rows + pr] = u_pos[precond.col[x]];
                int32_t v = static_cast<int32_t>(precond.val[x] % inst.modulus);
                if (v > half) v -= p;
                out.e_val[k * rows + pr] = static_cast<int16_t>(v);
            }
        }
    });
    return "";
}

// ----- deformation inputs (cuda/cuprym_deformation.cu:253-473): text scanning
namespace {

// Position just past the colon that follows the first quoted occurrence of `key`.
size_t scan_key(const std::string& text, const std::string& key) {
    const std::string needle = "\"" + key + "\"";
    const size_t at = text.find(needle);
    if (at == std::string::npos) throw std::runtime_error("missing JSON key '" + key + "'");
    const size_t colon = text.find(':', at + needle.size());
    if (colon == std::string::npos) throw std::runtime_error("missing ':' after JSON key '" + key + "'");
    return colon + 1;
}

uint64_t scan_u64(const std::string& text, const std::string& key) {
    size_t pos = scan_key(text, key);
    while (pos < text.size() && std::isspace(static_cast<unsigned char>(text[pos]))) ++pos;
    if (pos >= text.size() || !std::isdigit(static_cast<unsigned char>(text[pos])))
        throw std::runtime_error("expected unsigned integer for " + key);
    uint64_t v = 0;
    for (; pos < text.size() && std::isdigit(static_cast<unsigned char>(text[pos])); ++pos) {
        const uint64_t d = static_cast<uint64_t>(text[pos] - '0');
        if (v > (std::numeric_limits<uint64_t>::max() - d) / 10) throw std::runtime_error(key + " overflows u64");
        v = v * 10 + d;
    }
    return v;
}

// Every unsigned digit run inside the bracketed array that follows `key`.
std::vector<uint64_t> scan_u64_array(const std::string& text, const std::string& key, const std::string& label) {
    const size_t colon = scan_key(text, key);
    const size_t open = text.find('[', colon);
    if (open == std::string::npos) throw std::runtime_error("JSON key '" + key + "' is not an array");
    size_t depth = 0, close = std::string::npos;
    bool in_str = false, esc = false;
    for (size_t q = open; q < text.size() && close == std::string::npos; ++q) {
        const char ch = text[q];
        if (in_str) {
            if (esc) esc = false;
            else if (ch == '\\') esc = true;
            else if (ch == '"') in_str = false;
        } else if (ch == '"') {
            in_str = true;
        } else if (ch == '[') {
            ++depth;
        } else if (ch == ']' && --depth == 0) {
            close = q;
        }
    }
    if (close == std::string::npos) throw std::runtime_error("failed to find matching JSON delimiter");
    std::vector<uint64_t> out;
    for (size_t q = open; q <= close;) {
        if (!std::isdigit(static_cast<unsigned char>(text[q]))) {
            ++q;
            continue;
        }
        uint64_t v = 0;
        for (; q <= close && std::isdigit(static_cast<unsigned char>(text[q])); ++q) {
            const uint64_t d = static_cast<uint64_t>(text[q] - '0');
            if (v > (std::numeric_limits<uint64_t>::max() - d) / 10)
                throw std::runtime_error(label + " entry overflows u64");
            v = v * 10 + d;
        }
        out.push_back(v);
    }
    return out;
}

}  // namespace

DenseBlockFile load_dense_block_file(const std::string& path, uint32_t expected_prime) {
    const std::string text = read_file(path);
    const uint64_t rows = scan_u64(text, "rows"), cols = scan_u64(text, "columns"), prime = scan_u64(text, "prime");
    if (prime > std::numeric_limits<uint32_t>::max()) throw std::runtime_error("dense block scalar metadata is too large");
    DenseBlockFile b;
    b.rows = static_cast<size_t>(rows);
    b.columns = static_cast<size_t>(cols);
    b.prime = static_cast<uint32_t>(prime);
    if (b.prime != expected_prime) throw std::runtime_error("dense block prime does not match instance modulus");
    if (cols != 0 && rows > std::numeric_limits<size_t>::max() / cols)
        throw std::runtime_error("dense block value count overflows size_t");
    const std::vector<uint64_t> raw = scan_u64_array(text, "values", "values");
    if (raw.size() != b.rows * b.columns)
        throw std::runtime_error("values has " + std::to_string(raw.size()) + " entries; expected " +
                                 std::to_string(b.rows * b.columns));
    b.values.reserve(raw.size());
    for (uint64_t v : raw) {
        if (v >= expected_prime) throw std::runtime_error("values entry is not reduced modulo the instance modulus");
        if (v > 65535) throw std::runtime_error("values entry does not fit uint16_t CUDA storage");
        b.values.push_back(static_cast<uint32_t>(v));
    }
    return b;
}

std::vector<uint32_t> load_drop_columns_file(const std::string& path, size_t expected_count, size_t base_columns) {
    const std::string text = read_file(path);
    const std::vector<uint64_t> raw = scan_u64_array(text, "indices", "drop-column indices");
    if (raw.size() != expected_count) throw std::runtime_error("drop-column file has the wrong number of indices");
    std::vector<uint32_t> out;
    for (uint64_t v : raw) {
        if (v >= base_columns || v > std::numeric_limits<uint32_t>::max())
            throw std::runtime_error("drop-column index is outside the base column range");
        out.push_back(static_cast<uint32_t>(v));
    }
    std::sort(out.begin(), out.end());
    for (size_t i = 1; i < out.size(); ++i)
        if (out[i] == out[i - 1]) throw std::runtime_error("drop-column indices must be distinct");
    return out;
}

}  // namespace cyclic
}  // namespace bw
