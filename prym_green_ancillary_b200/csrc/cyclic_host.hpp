// Host-side assembly of the eliminated cyclic Koszul operator (paper mode):
// instance loading and validation, character maps, subset incidences, sector
// layouts, the seeded preconditioners / initial block, the paired-SL2 row
// mixing plan and its sidecar, and output names.  Follows the reference's
// cuda/cuprym_cyclic.cu:39-1400 (citations per function in lib_cyclic_host.cpp).
#pragma once

#include <cstddef>
#include <cstdint>
#include <random>
#include <string>
#include <vector>

namespace bw {
namespace cyclic {

constexpr const char* kRowmixAlgorithm = "paired-sl2-target-v1";

struct Instance {
    size_t genus = 0, n = 0, m = 0, r = 0;
    uint32_t modulus = 0;
    std::vector<uint32_t> mu;                  // ((i*n)+beta)*g + a
    std::vector<uint16_t> weight_v, weight_a0, weight_a1;
    std::vector<uint64_t> expected_sector_columns, expected_sector_rows, expected_sector_nnz;
    bool has_elimination = false;
    size_t w_index = 0;
    uint16_t w_weight = 0;
    std::vector<uint32_t> right_inverse;       // g x n   [a][beta]
    std::vector<uint32_t> kernel_basis;        // g x kdim [a][kappa]
    std::vector<uint16_t> kernel_weights;
    std::vector<uint64_t> expected_elim_columns, expected_elim_rows;

    uint32_t mu_at(size_t i, size_t beta, size_t a) const { return mu[(i * n + beta) * genus + a]; }
    size_t kernel_dim() const { return kernel_weights.size(); }
};

Instance load_instance(const std::string& path);
bool is_prime(uint32_t n);

struct CharMap {
    std::vector<uint32_t> offsets;   // r + 1
    std::vector<uint16_t> indices;
    size_t block(size_t ch) const { return offsets[ch + 1] - offsets[ch]; }
    size_t max_block() const;
};
CharMap build_char_map(const std::vector<uint16_t>& weights, size_t r);

// Koszul incidences of D: Lambda^d(U) (x) A0 -> Lambda^(d-1)(U) (x) A1 on a
// local basis U (original indices kept for mu lookups).
struct Incidence {
    size_t local_n = 0, degree = 0;
    size_t row_subsets = 0, column_subsets = 0, row_width = 0, column_width = 0;
    std::vector<uint16_t> row_subset_weights, column_subset_weights;
    // per row subset, row_width entries (i not in T): original i, column subset rank, negative
    std::vector<uint32_t> row_i, row_col;
    std::vector<uint8_t> row_neg;
    // per column subset, column_width entries (i in S): original i, row subset rank, negative
    std::vector<uint32_t> col_i, col_row;
    std::vector<uint8_t> col_neg;
};
Incidence build_incidences(size_t local_n, size_t degree, size_t r, const std::vector<size_t>& original,
                           const std::vector<uint16_t>& local_weights);

// Rows (subset, beta in A1) and columns (subset, a in A0) of one sector.
struct SectorLayout {
    size_t sector = 0;
    std::vector<uint32_t> row_offsets, row_subset;   // row_offsets: per row subset (+1)
    std::vector<uint16_t> row_beta;
    std::vector<uint32_t> col_offsets, col_subset;
    std::vector<uint16_t> col_a;
    uint64_t nnz = 0;
};
SectorLayout build_sector_layout(const Instance& inst, const Incidence& inc, const CharMap& a0, const CharMap& a1,
                                 size_t sector);

struct TensorLayout {
    std::vector<uint32_t> offsets, subset;
    std::vector<uint16_t> index;
};
TensorLayout build_tensor_layout(const std::vector<uint16_t>& subset_weights, const CharMap& map, size_t r,
                                 size_t sector);

// ----- seeded data and row mixing
uint64_t seeded_sector_value(uint64_t seed, size_t sector);
uint64_t splitmix64_next(uint64_t& state);
std::vector<uint32_t> random_vector(size_t size, uint32_t prime, std::mt19937_64& gen, bool nonzero);

struct RowMixPair {
    uint32_t first, second;
    uint16_t a, b;
};
struct RowMixPlan {
    size_t target_rows = 0, rounds = 0;
    uint64_t seed = 0, realized_seed = 0;
    std::vector<std::vector<RowMixPair>> round_pairs;
};
RowMixPlan generate_rowmix_plan(size_t target_rows, const std::string& op, size_t sector, uint32_t prime,
                                size_t rounds, uint64_t seed);
uint64_t rowmix_plan_hash(const RowMixPlan& plan);
uint64_t fnv1a64_vector_hash(const std::vector<uint32_t>& values);
std::string hex_u64(uint64_t v);

std::vector<uint32_t> deterministic_block(size_t rows, size_t cols, uint32_t prime, uint64_t salt);
uint32_t dot_mod(const std::vector<uint32_t>& a, const std::vector<uint32_t>& b, uint32_t p);

// <T x, y> == <x, T^t y> on deterministic blocks (cuda/cuprym_cyclic.cu:1568-1589).
void validate_rowmix_transpose_identity(const RowMixPlan& plan, size_t cols, uint32_t prime);

// Composite target preconditioner P = T^t Dr T (T = T_R ... T_1) as CSR, exact
// mod p; at most 16 entries per row for two rounds.
struct Csr {
    std::vector<uint32_t> row_ptr, col;
    std::vector<uint32_t> val;   // canonical residues
};
Csr composite_target_preconditioner(const RowMixPlan& plan, const std::vector<uint32_t>& row_precond,
                                    uint32_t prime);


// ----- file names and sidecar (cuda/cuprym_cyclic.cu:1289-1400)
std::string rowmix_label(size_t rounds, uint64_t seed);
std::string sector_filename(const std::string& out_dir, const std::string& op, size_t sector, size_t num_v,
                            size_t rowmix_rounds, uint64_t rowmix_seed);
std::string rowmix_sidecar_filename(const std::string& wdm_filename);
void ensure_output_absent(const std::string& wdm_filename);
void write_rowmix_sidecar(const std::string& wdm_filename, const std::string& op, size_t sector, size_t rows,
                          size_t cols, size_t num_v, uint32_t prime, uint64_t random_seed, const RowMixPlan& plan,
                          const std::vector<uint32_t>& row_precond, const std::vector<uint32_t>& col_precond,
                          const std::vector<uint32_t>& initial_block);

// ----- the assembled eliminated sector (everything the device operator needs)
struct EliminatedSector {
    size_t sector = 0, y_sector = 0;
    size_t x_cols = 0, z_cols = 0, t_rows = 0, y_rows = 0, target_rows = 0;
    Incidence dm, d2;
    SectorLayout dm_layout, d2_layout;
    TensorLayout z_layout;
    uint64_t dm_nnz = 0, d2_nnz = 0;
    size_t total_cols() const { return x_cols + z_cols; }
};
EliminatedSector assemble_eliminated_sector(const Instance& inst, size_t sector);

// ----- subset-major tables of the four Koszul gathers (device layout)
// Internal vectors hold every subset's block in two row slots (2 s, 2 s + 1),
// so a neighbour block is found from its subset rank alone.  One entry per
// subset of each degree, and one incidence word per (position, subset) laid
// out [position][subset] so that consecutive subsets read consecutive words.
// An incidence word is the neighbour subset's rank | (i + n * (sign
// negative)) << 26; a subset word is the first compact row of one of its
// blocks | its character << 26.
struct SubsetTables {
    std::vector<uint32_t> m1;   // (m-1)-subsets: z block (compact) | t character
    std::vector<uint32_t> m2;   // (m-2)-subsets: u block (compact) | u character
    std::vector<uint32_t> m0;   // m-subsets: x block (compact) | x character
    // D_m (row subsets, neighbours T u i), D_(m-1) (neighbours T u i),
    // D_(m-1)^t (neighbours S \ j), D_m^t (neighbours S \ j)
    std::vector<uint32_t> inc_dmf, inc_d2f, inc_d2t, inc_dmt;
    // the folded target preconditioner in ELL form: rows are the padded u
    // slots (compact row u_off(s) + q is 2 s + q; they write u2), columns are
    // positions of u in the row-mixing locality order; `ell` slots a row (a
    // multiple of four), laid out [slot][row]; empty slots and padding rows
    // hold column 0 with value 0; balanced values
    size_t ell = 0;
    std::vector<uint32_t> e_col;
    std::vector<int16_t> e_val;
};
// Empty string: the tables are built.  Otherwise the reason this sector does
// not fit the packed format (a character block above two rows, an index or
// rank beyond its field), and `out` is left empty.  `precond` is the folded
// target preconditioner over the compact target rows; its columns index u in
// the order u_pos (compact row -> position).
std::string build_subset_tables(const Instance& inst, const EliminatedSector& es, const Csr& precond,
                                const std::vector<uint32_t>& u_pos, SubsetTables& out);
// Row order with row-mixing partners adjacent (pos[row]); see lib_cyclic_host.cpp.
std::vector<uint32_t> rowmix_locality_order(const RowMixPlan& plan);

// ----- deformation inputs (cuda/cuprym_deformation.cu:426-473)
// Both files are read the way the reference reads them: a key is its first
// quoted occurrence anywhere in the text, a scalar is the unsigned digit run
// after the colon, and an array is every unsigned digit run between its
// brackets (nested arrays flatten, signs are not read).
struct DenseBlockFile {
    size_t rows = 0, columns = 0;
    uint32_t prime = 0;
    std::vector<uint32_t> values;   // rows x columns, row-major, reduced mod prime
};
DenseBlockFile load_dense_block_file(const std::string& path, uint32_t expected_prime);
// `expected_count` distinct base-column indices below `base_columns`, sorted ascending.
std::vector<uint32_t> load_drop_columns_file(const std::string& path, size_t expected_count, size_t base_columns);

}  // namespace cyclic
}  // namespace bw
