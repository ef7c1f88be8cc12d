// Paper-mode (eliminated cyclic operator) engine context.
#pragma once

#include "bw_common.cuh"
#include "cyclic_host.hpp"
#include "../../include/bw_engine.h"

#include <cstdlib>
#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace bw {

// Device view of one eliminated sector (all pointers device, read-only).
struct ElimDev {
    Mod mod;
    int n, g, kdim;
    uint64_t x_cols, z_cols, t_rows, y_rows, n_r;
    uint32_t dm_row_width, dm_col_width, d2_row_width, d2_col_width;
    // D_m: rows t = (S, beta) over (m-1)-subsets, columns x = (S', a) over m-subsets
    const uint32_t *t_off, *t_sub, *x_off, *x_sub;
    const uint16_t *t_beta, *x_a;
    const uint32_t *dm_row_inc, *dm_col_inc;   // packed: subset | i << 26 | negative << 31
    // D_(m-1): columns y = (S, a) over (m-1)-subsets, rows u = (S2, beta) over (m-2)-subsets
    const uint32_t *y_off, *y_sub, *u_off, *u_sub;
    const uint16_t *y_a, *u_beta;
    const uint32_t *d2_row_inc, *d2_col_inc;
    // z = (S, kappa) over (m-1)-subsets
    const uint32_t *z_off, *z_sub;
    const uint16_t* z_k;
    // coefficient lists: local index << 16 | balanced mu (int16)
    const uint32_t *fl_off, *tl_off;
    const int32_t *fl, *tl;
    const int32_t *R, *Bk;   // g x n, g x kdim (balanced)
    // Deformation variants (cuda/cuprym_deformation.cu:2554-3066): the source
    // is the base columns with drop0 / drop1 removed (replacement) followed by
    // n_extra dense columns; F = [F0 | dense_sign * dense].
    uint64_t base_cols, kept_cols;
    long long drop0, drop1;       // dropped base columns, -1 when none (drop0 < drop1)
    int n_extra, dense_sign;      // 0 / 0 for the eliminated operator
    const int32_t* dense;         // n_r x n_extra balanced, row-major
};

// Device view of the subset-major operator (bw_cyclic_subset.cu): one thread
// per subset computes every row of that subset's block; internal vectors are
// int16 with two row slots per subset.  The small tables (signed coefficients,
// R, B, character maps) are staged in shared memory from one blob per
// direction with the layout below (int32 words):
//   coef [2 n codes][r] x int4  (own rows x neighbour slots; code = sign * n + generator)
//   R [g][n], B [g][kdim], a0 offsets [r+1], a0 indices [g], a1 offsets [r+1],
//   a1 indices [n], kernel-weight offsets [r+1], indices [kdim], ych [r]
//   (ych[c] = y character of an (m-1)-subset whose t character is c).
struct SubsetDev {
    Mod mod;
    int n, g, kdim, r;
    uint32_t n1, n2, n0;                   // (m-1)-, (m-2)- and m-subsets
    uint32_t w_dmf, w_d2f, w_d2t, w_dmt;   // incidences per subset of each gather
    const uint32_t *m1, *m2, *m0;          // subset words: compact block row | character << 26
    const uint32_t *inc_dmf, *inc_d2f, *inc_d2t, *inc_dmt;
    const uint32_t* u_pos;                 // compact u row -> its position in u (row-mixing locality order)
    const uint32_t* e_col;                 // folded target preconditioner, ELL (rows: padded u2 slots; columns: u positions)
    const int16_t* e_val;
    uint32_t ell;                          // slots a row (a multiple of four)
    const int32_t *blob_f, *blob_t;
    int blob_words;
    int o_R, o_B, o_a0off, o_a0idx, o_a1off, o_a1idx, o_koff, o_kidx, o_ych;
    uint64_t x_cols, z_cols, kept_cols;
    long long drop0, drop1;
    int n_extra, dense_sign;
    const int32_t* dense;
};

// Preconditioners, initial block and row-mixing recipe of an existing WDM file
// (kernel-vector recovery reopens the operator of the sequence it recovers from).
struct CyclicSource {
    std::vector<uint32_t> row_precond, col_precond, initial_block;
    size_t rowmix_rounds = 0;
    uint64_t rowmix_seed = 0;
};

// Inputs of the augmented / replacement operators: the dense block JSON and,
// for replacement, the two dropped base columns.
struct DeformInputs {
    std::string dense_path, drop_path;
    bool recovery = false;   // word refusals as the recovery stage does
};

struct CyclicCtx {
    int device = 0, sms = 0;
    bool host_only = false;
    uint32_t p = 0;
    Mod mod{};
    std::string op = "eliminated";
    size_t num_v = 4;
    uint64_t seed = 1;
    cyclic::Instance inst;
    cyclic::EliminatedSector es;
    std::vector<uint32_t> row_precond, col_precond, initial_block;
    cyclic::RowMixPlan plan;
    cyclic::Csr precond;
    // source columns: base_cols = x + z; op_cols = the operator's (the vectors' rows)
    size_t base_cols = 0, op_cols = 0, kept_cols = 0;
    std::vector<uint32_t> drop;
    cyclic::DenseBlockFile dense;

    cudaStream_t stream = nullptr;
    std::vector<void*> allocations;
    uint64_t device_bytes = 0, launches = 0, graph_kernels = 0;
    ElimDev E{};
    int32_t* d_dc = nullptr;
    uint32_t *d_p_ptr = nullptr, *d_p_col = nullptr;
    int32_t* d_p_val = nullptr;
    int32_t *d_b = nullptr, *d_d = nullptr, *d_xs = nullptr, *d_y = nullptr, *d_h = nullptr, *d_u = nullptr,
            *d_u2 = nullptr, *d_t = nullptr;
    bool small = false;          // int32 accumulation is exact for this sector
    bool subset_path = false;    // the subset-major gathers run (bw_cyclic_subset.cu)
    std::string subset_reason;   // why not, when they do not
    bool stream_tables = false;  // its tables exceed half the L2: read them evict-first
    // The round's kernels start while the kernel before them finishes
    // (programmatic dependent launch; BW_CYCLIC_PDL=0 turns it off).
    bool pdl = true;
    SubsetDev S{};
    uint4 *d_xs16 = nullptr, *d_y16 = nullptr, *d_t16 = nullptr, *d_u16 = nullptr, *d_u2_16 = nullptr;
    int32_t* d_zs = nullptr;     // compact z rows and extra columns of the scaled source
    // The buffer X for which d_xs16 / d_zs hold d_dc (.) X (nullptr: none):
    // apply_square's backward kernels write the next application's source
    // from its output, so a sequence runs the source kernel only once.  Any
    // other write to X clears it (to_balanced, the compact entry points).
    const int32_t* xs_for = nullptr;
    uint64_t max_terms = 0;      // most products summed into one output by any kernel
    uint32_t* d_canon = nullptr;
    unsigned gram_grid = 1, dense_grid = 1;
    int32_t* d_dpart = nullptr;           // dense-transpose partials and counter
    unsigned int* d_dcounter = nullptr;
    int32_t* d_partials = nullptr;
    unsigned int* d_counter = nullptr;
    unsigned long long* d_seq_index = nullptr;
    uint32_t* d_seq = nullptr;
    size_t seq_alloc = 0, seq_capacity = 0, seq_len = 0;
    cudaGraphExec_t graphs[1] = {nullptr};
    // validation path (explicit rowmix rounds)
    uint32_t* d_pairs = nullptr;
    int32_t* d_dr = nullptr;
    std::vector<size_t> pair_offsets;

    static CyclicCtx* open(const std::string& instance_path, const std::string& op, size_t sector, size_t num_v,
                           uint64_t seed, size_t rowmix_rounds, uint64_t rowmix_seed, int dev,
                           const CyclicSource* src = nullptr, const DeformInputs* deform = nullptr);
    ~CyclicCtx();

    template <class T>
    T* upload(const std::vector<T>& host);
    template <class T>
    T* alloc(size_t count);
    unsigned grid_for(size_t rows) const;
    uint32_t* scratch_canonical();

    // Launches a kernel of 256-thread CTAs on the context's stream, as a
    // programmatic dependent launch when `pdl` is set (the kernel must call
    // cyc::pdl_wait() before touching data of the kernels before it).
    template <class... P, class... A>
    void launch_pdl(void (*kernel)(P...), unsigned grid, size_t smem, A&&... args) {
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(256);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = stream;
        cudaLaunchAttribute attr{};
        attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr.val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = &attr;
        cfg.numAttrs = pdl ? 1 : 0;
        BW_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...));
    }

    void to_balanced(const uint32_t* in, int32_t* out, size_t count);
    void to_canonical(const int32_t* in, uint32_t* out, size_t count);
    void forward(const int32_t* in, int32_t* u, bool precondition);
    // subset-major path (bw_cyclic_subset.cu): in -> d_u16, d_u16 -> d_u2_16, d_u2_16 -> out
    void setup_subset_path();
    void subset_source16(const int32_t* in, const int32_t* dc);   // d_xs16 / d_zs = dc (.) in
    void subset_forward16();                                        // d_xs16 / d_zs -> d_u16
    void subset_precondition16();
    void subset_backward16(const int32_t* dc, int32_t* out, bool next_source);
    void subset_pack_u(const int32_t* u32, uint4* u16);       // compact -> padded (u2)
    void subset_unpack_u(const uint4* u16, int32_t* u32);
    void subset_u_to_walk(const int32_t* u32);                 // compact -> d_u16 in locality order
    void subset_u_from_walk(int32_t* u32);
    void target_precondition(const int32_t* u, int32_t* u2);
    void backward(const int32_t* u2, int32_t* out, bool precondition);
    void apply_square(const int32_t* in, int32_t* out);
    void gram(const int32_t* a1, const int32_t* c1, const int32_t* a2, const int32_t* c2, int count);
    void round();
    void generate(size_t nlen_target, float* device_ms = nullptr);
    void download_state(std::vector<uint32_t>& current, std::vector<uint32_t>& packed);
    void apply_host(int what, const uint32_t* in, uint32_t* out);
    // kernel-vector recovery (bw_cyclic_recover.cu)
    struct Recovery;
    void recover(const std::vector<uint32_t>& generators, size_t generator_count, std::vector<uint32_t>& candidates,
                 std::vector<uint32_t>& product, long long& runtime_ms);
    void require_device() const {
        if (host_only) throw Error("this context was opened host-only (device < 0)", 3);
    }
};

}  // namespace bw

namespace bw {
// --validate-rowmix self-check of an open context (cuda/cuprym_cyclic.cu:1970-2132).
void validate_ctx(CyclicCtx& c, uint32_t columns);
}  // namespace bw
