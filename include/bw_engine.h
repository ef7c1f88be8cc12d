/*
 * C ABI of the B200 block-Wiedemann sequence engine over GF(p).
 *
 * Plain C types only (pointers, sizes, integers).  Every function returns 0 on
 * success and a nonzero status otherwise: 1 = invalid argument (a null
 * pointer, or a size or value outside an entry point's documented range) or
 * host error (files, parsing); 2 = CUDA error, including a tensor-core kernel
 * that gave up a bounded wait; 3 = failed precondition (a shape the engine
 * does not support, a call out of order such as a step without a session);
 * bw_last_error() then returns the message (thread-local, valid until the
 * next failing call on that thread).
 * No exception crosses this boundary.  Pointers documented as "device" are
 * CUDA device pointers of the context's device; "stream" is a cudaStream_t.
 * A NULL stream orders the call like the legacy default stream (the work runs
 * on the context's own stream after everything already issued on the legacy
 * stream, and later legacy-stream work waits for it).
 *
 * Residues are canonical uint32 values in [0, p); blocks are row-major
 * (row * width + column), the layout of the reference's dense blocks
 * (cuda/matrices.h:23-41, cuda/prym_cuda_helpers.h:67-85).
 */
#ifndef BW_ENGINE_H
#define BW_ENGINE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BW_ABI_VERSION 2

#if defined(__GNUC__)
#define BW_API __attribute__((visibility("default")))
#else
#define BW_API
#endif

/* Arithmetic form of the hot path. */
#define BW_FORM_PLAIN 0 /* uint32/int32 CUDA-core modular arithmetic */
#define BW_FORM_INT8 1  /* signed 8-bit limbs on tcgen05 kind::i8 tensor cores */

/* Message of the last failing call on this thread ("" if none). */
BW_API const char* bw_last_error(void);

/* ABI version (BW_ABI_VERSION). */
BW_API int bw_abi_version(void);

/* Fill count residues of the counter-based seeded stream (seed, tag) into a
 * device buffer: value idx is uniform in [lo, p).  The same stream on the host
 * is bw_seeded_fill_host.  No reference counterpart: the synthetic workloads'
 * inputs are defined by this stream. */
BW_API int bw_seeded_fill(uint32_t* d_out, uint64_t count, uint64_t seed, uint32_t tag,
                   uint32_t p, uint32_t lo, int device, void* stream);
BW_API int bw_seeded_fill_host(uint32_t* out, uint64_t count, uint64_t seed, uint32_t tag,
                        uint32_t p, uint32_t lo);

/* ------------------------------------------------------------------------
 * Synthetic Koszul operator
 *   d : Lambda^k(F^r) (x) R_q -> Lambda^(k-1)(F^r) (x) R_(q+1),
 *   (d y)[T, c] = sum_{i not in T} (-1)^pos(i, T u {i}) sum_b M_i[c, b] y[T u {i}, b],
 *   S = D d^T d, sequence a_i = X^T S^i Y.
 * Row order follows the reference's explicit differential
 * (tests/deformation_reference.py:75-89): lexicographic subsets, coefficient
 * index fastest.  The reference's nearest kernel is
 * cyclic_phi_forward_scaled_kernel / cyclic_phi_transpose_kernel
 * (cuda/cyclic_cuda_helpers.h:145-266) with dense maps in place of the
 * character-sparse mu.
 * ---------------------------------------------------------------------- */

typedef struct bw_koszul bw_koszul;

typedef struct bw_koszul_desc {
    uint32_t r;           /* generators (exterior rank), 2..31 */
    uint32_t k;           /* source exterior degree, 1..r */
    uint32_t dim_in;      /* dim R_q   (columns of each M_i); at most 64 in the INT8 form */
    uint32_t dim_out;     /* dim R_q+1 (rows of each M_i); at most 64 in the INT8 form */
    uint32_t prime;       /* odd prime < 2^15 */
    uint32_t block_width; /* n: columns of Y (4, 8, 16 or 32) */
    uint32_t proj_width;  /* m: columns of X (4, 8, 16 or 32) */
    uint32_t form;        /* BW_FORM_PLAIN or BW_FORM_INT8 */
    const uint32_t* maps; /* host, r * dim_out * dim_in canonical residues, M_i row-major */
    const uint32_t* diag; /* N_src nonzero residues of D (host or device, see diag_on_device) */
    uint32_t diag_on_device;
} bw_koszul_desc;

typedef struct bw_koszul_info {
    uint64_t n_src;          /* C(r,k) * dim_in  : rows of Y, X and S */
    uint64_t n_tgt;          /* C(r,k-1) * dim_out */
    uint64_t device_bytes;   /* device memory held by the context */
    uint64_t scratch_bytes;  /* of which projection scratch (partials + counters) */
    uint32_t form;
    uint32_t sm_count;
} bw_koszul_info;

/* Replaces the operator set-up of run_eliminated_sector
 * (cuda/cuprym_cyclic.cu:2136-2324) for the synthetic operator: builds the
 * incidence tables, uploads maps and diagonal, allocates the work blocks. */
BW_API int bw_koszul_create(const bw_koszul_desc* desc, int device, bw_koszul** out);
BW_API int bw_koszul_info_get(const bw_koszul* ctx, bw_koszul_info* out);
BW_API void bw_koszul_destroy(bw_koszul* ctx);

/* d_z = d d_y (device, canonical).  Replaces cyclic_phi_forward_scaled_kernel
 * (cuda/cyclic_cuda_helpers.h:145-204). */
BW_API int bw_koszul_forward(bw_koszul* ctx, const uint32_t* d_y, uint32_t* d_z, void* stream);
/* d_w = d^T d_z, times D when scale_by_diag (device, canonical).  Replaces
 * cyclic_phi_transpose_kernel (cuda/cyclic_cuda_helpers.h:206-266). */
BW_API int bw_koszul_transpose(bw_koszul* ctx, const uint32_t* d_z, uint32_t* d_w, int scale_by_diag,
                        void* stream);
/* d_out = S d_y (device, canonical).  Replaces apply_square
 * (cuda/cuprym_cyclic.cu:2408-2418). */
BW_API int bw_koszul_apply(bw_koszul* ctx, const uint32_t* d_y, uint32_t* d_out, void* stream);

/* Sequence session (replaces the hot loop of run_eliminated_sector,
 * cuda/cuprym_cyclic.cu:2420-2450, and compute_and_push_bigsp2, :886-897):
 *   start : loads X (n_src x m) and Y0 (n_src x n), writes a_0 = X^T Y0 into
 *           d_seq[0] (d_seq holds seq_capacity entries of m x n residues);
 *   step  : performs `steps` applications of S, appending a_i after each;
 *   finish: writes the current block S^i Y0 to d_y_out (may be NULL) and the
 *           number of entries written to *nlen_out (may be NULL). */
BW_API int bw_koszul_seq_start(bw_koszul* ctx, const uint32_t* d_x, const uint32_t* d_y0,
                        uint32_t* d_seq, uint64_t seq_capacity, void* stream);
BW_API int bw_koszul_seq_step(bw_koszul* ctx, uint64_t steps, void* stream);
BW_API int bw_koszul_seq_finish(bw_koszul* ctx, uint32_t* d_y_out, uint64_t* nlen_out, void* stream);

/* One-shot sequence of nlen entries through HOST buffers: copies X and Y0 to
 * the device, runs nlen-1 steps, copies the sequence (nlen x m x n) and the
 * final block back (h_y_final may be NULL).  Synchronous. */
BW_API int bw_koszul_sequence_host(bw_koszul* ctx, const uint32_t* h_x, const uint32_t* h_y0,
                            uint64_t nlen, uint32_t* h_seq, uint32_t* h_y_final);

/* Like bw_koszul_seq_step, but issues the steps one kernel at a time with
 * CUDA events around each launch on the session stream and returns the
 * average device time per launch (ms) of each kernel kind in ms_out[0..2]:
 * [0] forward d, [1] transpose d^T (with D), [2] projection.  For measurement
 * (roofline figures); the sequence it appends is the same. */
BW_API int bw_koszul_seq_step_timed(bw_koszul* ctx, uint64_t steps, float* ms_out, void* stream);

/* Number of engine kernel launches issued by this context since creation. */
BW_API uint64_t bw_koszul_launch_count(const bw_koszul* ctx);

/* The context's kernel plan as text: for the INT8 form, each direction's
 * producer (TMA gathers or 8 or 16 cp.async warps), generators per stage,
 * pipeline slots and shared memory, with the set-up autotuner's timing of
 * every candidate when it ran (a shape already tuned in this process reuses
 * the choice), and the projection's stage; for the plain form, the output
 * rows a thread of each direction's gathers (4 or 8, timed the same way).  No reference counterpart (the
 * reference has one fixed kernel configuration per block width,
 * cuda/cyclic_cuda_helpers.h:552-631). */
BW_API int bw_koszul_plan(const bw_koszul* ctx, char* buf, size_t cap);

/* Batch of synthetic operators ("sectors" of uneven shapes, block widths and
 * forms) whose sequences advance together: every batch step advances every
 * sector by one step, and 16 steps of all sectors run as one CUDA graph with
 * one branch per sector.  Replaces the reference's one-process-per-sector
 * scheduling of the sequence stage (scripts/reproduce.py:235-259) for the
 * synthetic operator; each sector's arithmetic is that of bw_koszul_*.
 * d_x[i], d_y0[i], d_seq[i] and d_y_out[i] are sector i's buffers as for
 * bw_koszul_seq_*; seq_capacity applies to every sector. */
typedef struct bw_koszul_batch bw_koszul_batch;
BW_API int bw_koszul_batch_create(const bw_koszul_desc* descs, uint32_t count, int device, bw_koszul_batch** out);
BW_API void bw_koszul_batch_destroy(bw_koszul_batch* batch);
/* Borrowed handle of sector `index` (bw_koszul_info_get, single applications
 * outside a session); valid until the batch is destroyed; do not destroy it. */
BW_API int bw_koszul_batch_sector(bw_koszul_batch* batch, uint32_t index, bw_koszul** out);
BW_API int bw_koszul_batch_seq_start(bw_koszul_batch* batch, const uint32_t* const* d_x, const uint32_t* const* d_y0,
                                     uint32_t* const* d_seq, uint64_t seq_capacity, void* stream);
BW_API int bw_koszul_batch_seq_step(bw_koszul_batch* batch, uint64_t steps, void* stream);
BW_API int bw_koszul_batch_seq_finish(bw_koszul_batch* batch, uint32_t* const* d_y_out, uint64_t* nlen_out,
                                      void* stream);
BW_API uint64_t bw_koszul_batch_launch_count(const bw_koszul_batch* batch);

/* ------------------------------------------------------------------------
 * Paper mode: the eliminated cyclic operator of one sector,
 *   F(x, z) = D_(m-1)(B z - R D_m x),  S = Dc F^t T^t Dr T F Dc,
 * and its symmetric moment sequence V^t S^k V (block width 4), exactly as the
 * reference's cuprym_cyclic executable computes it (cuda/cuprym_cyclic.cu).
 * ---------------------------------------------------------------------- */

typedef struct bw_cyclic bw_cyclic;

#define BW_CYCLIC_APPLY_SQUARE 0          /* S: cols x 4 -> cols x 4 */
#define BW_CYCLIC_APPLY_FORWARD 1         /* F, no preconditioners: cols x 4 -> rows x 4 */
#define BW_CYCLIC_APPLY_TRANSPOSE 2       /* F^t, no preconditioners: rows x 4 -> cols x 4 */
#define BW_CYCLIC_APPLY_SQUARE_UNFOLDED 3 /* S with T, Dr, T^t applied round by round */

typedef struct bw_cyclic_info {
    uint64_t rows;          /* target rows of F in this sector (N_r) */
    uint64_t cols;          /* source columns of the operator (N_c: x + z, +2 for augmented) */
    uint64_t x_cols, z_cols, t_rows, y_rows;
    uint64_t dm_nnz, d2_nnz;
    uint64_t default_nlen;  /* 2 N_c / 4 + 50 (cuda/cuprym_cyclic.cu:2316) */
    uint64_t seq_len;       /* moments held after bw_cyclic_generate */
    uint64_t rowmix_realized_seed, rowmix_hash;
    uint64_t device_bytes;
    uint32_t genus, prime, order, sector, y_sector, num_v;
} bw_cyclic_info;

/* Loads the instance JSON, assembles the sector, draws the seeded
 * preconditioners and initial block, builds the row-mixing plan and uploads
 * everything.  Replaces load_cyclic_instance, build_*_generic and the set-up
 * half of run_eliminated_sector (cuda/cuprym_cyclic.cu:483-819, 2136-2324),
 * and for op "augmented" / "replacement" the set-up of
 * run_deformation_eliminated_variant (cuda/cuprym_deformation.cu:2554-2797):
 *   augmented   F = [F0 | -b],  source = base columns + 2 dense columns;
 *   replacement F = F0 without the two columns of drop_path, + the 2 dense
 *               columns of dense_path (cuda/cuprym_deformation.cu:426-473).
 * dense_path is required for the deformation operators and drop_path for
 * replacement only (NULL or "" = none; ignored for "eliminated").  num_v must
 * be 4 (the paper recipe).  device < 0 opens a host-only context (assembly,
 * seeded data, plan, sidecar; every device call then fails with status 3). */
BW_API int bw_cyclic_open(const char* instance_path, const char* op, uint32_t sector, uint32_t num_v,
                          uint64_t seed, uint32_t rowmix_rounds, uint64_t rowmix_seed, const char* dense_path,
                          const char* drop_path, int device, bw_cyclic** out);
BW_API int bw_cyclic_info_get(const bw_cyclic* ctx, bw_cyclic_info* out);
BW_API void bw_cyclic_close(bw_cyclic* ctx);

/* One application (BW_CYCLIC_APPLY_*) through host buffers (row-major,
 * canonical).  Replaces apply_square / apply_forward / apply_backward
 * (cuda/cuprym_cyclic.cu:2330-2418). */
BW_API int bw_cyclic_apply_host(bw_cyclic* ctx, int what, const uint32_t* in, uint32_t* out);

/* Runs the symmetric sequence from the initial block: nlen moments (0 = the
 * default 2 N_c / 4 + 50), rounded up to whole rounds of 4 moments like the
 * reference's hot loop (cuda/cuprym_cyclic.cu:2420-2450). */
BW_API int bw_cyclic_generate(bw_cyclic* ctx, uint64_t nlen);
/* bw_cyclic_generate that also returns the device time of the rounds (CUDA
 * events around the round graphs on the context's stream, in ms); for
 * measurement. */
BW_API int bw_cyclic_generate_timed(bw_cyclic* ctx, uint64_t nlen, float* device_ms);

/* Copies the packed moments (seq_len x 10, upper triangles in WDM order) and
 * the current block (cols x 4, row-major) to host buffers (either may be NULL). */
BW_API int bw_cyclic_download(bw_cyclic* ctx, uint32_t* packed_seq, uint64_t seq_capacity, uint32_t* current);

/* Output names and files (cuda/cuprym_cyclic.cu:1295-1400, 965-1007):
 * output_path creates out_dir and writes the WDM path into buf;
 * check_outputs_absent fails if the WDM or its sidecar exists;
 * write_sidecar writes the .rowmix.json; write_wdm writes WDM.tmp, then renames. */
BW_API int bw_cyclic_output_path(const bw_cyclic* ctx, const char* out_dir, char* buf, size_t cap);
BW_API int bw_cyclic_check_outputs_absent(const char* wdm_path);
BW_API int bw_cyclic_write_sidecar(const bw_cyclic* ctx, const char* wdm_path);
BW_API int bw_cyclic_write_wdm(bw_cyclic* ctx, const char* wdm_path);

/* --validate-rowmix (cuda/cuprym_cyclic.cu:1970-2132): the rowmix transpose
 * identity on the host, the folded target preconditioner against the
 * round-by-round one on three deterministic blocks, and the symmetry
 * <S x, y> = <x, S y>, all on the device. */
BW_API int bw_cyclic_validate(bw_cyclic* ctx, uint32_t columns);

BW_API uint64_t bw_cyclic_launch_count(const bw_cyclic* ctx);

/* Which gather kernels the context runs: "subset: tables cached" or
 * "subset: tables evict-first" (one thread per subset, every character block
 * at most two rows: all shipped instances; the incidence tables are read
 * evict-first when they exceed half the L2) or "generic: <reason>" (one
 * thread per row).  Setting BW_CYCLIC_GENERIC=1 in the environment before
 * bw_cyclic_open selects the generic kernels; BW_CYCLIC_STREAM_TABLES=1 (=0)
 * forces the evict-first (cached) table reads at any size.  All give the same
 * residues.  No reference counterpart (the reference has the row kernels
 * only, cuda/cyclic_cuda_helpers.h:145-266). */
BW_API int bw_cyclic_gather_path(const bw_cyclic* ctx, char* buf, size_t cap);

/* Kernel-vector recovery (replaces cuda/cuprym_cyclic_kernel_vectors.cu,
 * recover_eliminated_kernel_vectors and recover_kernel_vectors_core,
 * :2550-2986, and recover_deformation_eliminated_variant,
 * cuda/cuprym_deformation_kernel_vectors.cu:3067-3487, for op "augmented" /
 * "replacement" with dense_path / drop_path as in bw_cyclic_open): reads the
 * WDM initial state and its row-mixing sidecar
 * (hashes and plan checked as in resolve_rowmix_options, :1554-1643), the
 * generator file (one v x v matrix per line), forms D = sum_k S^k V G_k^t on
 * the device, certifies F Dc D = 0 and writes the preconditioned and
 * original-coordinate candidates and the JSON report.  Empty or NULL paths
 * take the reference's defaults (WDM stem + _generators.txt, WDM +
 * _nullvectors_{1,2}.txt, WDM + _nullvectors_report.json).  cli_rounds and
 * cli_seed apply only without a sidecar (rounds_supplied/seed_supplied say
 * whether the caller passed them). */
BW_API int bw_cyclic_recover(const char* instance_path, const char* op, uint32_t sector, const char* wdm_path,
                             const char* generators_path, const char* preconditioned_out, const char* original_out,
                             const char* report_out, const char* dense_path, const char* drop_path,
                             int64_t cli_rounds, uint64_t cli_seed, int rounds_supplied, int seed_supplied,
                             int validate, int device);

/* Block projection d_out = X^T W (m x n canonical residues; X is rows x m and
 * W rows x n, canonical, device, W 16-byte aligned) that allocates nothing:
 * the cross-CTA scratch is a fixed 1 MiB + 256 B array inside the library.
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * a framework whose allocator owns all device memory, or code that must not
 * trigger the device-wide synchronisation of cudaMalloc / cudaFree.
 * Limits: m, n in {4, 8, 16, 32}; odd prime below 2^15; rows below 2^40;
 * other sizes are rejected with status 1.  The first call on a device (and
 * the first after cudaDeviceReset replaced its context) looks up the array's
 * device address (cudaGetSymbolAddress) and should come before any stream
 * capture.  All calls share the array: calls that overlap on the GPU race and
 * give wrong results; each call clears the arrival counter it needs at zero. */
BW_API int bw_project_noalloc(const uint32_t* d_x, const uint32_t* d_w, uint64_t rows, uint32_t m, uint32_t n,
                              uint32_t prime, uint32_t* d_out, int device, void* stream);

/* Reads a text file, decompressing it when it carries the zstd magic
 * (cuda/zstd_compat.h:67-77).  With buf == NULL only *len is set. */
BW_API int bw_file_read_text(const char* path, char* buf, size_t cap, size_t* len);

#ifdef __cplusplus
}
#endif

#endif /* BW_ENGINE_H */
