/*
 * CPU oracle for the synthetic Koszul block-Wiedemann path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA engine in
 * prym_green_ancillary_b200/: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference arms of bench.py may load it.  The product never
 * links or calls it.
 *
 * What it restates (plain C, u64 accumulation, % p, OpenMP over output rows):
 *
 *   d : Lambda^k(F^r) (x) R_q  ->  Lambda^(k-1)(F^r) (x) R_(q+1)
 *   (d y)[T, c] = sum_{i not in T} (-1)^pos(i, T u {i}) sum_b M_i[c, b] y[T u {i}, b]
 *
 * with rows/columns ordered exactly as the reference's explicit sparse-matrix
 * oracle `differential()` (tests/deformation_reference.py:75-89): subsets in
 * lexicographic (itertools.combinations) order, coefficient index fastest,
 * row = T_rank * dim_out + c, column = S_rank * dim_in + b, sign (-1)^position.
 * The loop structure of the forward and transpose applications follows the
 * reference's CPU Phi forward/transpose (cuda/cuprym_cyclic.cu:1591-1688):
 * one u64 sum per output entry, reduced once at the end.
 *
 * The square operator is S = D d^T d with D a nonzero diagonal on the source
 * space; the block-Wiedemann sequence is a_i = X^T S^i Y (i = 0..nlen-1), the
 * general (non-symmetric) form of the reference's moment loop
 * (cuda/cuprym_cyclic.cu:2420-2450).
 *
 * Parity pin: tests/golden/ holds sequences and operator applications
 * produced by the reference's own `differential()` matrices
 * (tests/golden/make_koszul_golden.py); test_oracle.py checks this file
 * against them.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* ---------------------------------------------------------------- subsets */

uint64_t orc_binom(int n, int k) {
    if (k < 0 || n < 0 || k > n) return 0;
    if (k > n - k) k = n - k;
    unsigned __int128 out = 1;
    for (int i = 0; i < k; ++i) out = out * (unsigned)(n - i) / (unsigned)(i + 1);
    return (uint64_t)out;
}

/* Lexicographic unrank of a k-subset of {0..r-1} (cuda/cuprym_cyclic.cu:184-211). */
void orc_unrank(uint64_t rank, int r, int k, int* out) {
    int start = 0;
    for (int pos = 0; pos < k; ++pos) {
        int remaining = k - pos - 1;
        for (int v = start; v < r; ++v) {
            uint64_t cnt = orc_binom(r - v - 1, remaining);
            if (rank < cnt) { out[pos] = v; start = v + 1; break; }
            rank -= cnt;
        }
    }
}

/* Lexicographic rank: the inverse of orc_unrank, by direct enumeration. */
uint64_t orc_rank(const int* s, int r, int k) {
    uint64_t rank = 0;
    int start = 0;
    for (int pos = 0; pos < k; ++pos) {
        for (int v = start; v < s[pos]; ++v) rank += orc_binom(r - v - 1, k - pos - 1);
        start = s[pos] + 1;
    }
    return rank;
}

/* ------------------------------------------------------- seeded residues */

static inline uint64_t orc_mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

/* Counter-based seeded stream: value number idx of stream (seed, tag). */
uint64_t orc_seeded_u64(uint64_t seed, uint32_t tag, uint64_t idx) {
    uint64_t base = orc_mix64(seed ^ (0xD1B54A32D192ED03ULL * (uint64_t)(tag + 1)));
    return orc_mix64(base + (idx + 1) * 0x9E3779B97F4A7C15ULL);
}

/* Uniform residue in [lo, p) (lo = 0 or 1) by 64x64->128 multiply-shift. */
uint32_t orc_seeded_residue(uint64_t seed, uint32_t tag, uint64_t idx, uint32_t p, uint32_t lo) {
    uint64_t z = orc_seeded_u64(seed, tag, idx);
    return lo + (uint32_t)(((unsigned __int128)z * (uint64_t)(p - lo)) >> 64);
}

void orc_fill_seeded(uint64_t seed, uint32_t tag, uint32_t p, uint32_t lo, uint32_t* out, uint64_t count) {
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)count; ++i) out[i] = orc_seeded_residue(seed, tag, (uint64_t)i, p, lo);
}

/* ------------------------------------------------------------- operators */

typedef struct {
    int r, k, ci, co, nb;
    uint32_t p;
} orc_shape;

/* Z rows of the target subsets [t0, t1) of d Y (Z indexed globally).
 * Y: N_src x nb row-major, Z: N_tgt x nb row-major, maps: r x co x ci. */
void orc_koszul_forward_range(int r, int k, int ci, int co, uint32_t p, int nb,
                              const uint32_t* maps, const uint32_t* Y, uint32_t* Z,
                              int64_t t0, int64_t t1) {
    #pragma omp parallel
    {
        int T[64], S[64];
        uint64_t* acc = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)co * (size_t)nb);
        #pragma omp for schedule(dynamic, 64)
        for (int64_t t = t0; t < t1; ++t) {
            orc_unrank((uint64_t)t, r, k - 1, T);
            memset(acc, 0, sizeof(uint64_t) * (size_t)co * (size_t)nb);
            int pos = 0;   /* number of T entries below i = position of i in S */
            for (int i = 0; i < r; ++i) {
                if (pos < k - 1 && T[pos] == i) { ++pos; continue; }
                /* S = T u {i} */
                for (int q = 0, w = 0; q < k; ++q) S[q] = (q == pos) ? i : T[w++];
                uint64_t s_rank = orc_rank(S, r, k);
                const uint32_t* ys = Y + s_rank * (uint64_t)ci * (uint64_t)nb;
                const uint32_t* m = maps + (uint64_t)i * (uint64_t)co * (uint64_t)ci;
                int neg = pos & 1;
                for (int c = 0; c < co; ++c) {
                    for (int b = 0; b < ci; ++b) {
                        uint64_t coeff = m[c * ci + b] % p;
                        if (neg && coeff) coeff = p - coeff;
                        for (int j = 0; j < nb; ++j) acc[c * nb + j] += coeff * ys[b * nb + j];
                    }
                    /* keep the u64 sums bounded: r * ci * p^2 < 2^64 for p < 2^24 */
                }
            }
            uint32_t* zt = Z + (uint64_t)t * (uint64_t)co * (uint64_t)nb;
            for (int e = 0; e < co * nb; ++e) zt[e] = (uint32_t)(acc[e] % p);
        }
        free(acc);
    }
}

/* Z = d Y over all target subsets. */
void orc_koszul_forward(int r, int k, int ci, int co, uint32_t p, int nb,
                        const uint32_t* maps, const uint32_t* Y, uint32_t* Z) {
    orc_koszul_forward_range(r, k, ci, co, p, nb, maps, Y, Z, 0, (int64_t)orc_binom(r, k - 1));
}

/* W rows of the source subsets [s0, s1) of d^T Z (no diagonal).
 * Z: N_tgt x nb, W: N_src x nb. */
void orc_koszul_transpose_range(int r, int k, int ci, int co, uint32_t p, int nb,
                                const uint32_t* maps, const uint32_t* Z, uint32_t* W,
                                int64_t s0, int64_t s1) {
    #pragma omp parallel
    {
        int S[64], T[64];
        uint64_t* acc = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)ci * (size_t)nb);
        #pragma omp for schedule(dynamic, 64)
        for (int64_t s = s0; s < s1; ++s) {
            orc_unrank((uint64_t)s, r, k, S);
            memset(acc, 0, sizeof(uint64_t) * (size_t)ci * (size_t)nb);
            for (int pos = 0; pos < k; ++pos) {
                int i = S[pos];
                for (int q = 0, w = 0; q < k; ++q) if (q != pos) T[w++] = S[q];
                uint64_t t_rank = orc_rank(T, r, k - 1);
                const uint32_t* zt = Z + t_rank * (uint64_t)co * (uint64_t)nb;
                const uint32_t* m = maps + (uint64_t)i * (uint64_t)co * (uint64_t)ci;
                int neg = pos & 1;
                for (int b = 0; b < ci; ++b) {
                    for (int c = 0; c < co; ++c) {
                        uint64_t coeff = m[c * ci + b] % p;
                        if (neg && coeff) coeff = p - coeff;
                        for (int j = 0; j < nb; ++j) acc[b * nb + j] += coeff * zt[c * nb + j];
                    }
                }
            }
            uint32_t* ws = W + (uint64_t)s * (uint64_t)ci * (uint64_t)nb;
            for (int e = 0; e < ci * nb; ++e) ws[e] = (uint32_t)(acc[e] % p);
        }
        free(acc);
    }
}

/* W = d^T Z over all source subsets. */
void orc_koszul_transpose(int r, int k, int ci, int co, uint32_t p, int nb,
                          const uint32_t* maps, const uint32_t* Z, uint32_t* W) {
    orc_koszul_transpose_range(r, k, ci, co, p, nb, maps, Z, W, 0, (int64_t)orc_binom(r, k));
}

static void orc_scale_rows(int64_t rows, int nb, uint32_t p, const uint32_t* diag, uint32_t* Y) {
    #pragma omp parallel for schedule(static)
    for (int64_t row = 0; row < rows; ++row) {
        uint64_t d = diag[row];
        for (int j = 0; j < nb; ++j) Y[row * nb + j] = (uint32_t)((d * Y[row * nb + j]) % p);
    }
}

/* out = D d^T d Y. */
void orc_koszul_apply(int r, int k, int ci, int co, uint32_t p, int nb,
                      const uint32_t* maps, const uint32_t* diag,
                      const uint32_t* Y, uint32_t* out) {
    uint64_t n_tgt = orc_binom(r, k - 1) * (uint64_t)co;
    uint32_t* Z = (uint32_t*)malloc(sizeof(uint32_t) * n_tgt * (uint64_t)nb);
    orc_koszul_forward(r, k, ci, co, p, nb, maps, Y, Z);
    orc_koszul_transpose(r, k, ci, co, p, nb, maps, Z, out);
    orc_scale_rows((int64_t)(orc_binom(r, k) * (uint64_t)ci), nb, p, diag, out);
    free(Z);
}

/* P = X^T Y (m x nb), X: rows x m, Y: rows x nb. */
void orc_project(int64_t rows, int m, int nb, uint32_t p,
                 const uint32_t* X, const uint32_t* Y, uint32_t* P) {
    uint64_t* acc = (uint64_t*)calloc((size_t)m * (size_t)nb, sizeof(uint64_t));
    #pragma omp parallel
    {
        uint64_t* loc = (uint64_t*)calloc((size_t)m * (size_t)nb, sizeof(uint64_t));
        #pragma omp for schedule(static)
        for (int64_t row = 0; row < rows; ++row) {
            for (int x = 0; x < m; ++x) {
                uint64_t xv = X[row * m + x];
                for (int j = 0; j < nb; ++j) loc[x * nb + j] += xv * Y[row * nb + j];
            }
            if ((row & 1023) == 1023) for (int e = 0; e < m * nb; ++e) loc[e] %= p;
        }
        #pragma omp critical
        for (int e = 0; e < m * nb; ++e) acc[e] = (acc[e] + loc[e] % p) % p;
        free(loc);
    }
    for (int e = 0; e < m * nb; ++e) P[e] = (uint32_t)(acc[e] % p);
    free(acc);
}

/* seq[i] = X^T S^i Y0 for i = 0..nlen-1 (m x nb each); Y_final = S^(nlen-1) Y0. */
void orc_koszul_sequence(int r, int k, int ci, int co, uint32_t p, int nb, int m,
                         const uint32_t* maps, const uint32_t* diag,
                         const uint32_t* X, const uint32_t* Y0, int64_t nlen,
                         uint32_t* seq, uint32_t* Y_final) {
    int64_t n_src = (int64_t)(orc_binom(r, k) * (uint64_t)ci);
    uint32_t* a = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n_src * (size_t)nb);
    uint32_t* b = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n_src * (size_t)nb);
    memcpy(a, Y0, sizeof(uint32_t) * (size_t)n_src * (size_t)nb);
    orc_project(n_src, m, nb, p, X, a, seq);
    for (int64_t i = 1; i < nlen; ++i) {
        orc_koszul_apply(r, k, ci, co, p, nb, maps, diag, a, b);
        uint32_t* t = a; a = b; b = t;
        orc_project(n_src, m, nb, p, X, a, seq + i * (int64_t)m * nb);
    }
    if (Y_final) memcpy(Y_final, a, sizeof(uint32_t) * (size_t)n_src * (size_t)nb);
    free(a);
    free(b);
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
