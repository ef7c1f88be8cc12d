// Paper-mode engine: the eliminated cyclic Koszul operator of one sector,
//   F(x, z) = D_(m-1) (B z - R D_m x),   S = Dc F^t T^t Dr T F Dc,
// and its symmetric block-Wiedemann sequence V^t S^k V (block width 4).
//
// Replaces the device work of cuda/cuprym_cyclic.cu (run_eliminated_sector,
// :2136-2496) and cuda/cyclic_cuda_helpers.h.  Differences in structure, not
// in results (every output is the canonical residue the reference produces):
//   * one thread per block row holding the 4 columns as one 16-byte vector;
//   * t = D_m x, y = B z - R t fused into one kernel, and t_adj = R^t h,
//     x_adj = D_m^t t_adj, z_adj = B^t h, the adjoint assembly fused into one;
//   * the target preconditioner T^t Dr T (two paired-SL2 rounds, a diagonal
//     and the two transposed rounds) folded on the host into one exact sparse
//     matrix with at most 16 entries per row, applied in one pass;
//   * both Gram moments of a half-round in one reduction kernel whose last CTA
//     packs the upper triangles (no atomics, deterministic);
//   * one half-round pair captured as a CUDA graph and replayed.
#include "bw_cyclic.cuh"
#include "bw_cyclic_dev.cuh"

#include <algorithm>
#include <cstring>
#include <iostream>

namespace bw {

namespace {

constexpr int kThreads = 256;

using cyc::Acc4;
using cyc::ld4;
using cyc::neg4;
using cyc::red64;
using cyc::scale4;
using cyc::st4;

__device__ __forceinline__ void decode_inc(uint32_t e, uint32_t& sub, int& i, bool& neg) {
    sub = e & 0x3FFFFFFu;
    i = static_cast<int>((e >> 26) & 31u);
    neg = (e >> 31) != 0;
}
__device__ __forceinline__ void decode_coef(int32_t e, int& local, int32_t& coef) {
    local = static_cast<int>(static_cast<uint32_t>(e) >> 16);
    coef = static_cast<int16_t>(e & 0xFFFF);
}

#define BW_ROWS(var, count)                                                                     \
    for (long long var = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; var < (count); \
         var += static_cast<long long>(gridDim.x) * blockDim.x)

// Operator column of base column q: q itself, or (replacement) q less the
// dropped columns before it, -1 for a dropped column.
__device__ __forceinline__ long long op_col(const ElimDev& E, long long q) { return cyc::op_col(E.drop0, E.drop1, q); }

// xs = the scaled source in base order: rows [0, base_cols) take operator
// column op_col(q) times dc (zero for a dropped column), rows base_cols + j
// take the extra column kept_cols + j (dc == nullptr: no scaling).
__global__ void cyc_source_kernel(ElimDev E, const int32_t* __restrict__ in, const int32_t* __restrict__ dc,
                                  int32_t* __restrict__ xs) {
    BW_ROWS(q, static_cast<long long>(E.base_cols) + E.n_extra) {
        const long long src = q < static_cast<long long>(E.base_cols)
                                  ? op_col(E, q)
                                  : static_cast<long long>(E.kept_cols) + (q - static_cast<long long>(E.base_cols));
        if (src < 0) {
            st4(xs, q, make_int4(0, 0, 0, 0));
            continue;
        }
        const int4 v = ld4(in, src);
        st4(xs, q, dc ? scale4(v, __ldg(dc + src), E.mod) : v);
    }
}

// out[row] = dc[row] * in[row]  (dc == nullptr: copy)
__global__ void cyc_scale_kernel(const int32_t* __restrict__ in, const int32_t* __restrict__ dc,
                                 int32_t* __restrict__ out, long long rows, Mod mod) {
    BW_ROWS(row, rows) {
        int4 v = ld4(in, row);
        st4(out, row, dc ? scale4(v, __ldg(dc + row), mod) : v);
    }
}

// Koszul forward row of D on a block `in` whose column blocks start at col_off:
//   sum_{i not in S} +-sum_a mu[i,beta,a] in[(S u i, a)]
template <bool SMALL>
__device__ __forceinline__ int4 koszul_row(const ElimDev& E, const uint32_t* __restrict__ inc, uint32_t width,
                                           const uint32_t* __restrict__ col_off, const int32_t* __restrict__ in,
                                           int beta) {
    Acc4<SMALL> acc;
    for (uint32_t pos = 0; pos < width; ++pos) {
        uint32_t cs;
        int i;
        bool neg;
        decode_inc(__ldg(inc + pos), cs, i, neg);
        const uint32_t base = __ldg(col_off + cs);
        const int li = i * E.n + beta;
        const uint32_t k1 = __ldg(E.fl_off + li + 1);
        for (uint32_t k = __ldg(E.fl_off + li); k < k1; ++k) {
            int la;
            int32_t c;
            decode_coef(__ldg(E.fl + k), la, c);
            acc.mac(neg ? -c : c, ld4(in, base + la));
        }
    }
    return acc.reduce(E.mod);
}

// Koszul transpose column of D on a block `in` whose row blocks start at row_off:
//   sum_{j in S} +-sum_beta mu[j,beta,a] in[(S \ j, beta)]
template <bool SMALL>
__device__ __forceinline__ int4 koszul_col(const ElimDev& E, const uint32_t* __restrict__ inc, uint32_t width,
                                           const uint32_t* __restrict__ row_off, const int32_t* __restrict__ in,
                                           int a) {
    Acc4<SMALL> acc;
    for (uint32_t pos = 0; pos < width; ++pos) {
        uint32_t rs;
        int j;
        bool neg;
        decode_inc(__ldg(inc + pos), rs, j, neg);
        const uint32_t base = __ldg(row_off + rs);
        const int lj = j * E.g + a;
        const uint32_t k1 = __ldg(E.tl_off + lj + 1);
        for (uint32_t k = __ldg(E.tl_off + lj); k < k1; ++k) {
            int lb;
            int32_t c;
            decode_coef(__ldg(E.tl + k), lb, c);
            acc.mac(neg ? -c : c, ld4(in, base + lb));
        }
    }
    return acc.reduce(E.mod);
}

// t = D_m xs  (rows (S, beta) over (m-1)-subsets)
template <bool SMALL>
__global__ void cyc_dm_forward_kernel(ElimDev E, const int32_t* __restrict__ xs, int32_t* __restrict__ t) {
    BW_ROWS(tr, E.t_rows) {
        const uint32_t S = __ldg(E.t_sub + tr);
        st4(t, tr, koszul_row<SMALL>(E, E.dm_row_inc + static_cast<size_t>(S) * E.dm_row_width, E.dm_row_width,
                                     E.x_off, xs, __ldg(E.t_beta + tr)));
    }
}

// y(S, a) = sum_kappa B[a,kappa] zs(S,kappa) - sum_beta R[a,beta] t(S,beta)
template <bool SMALL>
__global__ void cyc_elim_y_kernel(ElimDev E, const int32_t* __restrict__ xs, const int32_t* __restrict__ t,
                                  int32_t* __restrict__ y) {
    BW_ROWS(yr, E.y_rows) {
        const uint32_t S = __ldg(E.y_sub + yr);
        const int a = __ldg(E.y_a + yr);
        Acc4<SMALL> acc;
        const uint32_t z1 = __ldg(E.z_off + S + 1);
        for (uint32_t zr = __ldg(E.z_off + S); zr < z1; ++zr) {
            const int32_t c = __ldg(E.Bk + a * E.kdim + __ldg(E.z_k + zr));
            if (c) acc.mac(c, ld4(xs, static_cast<long long>(E.x_cols) + zr));
        }
        const uint32_t t1 = __ldg(E.t_off + S + 1);
        for (uint32_t tr = __ldg(E.t_off + S); tr < t1; ++tr) {
            const int32_t c = __ldg(E.R + a * E.n + __ldg(E.t_beta + tr));
            if (c) acc.mac(-c, ld4(t, tr));
        }
        st4(y, yr, acc.reduce(E.mod));
    }
}

// u = D_(m-1) y  (rows (S2, beta) over (m-2)-subsets), plus dense_sign *
// dense xs_extra for the deformation variants (|terms| stay below 2^31: a
// balanced residue plus two products of balanced residues).
template <bool SMALL>
__global__ void cyc_d2_forward_kernel(ElimDev E, const int32_t* __restrict__ y, const int32_t* __restrict__ xs,
                                      int32_t* __restrict__ u) {
    BW_ROWS(ur, E.n_r) {
        const uint32_t S2 = __ldg(E.u_sub + ur);
        int4 v = koszul_row<SMALL>(E, E.d2_row_inc + static_cast<size_t>(S2) * E.d2_row_width, E.d2_row_width,
                                   E.y_off, y, __ldg(E.u_beta + ur));
        if (E.n_extra) {
            for (int j = 0; j < E.n_extra; ++j) {
                const int32_t c = E.dense_sign * __ldg(E.dense + ur * E.n_extra + j);
                const int4 e = ld4(xs, static_cast<long long>(E.base_cols) + j);
                v.x += c * e.x;
                v.y += c * e.y;
                v.z += c * e.z;
                v.w += c * e.w;
            }
            v = make_int4(reduce_balanced(v.x, E.mod), reduce_balanced(v.y, E.mod), reduce_balanced(v.z, E.mod),
                          reduce_balanced(v.w, E.mod));
        }
        st4(u, ur, v);
    }
}

// out = P u  (P = T^t Dr T in CSR)
template <bool SMALL>
__global__ void cyc_spmv_kernel(const uint32_t* __restrict__ ptr, const uint32_t* __restrict__ col,
                                const int32_t* __restrict__ val, const int32_t* __restrict__ u,
                                int32_t* __restrict__ out, long long rows, Mod mod) {
    BW_ROWS(row, rows) {
        Acc4<SMALL> acc;
        const uint32_t e1 = __ldg(ptr + row + 1);
        for (uint32_t e = __ldg(ptr + row); e < e1; ++e) acc.mac(__ldg(val + e), ld4(u, __ldg(col + e)));
        st4(out, row, acc.reduce(mod));
    }
}

// h = D_(m-1)^t u2  (rows (S, a) over (m-1)-subsets)
template <bool SMALL>
__global__ void cyc_d2_transpose_kernel(ElimDev E, const int32_t* __restrict__ u2, int32_t* __restrict__ h) {
    BW_ROWS(yr, E.y_rows) {
        const uint32_t S = __ldg(E.y_sub + yr);
        st4(h, yr, koszul_col<SMALL>(E, E.d2_col_inc + static_cast<size_t>(S) * E.d2_col_width, E.d2_col_width,
                                     E.u_off, u2, __ldg(E.y_a + yr)));
    }
}

// rows [0, t_rows):            t_adj(S, beta) = sum_a R[a,beta] h(S, a)
// rows [t_rows, t_rows+z_cols): out_z(S, kappa) = dc * sum_a B[a,kappa] h(S, a)
template <bool SMALL>
__global__ void cyc_adjoint_t_z_kernel(ElimDev E, const int32_t* __restrict__ h, const int32_t* __restrict__ dc,
                                       int32_t* __restrict__ t_adj, int32_t* __restrict__ out) {
    BW_ROWS(row, static_cast<long long>(E.t_rows) + E.z_cols) {
        Acc4<SMALL> acc;
        if (row < E.t_rows) {
            const uint32_t S = __ldg(E.t_sub + row);
            const int beta = __ldg(E.t_beta + row);
            const uint32_t y1 = __ldg(E.y_off + S + 1);
            for (uint32_t yr = __ldg(E.y_off + S); yr < y1; ++yr) {
                const int32_t c = __ldg(E.R + __ldg(E.y_a + yr) * E.n + beta);
                if (c) acc.mac(c, ld4(h, yr));
            }
            st4(t_adj, row, acc.reduce(E.mod));
        } else {
            const long long zr = row - E.t_rows;
            const uint32_t S = __ldg(E.z_sub + zr);
            const int kap = __ldg(E.z_k + zr);
            const uint32_t y1 = __ldg(E.y_off + S + 1);
            for (uint32_t yr = __ldg(E.y_off + S); yr < y1; ++yr) {
                const int32_t c = __ldg(E.Bk + __ldg(E.y_a + yr) * E.kdim + kap);
                if (c) acc.mac(c, ld4(h, yr));
            }
            const long long orow = op_col(E, static_cast<long long>(E.x_cols) + zr);
            if (orow < 0) continue;   // dropped base column (replacement)
            const int4 v = acc.reduce(E.mod);
            st4(out, orow, dc ? scale4(v, __ldg(dc + orow), E.mod) : v);
        }
    }
}

// out_x(S', a) = -dc * (D_m^t t_adj)(S', a)
template <bool SMALL>
__global__ void cyc_dm_transpose_kernel(ElimDev E, const int32_t* __restrict__ t_adj, const int32_t* __restrict__ dc,
                                        int32_t* __restrict__ out) {
    BW_ROWS(xr, E.x_cols) {
        const long long orow = op_col(E, xr);
        if (orow < 0) continue;   // dropped base column (replacement)
        const uint32_t S = __ldg(E.x_sub + xr);
        const int4 v = neg4(koszul_col<SMALL>(E, E.dm_col_inc + static_cast<size_t>(S) * E.dm_col_width,
                                              E.dm_col_width, E.t_off, t_adj, __ldg(E.x_a + xr)));
        st4(out, orow, dc ? scale4(v, __ldg(dc + orow), E.mod) : v);
    }
}

// One paired-SL2 round on the target block (validation path).
__global__ void cyc_rowmix_kernel(const uint32_t* __restrict__ pairs, long long count, int32_t* __restrict__ block,
                                  bool transpose, Mod mod) {
    for (long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; q < count;
         q += static_cast<long long>(gridDim.x) * blockDim.x) {
        const uint32_t f = __ldg(pairs + 3 * q), s = __ldg(pairs + 3 * q + 1), ab = __ldg(pairs + 3 * q + 2);
        const long long a = ab & 0xFFFF, b = ab >> 16, oab = 1 + a * b;
        const int4 x = ld4(block, f), y = ld4(block, s);
        int4 nf, ns;
        if (transpose) {
            nf = make_int4(red64(x.x + b * y.x, mod), red64(x.y + b * y.y, mod), red64(x.z + b * y.z, mod),
                           red64(x.w + b * y.w, mod));
            ns = make_int4(red64(a * x.x + oab * y.x, mod), red64(a * x.y + oab * y.y, mod),
                           red64(a * x.z + oab * y.z, mod), red64(a * x.w + oab * y.w, mod));
        } else {
            nf = make_int4(red64(x.x + a * y.x, mod), red64(x.y + a * y.y, mod), red64(x.z + a * y.z, mod),
                           red64(x.w + a * y.w, mod));
            ns = make_int4(red64(b * x.x + oab * y.x, mod), red64(b * x.y + oab * y.y, mod),
                           red64(b * x.z + oab * y.z, mod), red64(b * x.w + oab * y.w, mod));
        }
        st4(block, f, nf);
        st4(block, s, ns);
    }
}

__device__ __forceinline__ int tri_index(int row, int col) { return row * (2 * 4 - row + 1) / 2 + (col - row); }

// Gram moments of one half-round: G1 = A1^t C1 and (count == 2) G2 = A2^t C2,
// upper triangles packed into seq at positions *seq_index (+1), canonical.
// partials: gridDim.x x 20 int32; counter left at 0.
__global__ void __launch_bounds__(kThreads) cyc_gram_kernel(
    const int32_t* __restrict__ A1, const int32_t* __restrict__ C1, const int32_t* __restrict__ A2,
    const int32_t* __restrict__ C2, int count, long long rows, int32_t* __restrict__ partials,
    unsigned int* __restrict__ counter, uint32_t* __restrict__ seq, unsigned long long* __restrict__ seq_index,
    Mod mod) {
    cyc::pdl_trigger();
    cyc::pdl_wait();
    int32_t acc[20];
#pragma unroll
    for (int e = 0; e < 20; ++e) acc[e] = 0;
    int cnt = 0;
    for (long long row = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; row < rows;
         row += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int4 a1 = ld4(A1, row), c1 = ld4(C1, row);
        const int av[4] = {a1.x, a1.y, a1.z, a1.w}, cv[4] = {c1.x, c1.y, c1.z, c1.w};
#pragma unroll
        for (int r0 = 0; r0 < 4; ++r0)
#pragma unroll
            for (int c0 = r0; c0 < 4; ++c0) acc[tri_index(r0, c0)] += av[r0] * cv[c0];
        if (count == 2) {
            const int4 a2 = ld4(A2, row), c2 = ld4(C2, row);
            const int bv[4] = {a2.x, a2.y, a2.z, a2.w}, dv[4] = {c2.x, c2.y, c2.z, c2.w};
#pragma unroll
            for (int r0 = 0; r0 < 4; ++r0)
#pragma unroll
                for (int c0 = r0; c0 < 4; ++c0) acc[10 + tri_index(r0, c0)] += bv[r0] * dv[c0];
        }
        if (++cnt == 8) {
            cnt = 0;
#pragma unroll
            for (int e = 0; e < 20; ++e) acc[e] = reduce_partial(acc[e], mod);
        }
    }
    __shared__ int32_t red[kThreads / 32][20];
    __shared__ bool am_last;
    // warp reduction (values below 2p; 32 of them stay far inside int32)
#pragma unroll
    for (int e = 0; e < 20; ++e) {
        int32_t v = reduce_balanced(acc[e], mod);
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        acc[e] = v;
    }
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (lane == 0)
#pragma unroll
        for (int e = 0; e < 20; ++e) red[warp][e] = reduce_balanced(acc[e], mod);
    __syncthreads();
    int32_t mine = 0, total = 0;
    if (threadIdx.x < 20) {
        for (int w = 0; w < kThreads / 32; ++w) mine += red[w][threadIdx.x];
        mine = reduce_balanced(mine, mod);
    }
    if (!cyc::grid_sum(partials, counter, 20, mine, total, &am_last)) return;
    const unsigned long long pos = *reinterpret_cast<volatile unsigned long long*>(seq_index);
    if (threadIdx.x < 10 * count) {
        const int which = threadIdx.x / 10, e = threadIdx.x % 10;
        seq[(pos + which) * 10 + e] = to_canonical(reduce_balanced(total, mod), mod);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        *seq_index = pos + count;
        *counter = 0;
        __threadfence();
    }
}

// Extra source rows of the deformation transpose:
//   out[kept_cols + j][c] = dense_sign * dc[kept_cols + j] * sum_row dense[row][j] u2[row][c]
// (dc == nullptr: unscaled).  Each CTA sums a stripe of rows; the CTA sums
// meet in an 8-entry accumulator (cyc::grid_sum) and the last CTA writes the
// n_extra rows (deterministic; accumulator and counter reset themselves).
__global__ void __launch_bounds__(kThreads) cyc_dense_t_kernel(ElimDev E, const int32_t* __restrict__ u2,
                                                               const int32_t* __restrict__ dc,
                                                               int32_t* __restrict__ out, int32_t* __restrict__ partials,
                                                               unsigned int* __restrict__ counter) {
    int32_t acc[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) acc[e] = 0;
    int cnt = 0;
    for (long long row = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; row < static_cast<long long>(E.n_r);
         row += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int4 v = ld4(u2, row);
        for (int j = 0; j < E.n_extra; ++j) {
            const int32_t d = __ldg(E.dense + row * E.n_extra + j);
            acc[4 * j] += d * v.x;
            acc[4 * j + 1] += d * v.y;
            acc[4 * j + 2] += d * v.z;
            acc[4 * j + 3] += d * v.w;
        }
        if (++cnt == 8) {   // 8 products of balanced residues stay below 2^31
            cnt = 0;
#pragma unroll
            for (int e = 0; e < 8; ++e) acc[e] = reduce_partial(acc[e], E.mod);
        }
    }
    __shared__ int32_t red[kThreads / 32][8];
    __shared__ bool am_last;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        int32_t v = reduce_balanced(acc[e], E.mod);
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (lane == 0) red[warp][e] = reduce_balanced(v, E.mod);
    }
    __syncthreads();
    int32_t mine = 0, total = 0;
    if (threadIdx.x < 8) {
        for (int w = 0; w < kThreads / 32; ++w) mine += red[w][threadIdx.x];
        mine = reduce_balanced(mine, E.mod);
    }
    if (!cyc::grid_sum(partials, counter, 8, mine, total, &am_last)) return;
    if (threadIdx.x < 4 * E.n_extra) {
        const int j = threadIdx.x / 4, c = threadIdx.x % 4;
        const long long orow = static_cast<long long>(E.kept_cols) + j;
        int32_t v = E.dense_sign * reduce_balanced(total, E.mod);
        if (dc) v = reduce_balanced(v * __ldg(dc + orow), E.mod);
        out[orow * 4 + c] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        *counter = 0;
        __threadfence();
    }
}

__global__ void cyc_to_balanced_kernel(const uint32_t* __restrict__ in, int32_t* __restrict__ out, long long n,
                                       Mod mod) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        out[i] = to_balanced(in[i] % static_cast<uint32_t>(mod.p), mod);
}
__global__ void cyc_to_canonical_kernel(const int32_t* __restrict__ in, uint32_t* __restrict__ out, long long n,
                                        Mod mod) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        out[i] = to_canonical(in[i], mod);
}

}  // namespace

// ------------------------------------------------------------------ host

CyclicCtx::~CyclicCtx() {
    if (host_only) return;
    cudaSetDevice(device);
    for (auto& g : graphs)
        if (g) cudaGraphExecDestroy(g);
    for (void* p : allocations) cudaFree(p);
    if (stream) cudaStreamDestroy(stream);
}

template <class T>
T* CyclicCtx::upload(const std::vector<T>& host) {
    void* p = nullptr;
    const size_t bytes = std::max<size_t>(host.size(), 1) * sizeof(T);
    BW_CUDA(cudaMalloc(&p, bytes));
    allocations.push_back(p);
    device_bytes += bytes;
    if (!host.empty()) BW_CUDA(cudaMemcpyAsync(p, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
    return static_cast<T*>(p);
}

template <class T>
T* CyclicCtx::alloc(size_t count) {
    void* p = nullptr;
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    BW_CUDA(cudaMalloc(&p, bytes));
    allocations.push_back(p);
    device_bytes += bytes;
    return static_cast<T*>(p);
}

// used by the subset-major path (bw_cyclic_subset.cu)
template uint4* CyclicCtx::alloc<uint4>(size_t);
template int16_t* CyclicCtx::upload<int16_t>(const std::vector<int16_t>&);
template uint32_t* CyclicCtx::upload<uint32_t>(const std::vector<uint32_t>&);
template int32_t* CyclicCtx::upload<int32_t>(const std::vector<int32_t>&);
template int32_t* CyclicCtx::alloc<int32_t>(size_t);

unsigned CyclicCtx::grid_for(size_t rows) const {
    const size_t blocks = (rows + kThreads - 1) / kThreads;
    return static_cast<unsigned>(std::max<size_t>(1, std::min<size_t>(blocks, static_cast<size_t>(sms) * 8)));
}

namespace {
std::vector<uint32_t> pack_incidence(const std::vector<uint32_t>& sub, const std::vector<uint32_t>& idx,
                                     const std::vector<uint8_t>& neg) {
    std::vector<uint32_t> out(sub.size());
    for (size_t e = 0; e < sub.size(); ++e) {
        if (sub[e] >= (1u << 26) || idx[e] >= 32) throw Error("incidence does not fit the packed device format", 3);
        out[e] = sub[e] | (idx[e] << 26) | (neg[e] ? 0x80000000u : 0u);
    }
    return out;
}
std::vector<int32_t> balanced(const std::vector<uint32_t>& v, const Mod& m) {
    std::vector<int32_t> out(v.size());
    for (size_t i = 0; i < v.size(); ++i) out[i] = to_balanced(v[i] % static_cast<uint32_t>(m.p), m);
    return out;
}
}  // namespace

CyclicCtx* CyclicCtx::open(const std::string& instance_path, const std::string& op, size_t sector, size_t num_v,
                           uint64_t seed, size_t rowmix_rounds, uint64_t rowmix_seed, int dev,
                           const CyclicSource* src, const DeformInputs* deform) {
    BW_REQUIRE(op == "eliminated" || op == "augmented" || op == "replacement",
               "--operator must be one of: eliminated, augmented, replacement.");
    BW_REQUIRE(num_v == 4, "the paper pipeline requires exactly 4 block vectors");
    std::unique_ptr<CyclicCtx> c(new CyclicCtx());
    c->op = op;
    c->num_v = num_v;
    c->seed = seed;
    c->inst = cyclic::load_instance(instance_path);
    BW_REQUIRE(sector < c->inst.r, "--sector must be in 0.." + std::to_string(c->inst.r - 1));
    BW_REQUIRE(cyclic::is_prime(c->inst.modulus), "Modulus " + std::to_string(c->inst.modulus) + " is not prime.");
    BW_REQUIRE(c->inst.modulus >= 3 && c->inst.modulus < 32768, "the engine supports odd primes below 2^15");
    c->p = c->inst.modulus;
    c->mod = make_mod(c->p);
    c->es = cyclic::assemble_eliminated_sector(c->inst, sector);
    const auto& es = c->es;
    const auto& inst = c->inst;
    c->base_cols = c->op_cols = c->kept_cols = es.total_cols();
    const bool deformation = op != "eliminated";
    if (deformation) {
        // run_deformation_eliminated_variant / recover_deformation_eliminated_variant
        // (cuda/cuprym_deformation.cu:2600-2623, cuda/cuprym_deformation_kernel_vectors.cu:3094-3138)
        const bool rec = deform && deform->recovery;
        BW_REQUIRE(deform && !deform->dense_path.empty(),
                   rec ? "deformation recovery requires --dense-file" : "deformation operators require --dense-file");
        c->dense = cyclic::load_dense_block_file(deform->dense_path, c->p);
        BW_REQUIRE(c->dense.rows == es.target_rows && c->dense.columns == 2,
                   rec ? "dense block dimensions do not match the deformation target sector"
                       : "dense block dimensions do not match the eliminated target sector");
        if (op == "replacement") {
            BW_REQUIRE(!deform->drop_path.empty(), rec ? "replacement recovery requires --drop-columns"
                                                       : "replacement operator requires --drop-columns");
            c->drop = cyclic::load_drop_columns_file(deform->drop_path, c->dense.columns, c->base_cols);
            c->kept_cols = c->base_cols - c->drop.size();
        } else {
            BW_REQUIRE(deform->drop_path.empty(), "--drop-columns is only meaningful for replacement");
        }
        c->op_cols = (op == "augmented" ? c->base_cols : c->kept_cols) + c->dense.columns;
    }
    const size_t ncols = c->op_cols;

    if (src) {
        // Recovery: preconditioners, initial block and mixing recipe come from the WDM file and sidecar.
        BW_REQUIRE(src->row_precond.size() == es.target_rows,
                   deformation ? "WDM row count does not match deformation sector"
                               : "WDM row count does not match eliminated sector");
        BW_REQUIRE(src->col_precond.size() == ncols, deformation ? "WDM column count does not match deformation operator"
                                                                 : "WDM column count does not match eliminated sector");
        BW_REQUIRE(src->initial_block.size() == ncols * num_v, "WDM initial block has the wrong size");
        c->row_precond = src->row_precond;
        c->col_precond = src->col_precond;
        c->initial_block = src->initial_block;
        rowmix_rounds = src->rowmix_rounds;
        rowmix_seed = src->rowmix_seed;
    } else {
        // Seeded data in the reference's draw order (cuda/cuprym_cyclic.cu:2196-2199).
        std::mt19937_64 gen(cyclic::seeded_sector_value(seed, sector));
        c->row_precond = cyclic::random_vector(es.target_rows, c->p, gen, true);
        c->col_precond = cyclic::random_vector(ncols, c->p, gen, true);
        c->initial_block = cyclic::random_vector(ncols * num_v, c->p, gen, false);
    }
    c->plan = cyclic::generate_rowmix_plan(es.target_rows, op, sector, c->p, rowmix_rounds, rowmix_seed);
    if (rowmix_rounds > 0) {
        c->precond = cyclic::composite_target_preconditioner(c->plan, c->row_precond, c->p);
    } else {
        c->precond.row_ptr.resize(es.target_rows + 1);
        for (size_t i = 0; i <= es.target_rows; ++i) c->precond.row_ptr[i] = static_cast<uint32_t>(i);
        c->precond.col.resize(es.target_rows);
        for (size_t i = 0; i < es.target_rows; ++i) c->precond.col[i] = static_cast<uint32_t>(i);
        c->precond.val = c->row_precond;
    }

    c->device = dev;
    if (dev < 0) {   // host-only context: assembly, seeded data, plan and sidecar, no device work
        c->host_only = true;
        return c.release();
    }
    BW_CUDA(cudaSetDevice(dev));
    c->sms = sm_count(dev);
    BW_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));

    // Coefficient lists: forward (i, beta) -> (local a, mu[i,beta,a]); transpose (j, a) -> (local beta, mu[j,beta,a]).
    const cyclic::CharMap a0 = cyclic::build_char_map(inst.weight_a0, inst.r);
    const cyclic::CharMap a1 = cyclic::build_char_map(inst.weight_a1, inst.r);
    std::vector<uint32_t> fl_off(inst.n * inst.n + 1), tl_off(inst.n * inst.genus + 1);
    std::vector<int32_t> fl, tl;
    auto pack = [&](int local, uint32_t mu) {
        const int32_t b = ::bw::to_balanced(mu, c->mod);
        return static_cast<int32_t>((static_cast<uint32_t>(local) << 16) | (static_cast<uint32_t>(b) & 0xFFFFu));
    };
    for (size_t i = 0; i < inst.n; ++i)
        for (size_t beta = 0; beta < inst.n; ++beta) {
            fl_off[i * inst.n + beta] = static_cast<uint32_t>(fl.size());
            const uint32_t q = static_cast<uint32_t>((inst.weight_a1[beta] + inst.r - inst.weight_v[i] % inst.r) % inst.r);
            for (uint32_t idx = a0.offsets[q]; idx < a0.offsets[q + 1]; ++idx) {
                const uint32_t mu = inst.mu_at(i, beta, a0.indices[idx]);
                if (mu) fl.push_back(pack(static_cast<int>(idx - a0.offsets[q]), mu));
            }
        }
    fl_off[inst.n * inst.n] = static_cast<uint32_t>(fl.size());
    for (size_t j = 0; j < inst.n; ++j)
        for (size_t a = 0; a < inst.genus; ++a) {
            tl_off[j * inst.genus + a] = static_cast<uint32_t>(tl.size());
            const uint32_t q = static_cast<uint32_t>((inst.weight_a0[a] + inst.weight_v[j]) % inst.r);
            for (uint32_t idx = a1.offsets[q]; idx < a1.offsets[q + 1]; ++idx) {
                const uint32_t mu = inst.mu_at(j, a1.indices[idx], a);
                if (mu) tl.push_back(pack(static_cast<int>(idx - a1.offsets[q]), mu));
            }
        }
    tl_off[inst.n * inst.genus] = static_cast<uint32_t>(tl.size());

    // Most products any kernel sums into one output (the reference's
    // eliminated_accumulation_terms, cuda/cuprym_cyclic.cu:1080-1121, extended
    // to the folded target preconditioner); int32 sums are exact when
    // terms * ((p-1)/2)^2 + 2p < 2^31.
    {
        const cyclic::CharMap km = cyclic::build_char_map(inst.kernel_weights, inst.r);
        const uint64_t ma0 = a0.max_block(), ma1 = a1.max_block(), mk = km.max_block();
        uint64_t spmv = 0;
        for (size_t i = 0; i + 1 < c->precond.row_ptr.size(); ++i)
            spmv = std::max<uint64_t>(spmv, c->precond.row_ptr[i + 1] - c->precond.row_ptr[i]);
        c->max_terms = std::max({es.dm.row_width * ma0, es.d2.row_width * ma0, mk + ma1, spmv,
                                 es.d2.column_width * ma1, ma0, es.dm.column_width * ma1, uint64_t{1}});
        const uint64_t half = (c->p - 1) / 2;
        c->small = c->max_terms * half * half + 2ull * c->p < (1ull << 31);
    }

    ElimDev& E = c->E;
    E.mod = c->mod;
    E.n = static_cast<int>(inst.n);
    E.g = static_cast<int>(inst.genus);
    E.kdim = static_cast<int>(inst.kernel_dim());
    E.x_cols = es.x_cols;
    E.z_cols = es.z_cols;
    E.t_rows = es.t_rows;
    E.y_rows = es.y_rows;
    E.n_r = es.target_rows;
    E.dm_row_width = static_cast<uint32_t>(es.dm.row_width);
    E.dm_col_width = static_cast<uint32_t>(es.dm.column_width);
    E.d2_row_width = static_cast<uint32_t>(es.d2.row_width);
    E.d2_col_width = static_cast<uint32_t>(es.d2.column_width);
    E.base_cols = c->base_cols;
    E.kept_cols = c->kept_cols;
    E.drop0 = c->drop.size() > 0 ? static_cast<long long>(c->drop[0]) : -1;
    E.drop1 = c->drop.size() > 1 ? static_cast<long long>(c->drop[1]) : -1;
    E.n_extra = static_cast<int>(c->dense.columns);
    E.dense_sign = op == "augmented" ? -1 : 1;
    E.dense = deformation ? c->upload(balanced(c->dense.values, c->mod)) : nullptr;
    // Subset-major gathers where the sector fits their format, else the
    // generic row kernels and their tables.
    c->setup_subset_path();
    if (!c->subset_path) {
        E.t_off = c->upload(es.dm_layout.row_offsets);
        E.t_beta = c->upload(es.dm_layout.row_beta);
        E.t_sub = c->upload(es.dm_layout.row_subset);
        E.x_off = c->upload(es.dm_layout.col_offsets);
        E.x_sub = c->upload(es.dm_layout.col_subset);
        E.x_a = c->upload(es.dm_layout.col_a);
        E.dm_row_inc = c->upload(pack_incidence(es.dm.row_col, es.dm.row_i, es.dm.row_neg));
        E.dm_col_inc = c->upload(pack_incidence(es.dm.col_row, es.dm.col_i, es.dm.col_neg));
        E.y_off = c->upload(es.d2_layout.col_offsets);
        E.y_sub = c->upload(es.d2_layout.col_subset);
        E.y_a = c->upload(es.d2_layout.col_a);
        E.u_off = c->upload(es.d2_layout.row_offsets);
        E.u_sub = c->upload(es.d2_layout.row_subset);
        E.u_beta = c->upload(es.d2_layout.row_beta);
        E.d2_row_inc = c->upload(pack_incidence(es.d2.row_col, es.d2.row_i, es.d2.row_neg));
        E.d2_col_inc = c->upload(pack_incidence(es.d2.col_row, es.d2.col_i, es.d2.col_neg));
        E.z_off = c->upload(es.z_layout.offsets);
        E.z_sub = c->upload(es.z_layout.subset);
        E.z_k = c->upload(es.z_layout.index);
        E.fl_off = c->upload(fl_off);
        E.fl = c->upload(fl);
        E.tl_off = c->upload(tl_off);
        E.tl = c->upload(tl);
        E.R = c->upload(balanced(inst.right_inverse, c->mod));
        E.Bk = c->upload(balanced(inst.kernel_basis, c->mod));
    }
    c->d_dc = c->upload(balanced(c->col_precond, c->mod));
    if (!c->subset_path) {
        c->d_p_ptr = c->upload(c->precond.row_ptr);
        c->d_p_col = c->upload(c->precond.col);
        c->d_p_val = c->upload(balanced(c->precond.val, c->mod));
    }

    const size_t nc = ncols, v = num_v;
    c->d_b = c->alloc<int32_t>(nc * v);
    c->d_d = c->alloc<int32_t>(nc * v);
    if (!c->subset_path) {
        c->d_xs = c->alloc<int32_t>((c->base_cols + c->dense.columns) * v);
        c->d_y = c->alloc<int32_t>(std::max<size_t>(es.y_rows, 1) * v);
        c->d_t = c->alloc<int32_t>(std::max<size_t>(es.t_rows, 1) * v);
        c->d_h = c->alloc<int32_t>(std::max<size_t>(es.y_rows, 1) * v);
    }
    c->d_u = c->alloc<int32_t>(std::max<size_t>(es.target_rows, 1) * v);
    c->d_u2 = c->alloc<int32_t>(std::max<size_t>(es.target_rows, 1) * v);
    c->gram_grid = static_cast<unsigned>(std::max<size_t>(1, std::min<size_t>((nc + kThreads - 1) / kThreads,
                                                                                static_cast<size_t>(c->sms) * 8)));
    c->d_partials = c->alloc<int32_t>(20);   // grid-sum accumulators (zero between launches)
    BW_CUDA(cudaMemsetAsync(c->d_partials, 0, 20 * sizeof(int32_t), c->stream));
    c->d_counter = c->alloc<unsigned int>(1);
    if (deformation) {
        c->dense_grid = static_cast<unsigned>(std::max<size_t>(
            1, std::min<size_t>((es.target_rows + kThreads - 1) / kThreads, static_cast<size_t>(c->sms) * 2)));
        c->d_dpart = c->alloc<int32_t>(8);
        BW_CUDA(cudaMemsetAsync(c->d_dpart, 0, 8 * sizeof(int32_t), c->stream));
        c->d_dcounter = c->alloc<unsigned int>(1);
        BW_CUDA(cudaMemsetAsync(c->d_dcounter, 0, sizeof(unsigned int), c->stream));
    }
    c->d_seq_index = c->alloc<unsigned long long>(1);
    BW_CUDA(cudaMemsetAsync(c->d_counter, 0, sizeof(unsigned int), c->stream));
    BW_CUDA(cudaMemsetAsync(c->d_seq_index, 0, sizeof(unsigned long long), c->stream));
    // the initial block (canonical -> balanced)
    uint32_t* tmp = c->upload(c->initial_block);
    c->to_balanced(tmp, c->d_b, nc * v);
    BW_CUDA(cudaStreamSynchronize(c->stream));
    return c.release();
}

void CyclicCtx::to_balanced(const uint32_t* in, int32_t* out, size_t count) {
    if (out == xs_for) xs_for = nullptr;
    cyc_to_balanced_kernel<<<grid_for(count), kThreads, 0, stream>>>(in, out, static_cast<long long>(count), mod);
    BW_CHECK_LAUNCH();
    ++launches;
}

void CyclicCtx::to_canonical(const int32_t* in, uint32_t* out, size_t count) {
    cyc_to_canonical_kernel<<<grid_for(count), kThreads, 0, stream>>>(in, out, static_cast<long long>(count), mod);
    BW_CHECK_LAUNCH();
    ++launches;
}

void CyclicCtx::forward(const int32_t* in, int32_t* u, bool precondition) {
    if (subset_path) {
        subset_source16(in, precondition ? d_dc : nullptr);
        subset_forward16();
        subset_u_from_walk(u);
        return;
    }
    cyc_source_kernel<<<grid_for(base_cols + dense.columns), kThreads, 0, stream>>>(E, in, precondition ? d_dc : nullptr,
                                                                                    d_xs);
    BW_CHECK_LAUNCH();
    if (small) {
        cyc_dm_forward_kernel<true><<<grid_for(es.t_rows), kThreads, 0, stream>>>(E, d_xs, d_t);
        cyc_elim_y_kernel<true><<<grid_for(es.y_rows), kThreads, 0, stream>>>(E, d_xs, d_t, d_y);
        cyc_d2_forward_kernel<true><<<grid_for(es.target_rows), kThreads, 0, stream>>>(E, d_y, d_xs, u);
    } else {
        cyc_dm_forward_kernel<false><<<grid_for(es.t_rows), kThreads, 0, stream>>>(E, d_xs, d_t);
        cyc_elim_y_kernel<false><<<grid_for(es.y_rows), kThreads, 0, stream>>>(E, d_xs, d_t, d_y);
        cyc_d2_forward_kernel<false><<<grid_for(es.target_rows), kThreads, 0, stream>>>(E, d_y, d_xs, u);
    }
    BW_CHECK_LAUNCH();
    launches += 4;
}

void CyclicCtx::backward(const int32_t* u2, int32_t* out, bool precondition) {
    const int32_t* dc = precondition ? d_dc : nullptr;
    if (subset_path) {
        subset_pack_u(u2, d_u2_16);
        subset_backward16(dc, out, false);
        return;
    }
    const size_t tz = es.t_rows + es.z_cols;
    if (small) {
        cyc_d2_transpose_kernel<true><<<grid_for(es.y_rows), kThreads, 0, stream>>>(E, u2, d_h);
        cyc_adjoint_t_z_kernel<true><<<grid_for(tz), kThreads, 0, stream>>>(E, d_h, dc, d_t, out);
        cyc_dm_transpose_kernel<true><<<grid_for(es.x_cols), kThreads, 0, stream>>>(E, d_t, dc, out);
    } else {
        cyc_d2_transpose_kernel<false><<<grid_for(es.y_rows), kThreads, 0, stream>>>(E, u2, d_h);
        cyc_adjoint_t_z_kernel<false><<<grid_for(tz), kThreads, 0, stream>>>(E, d_h, dc, d_t, out);
        cyc_dm_transpose_kernel<false><<<grid_for(es.x_cols), kThreads, 0, stream>>>(E, d_t, dc, out);
    }
    BW_CHECK_LAUNCH();
    launches += 3;
    if (E.n_extra) {
        cyc_dense_t_kernel<<<dense_grid, kThreads, 0, stream>>>(E, u2, dc, out, d_dpart, d_dcounter);
        BW_CHECK_LAUNCH();
        ++launches;
    }
}

void CyclicCtx::target_precondition(const int32_t* u, int32_t* u2) {
    if (subset_path) {
        subset_u_to_walk(u);
        subset_precondition16();
        subset_unpack_u(d_u2_16, u2);
        return;
    }
    if (small)
        cyc_spmv_kernel<true><<<grid_for(es.target_rows), kThreads, 0, stream>>>(
            d_p_ptr, d_p_col, d_p_val, u, u2, static_cast<long long>(es.target_rows), mod);
    else
        cyc_spmv_kernel<false><<<grid_for(es.target_rows), kThreads, 0, stream>>>(
            d_p_ptr, d_p_col, d_p_val, u, u2, static_cast<long long>(es.target_rows), mod);
    BW_CHECK_LAUNCH();
    ++launches;
}

void CyclicCtx::apply_square(const int32_t* in, int32_t* out) {
    if (subset_path) {   // padded int16 internals end to end
        if (xs_for != in) subset_source16(in, d_dc);   // else the previous backward wrote it
        subset_forward16();
        subset_precondition16();
        subset_backward16(d_dc, out, true);
        return;
    }
    forward(in, d_u, true);
    target_precondition(d_u, d_u2);
    backward(d_u2, out, true);
}

void CyclicCtx::gram(const int32_t* a1, const int32_t* c1, const int32_t* a2, const int32_t* c2, int count) {
    launch_pdl(cyc_gram_kernel, gram_grid, 0, a1, c1, a2 ? a2 : a1, c2 ? c2 : c1, count,
               static_cast<long long>(op_cols), d_partials, d_counter, d_seq, d_seq_index, mod);
    BW_CHECK_LAUNCH();
    ++launches;
}

// One round of the reference's loop (cuda/cuprym_cyclic.cu:2443-2449):
// D = S B; push B^t D, D^t D; B = S D; push B^t D, B^t B.
void CyclicCtx::round() {
    apply_square(d_b, d_d);
    gram(d_b, d_d, d_d, d_d, 2);
    apply_square(d_d, d_b);
    gram(d_b, d_d, d_b, d_b, 2);
}

void CyclicCtx::generate(size_t nlen_target, float* device_ms) {
    const size_t nc = op_cols;
    const size_t default_nlen = (2 * nc) / num_v + 50;
    const size_t max_nlen = nlen_target == 0 ? default_nlen : nlen_target;
    const size_t rounds = (max_nlen - 1 + 3) / 4;
    seq_capacity = max_nlen + 5;
    if (!d_seq || seq_alloc < seq_capacity) {
        d_seq = alloc<uint32_t>(seq_capacity * 10);
        seq_alloc = seq_capacity;
        for (auto& g : graphs)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
    }
    BW_CUDA(cudaMemsetAsync(d_seq_index, 0, sizeof(unsigned long long), stream));
    BW_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(unsigned int), stream));
    // restart from the initial block
    uint32_t* tmp = scratch_canonical();
    BW_CUDA(cudaMemcpyAsync(tmp, initial_block.data(), nc * num_v * 4, cudaMemcpyHostToDevice, stream));
    to_balanced(tmp, d_b, nc * num_v);
    gram(d_b, d_b, nullptr, nullptr, 1);
    // the first application's source, outside the round graph: every later
    // source is written by the backward kernels of the application before
    if (subset_path && rounds > 0) subset_source16(d_b, d_dc);
    if (rounds > 0) {
        if (!graphs[0]) {
            const uint64_t l0 = launches;
            cudaGraph_t graph;
            BW_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            try {
                round();
            } catch (...) {
                cudaStreamEndCapture(stream, &graph);
                throw;
            }
            BW_CUDA(cudaStreamEndCapture(stream, &graph));
            graph_kernels = launches - l0;
            launches = l0;
            BW_CUDA(cudaGraphInstantiate(&graphs[0], graph, 0));
            cudaGraphDestroy(graph);
        }
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (device_ms) {
            BW_CUDA(cudaEventCreate(&e0));
            BW_CUDA(cudaEventCreate(&e1));
            BW_CUDA(cudaEventRecord(e0, stream));
        }
        for (size_t r = 0; r < rounds; ++r) {
            BW_CUDA(cudaGraphLaunch(graphs[0], stream));
            launches += graph_kernels;
        }
        if (device_ms) {
            BW_CUDA(cudaEventRecord(e1, stream));
            BW_CUDA(cudaEventSynchronize(e1));
            BW_CUDA(cudaEventElapsedTime(device_ms, e0, e1));
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
        }
    } else if (device_ms) {
        *device_ms = 0;
    }
    seq_len = 1 + 4 * rounds;
    BW_CUDA(cudaStreamSynchronize(stream));
}

uint32_t* CyclicCtx::scratch_canonical() {
    if (!d_canon) d_canon = alloc<uint32_t>(std::max<size_t>(op_cols, es.target_rows) * num_v);
    return d_canon;
}

void CyclicCtx::download_state(std::vector<uint32_t>& current, std::vector<uint32_t>& packed) {
    const size_t nc = op_cols;
    uint32_t* tmp = scratch_canonical();
    to_canonical(d_b, tmp, nc * num_v);
    current.resize(nc * num_v);
    packed.resize(seq_len * 10);
    BW_CUDA(cudaMemcpyAsync(current.data(), tmp, current.size() * 4, cudaMemcpyDeviceToHost, stream));
    BW_CUDA(cudaMemcpyAsync(packed.data(), d_seq, packed.size() * 4, cudaMemcpyDeviceToHost, stream));
    BW_CUDA(cudaStreamSynchronize(stream));
}

// Host-buffer operator applications (validation and tests).
void CyclicCtx::apply_host(int what, const uint32_t* in, uint32_t* out) {
    const size_t nc = op_cols, nr = es.target_rows, v = num_v;
    uint32_t* tmp = scratch_canonical();
    if (what == BW_CYCLIC_APPLY_SQUARE || what == BW_CYCLIC_APPLY_FORWARD) {
        BW_CUDA(cudaMemcpyAsync(tmp, in, nc * v * 4, cudaMemcpyHostToDevice, stream));
        to_balanced(tmp, d_d, nc * v);
        if (what == BW_CYCLIC_APPLY_SQUARE) {
            apply_square(d_d, d_d);   // in place is safe: the first kernel copies into d_xs
            to_canonical(d_d, tmp, nc * v);
            BW_CUDA(cudaMemcpyAsync(out, tmp, nc * v * 4, cudaMemcpyDeviceToHost, stream));
        } else {
            forward(d_d, d_u, false);
            to_canonical(d_u, tmp, nr * v);
            BW_CUDA(cudaMemcpyAsync(out, tmp, nr * v * 4, cudaMemcpyDeviceToHost, stream));
        }
    } else if (what == BW_CYCLIC_APPLY_TRANSPOSE) {
        BW_CUDA(cudaMemcpyAsync(tmp, in, nr * v * 4, cudaMemcpyHostToDevice, stream));
        to_balanced(tmp, d_u2, nr * v);
        backward(d_u2, d_d, false);
        to_canonical(d_d, tmp, nc * v);
        BW_CUDA(cudaMemcpyAsync(out, tmp, nc * v * 4, cudaMemcpyDeviceToHost, stream));
    } else if (what == BW_CYCLIC_APPLY_SQUARE_UNFOLDED) {
        // The reference's order of operations for the target preconditioner:
        // rowmix rounds, Dr, transposed rounds in reverse (validation of the folded P).
        BW_CUDA(cudaMemcpyAsync(tmp, in, nc * v * 4, cudaMemcpyHostToDevice, stream));
        to_balanced(tmp, d_d, nc * v);
        forward(d_d, d_u, true);
        if (plan.rounds > 0) {
            if (!d_pairs) {
                std::vector<uint32_t> flat;
                for (const auto& round : plan.round_pairs) {
                    pair_offsets.push_back(flat.size() / 3);
                    for (const auto& pr : round) {
                        flat.push_back(pr.first);
                        flat.push_back(pr.second);
                        flat.push_back(static_cast<uint32_t>(pr.a) | (static_cast<uint32_t>(pr.b) << 16));
                    }
                }
                pair_offsets.push_back(flat.size() / 3);
                d_pairs = upload(flat);
                d_dr = upload(balanced(row_precond, mod));
            }
            for (size_t r = 0; r < plan.rounds; ++r) {
                const long long cnt = static_cast<long long>(pair_offsets[r + 1] - pair_offsets[r]);
                cyc_rowmix_kernel<<<grid_for(cnt), kThreads, 0, stream>>>(d_pairs + 3 * pair_offsets[r], cnt, d_u,
                                                                          false, mod);
                BW_CHECK_LAUNCH();
            }
            cyc_scale_kernel<<<grid_for(nr), kThreads, 0, stream>>>(d_u, d_dr, d_u2, static_cast<long long>(nr), mod);
            BW_CHECK_LAUNCH();
            for (size_t r = plan.rounds; r > 0; --r) {
                const long long cnt = static_cast<long long>(pair_offsets[r] - pair_offsets[r - 1]);
                cyc_rowmix_kernel<<<grid_for(cnt), kThreads, 0, stream>>>(d_pairs + 3 * pair_offsets[r - 1], cnt,
                                                                          d_u2, true, mod);
                BW_CHECK_LAUNCH();
            }
        } else {
            target_precondition(d_u, d_u2);
        }
        backward(d_u2, d_d, true);
        to_canonical(d_d, tmp, nc * v);
        BW_CUDA(cudaMemcpyAsync(out, tmp, nc * v * 4, cudaMemcpyDeviceToHost, stream));
    } else {
        throw Error("unknown application kind", 1);
    }
    BW_CUDA(cudaStreamSynchronize(stream));
}

}  // namespace bw
