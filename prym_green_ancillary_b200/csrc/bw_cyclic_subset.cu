// Subset-major paper-mode operator: the four Koszul gathers of the eliminated
// operator with one thread per subset, on 16-bit vectors in padded blocks.
//
// Every character block of the shipped instances has at most two rows (A0
// blocks two, A1 blocks one or two, kernel-weight blocks at most one), and
// the rows of one subset's block read the same neighbour blocks with
// different coefficients.  So:
//   * the internal vectors (scaled source x, y, u, u2, t_adj) hold balanced
//     residues as int16 and give every subset's block two row slots: a block
//     is one aligned 16-byte load, found from the subset's rank alone;
//   * one thread takes a subset, loads each incidence word (neighbour rank,
//     generator, sign) and each neighbour block once, and accumulates both
//     rows of its own block;
//   * the signed coefficients of mu for (sign, generator, own character) are
//     four int32 in shared memory: one 16-byte load per incidence, indexed by
//     the code the incidence word carries (sign * n + generator).
// An incidence thus costs one coalesced word, one 16-byte load, one 16-byte
// shared load and sixteen multiply-adds.
//
// Two of the reference's kernel pairs are fused, with their intermediates in
// registers:
//   * D_m forward (cuda/cyclic_cuda_helpers.h:145-204) with the elimination
//     y = B z - R t (cyclic_elim_z_to_y_kernel, cyclic_elim_subtract_Rt_kernel,
//     :718-791): t never reaches memory;
//   * D_(m-1) transpose (:206-266) with t_adj = R^t h, z_adj = B^t h and the
//     z part of the adjoint assembly (cyclic_elim_RT_h_kernel,
//     cyclic_elim_BT_h_kernel, cyclic_elim_assemble_adjoint_kernel, :793-895):
//     h never reaches memory.
// The folded target preconditioner runs in ELL form with int16 values; it
// reads u kept in an order with row-mixing partners adjacent (so a row's
// sixteen columns lie within nine consecutive rows) and writes u2 in the
// padded subset layout.  The operator's inputs and outputs (the block B,
// S B) stay compact int32; results are the same canonical residues as the
// generic row kernels of bw_cyclic.cu, which remain for instances outside
// this format.
#include "bw_cyclic.cuh"
#include "bw_cyclic_dev.cuh"

#include <algorithm>

namespace bw {

namespace {

constexpr int kThreads = 256;
constexpr uint32_t kLow26 = (1u << 26) - 1;

using cyc::Acc4;
using cyc::ld4;
using cyc::neg4;
using cyc::scale4;
using cyc::st4;

// ----- 16-bit rows: 4 columns in 8 bytes, a block of two rows in 16
__device__ __forceinline__ uint32_t pack2(int32_t a, int32_t b) {
    return (static_cast<uint32_t>(a) & 0xFFFFu) | (static_cast<uint32_t>(b) << 16);
}
__device__ __forceinline__ int32_t lo16(uint32_t w) { return static_cast<int16_t>(w & 0xFFFFu); }
__device__ __forceinline__ int32_t hi16(uint32_t w) { return static_cast<int32_t>(w) >> 16; }
__device__ __forceinline__ uint2 pack_row(const int4& v) { return make_uint2(pack2(v.x, v.y), pack2(v.z, v.w)); }
__device__ __forceinline__ int4 unpack_row(uint32_t a, uint32_t b) { return make_int4(lo16(a), hi16(a), lo16(b), hi16(b)); }
__device__ __forceinline__ void st_block(uint4* v, uint32_t s, const int4& r0, const int4& r1) {
    const uint2 a = pack_row(r0), b = pack_row(r1);
    v[s] = make_uint4(a.x, a.y, b.x, b.y);
}

// Views of the staged shared-memory tables.
struct Tables {
    const int4* coef;
    const int32_t *R, *B, *a0off, *a0idx, *a1off, *a1idx, *koff, *kidx, *ych;
};

// Staging reads only the constant tables, so it overlaps the end of the kernel
// before (programmatic dependent launch); the wait follows it.
__device__ __forceinline__ Tables stage(const SubsetDev& D, const int32_t* __restrict__ blob, int32_t* sm) {
    cyc::pdl_trigger();
    for (int w = threadIdx.x; w < D.blob_words; w += blockDim.x) sm[w] = __ldg(blob + w);
    __syncthreads();
    cyc::pdl_wait();
    Tables t;
    t.coef = reinterpret_cast<const int4*>(sm);
    t.R = sm + D.o_R;
    t.B = sm + D.o_B;
    t.a0off = sm + D.o_a0off;
    t.a0idx = sm + D.o_a0idx;
    t.a1off = sm + D.o_a1off;
    t.a1idx = sm + D.o_a1idx;
    t.koff = sm + D.o_koff;
    t.kidx = sm + D.o_kidx;
    t.ych = sm + D.o_ych;
    return t;
}

// Streamed table words: evict-first when the sector's tables exceed the L2
// (they would only push the gathered vector out), cached otherwise (small
// sectors keep tables and vectors in L2 from one application to the next).
template <bool STREAM, class T>
__device__ __forceinline__ T ld_table(const T* p) {
    if constexpr (STREAM)
        return __ldcs(p);
    else
        return __ldg(p);
}

// acc_k += c_k0 * row0 + c_k1 * row1 for the neighbour block b (two int16
// rows) and c = (c_00, c_01, c_10, c_11).
template <bool SMALL>
__device__ __forceinline__ void mac_block(const int4& c, const uint4& b, Acc4<SMALL>& acc0, Acc4<SMALL>& acc1) {
    const int4 r0 = unpack_row(b.x, b.y), r1 = unpack_row(b.z, b.w);
    acc0.mac(c.x, r0);
    acc0.mac(c.y, r1);
    acc1.mac(c.z, r0);
    acc1.mac(c.w, r1);
}

// Both rows of subset s against its `width` neighbour blocks.  The coefficient
// table is [code = sign * n + generator][own character]; a neighbour block with
// one row has zero coefficients for its second slot (which holds zeros).
// Incidence words are read once per application (ld_table).  `nin` is the
// number of blocks of `in`, which carries one more, all-zero block at nin.
template <bool SMALL, bool STREAM>
__device__ __forceinline__ void gather_block(const uint32_t* __restrict__ inc, uint32_t nsub, uint32_t s,
                                             uint32_t width, const int4* coef, int r, int ch,
                                             const uint4* __restrict__ in, uint32_t nin, Acc4<SMALL>& acc0,
                                             Acc4<SMALL>& acc1) {
    // Chunks of four incidences: a chunk's blocks are loaded together, and
    // the next chunk's words while those blocks are in flight.  Only the
    // words of a last, partial chunk are loaded under a mask; its empty slots
    // hold the zero block (code 0), so the products run unmasked.
    constexpr int U = 4;
    const uint32_t* p = inc + s;
    const size_t step = nsub;
    const uint32_t full = width / U, rem = width % U, chunks = full + (rem ? 1u : 0u);
    auto words = [&](uint32_t k, uint32_t (&w)[U]) {
        const uint32_t* q = p + static_cast<size_t>(k) * U * step;
        if (k < full) {
#pragma unroll
            for (int u = 0; u < U; ++u) w[u] = ld_table<STREAM>(q + u * step);
        } else {
#pragma unroll
            for (int u = 0; u < U; ++u) w[u] = static_cast<uint32_t>(u) < rem ? ld_table<STREAM>(q + u * step) : nin;
        }
    };
    uint32_t e[U];
    if (chunks == 0) return;
    words(0, e);
    for (uint32_t k = 0; k < chunks; ++k) {
        uint4 b[U];
#pragma unroll
        for (int u = 0; u < U; ++u) b[u] = __ldg(in + (e[u] & kLow26));
        uint32_t next[U];
        if (k + 1 < chunks) words(k + 1, next);
#pragma unroll
        for (int u = 0; u < U; ++u) mac_block<SMALL>(coef[static_cast<int>(e[u] >> 26) * r + ch], b[u], acc0, acc1);
        if (k + 1 < chunks) {
#pragma unroll
            for (int u = 0; u < U; ++u) e[u] = next[u];
        }
    }
}

#define BW_ITEMS(var, count)                                                                         \
    for (long long var = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; var < (count); \
         var += static_cast<long long>(gridDim.x) * blockDim.x)

// Scaled source: items [0, n0) are m-subsets, whose x block (compact rows
// x_off, x_off + 1 of the operator column op_col, times dc) goes to the padded
// xs; items n0 + j are the compact z rows and the extra dense columns (int32).
__global__ void __launch_bounds__(kThreads) sub_source_kernel(SubsetDev D, const int32_t* __restrict__ in,
                                                              const int32_t* __restrict__ dc, uint4* __restrict__ xs,
                                                              int32_t* __restrict__ zs) {
    extern __shared__ int32_t sm[];
    const Tables T = stage(D, D.blob_f, sm);
    const long long n0 = D.n0, total = n0 + static_cast<long long>(D.z_cols) + D.n_extra;
    BW_ITEMS(item, total) {
        if (item < n0) {
            const uint32_t dx = __ldg(D.m0 + item);
            const int xch = static_cast<int>(dx >> 26);
            const int nx = T.a0off[xch + 1] - T.a0off[xch];
            int4 r[2] = {make_int4(0, 0, 0, 0), make_int4(0, 0, 0, 0)};
            for (int q = 0; q < nx; ++q) {
                const long long c = cyc::op_col(D.drop0, D.drop1, static_cast<long long>(dx & kLow26) + q);
                if (c < 0) continue;   // dropped base column (replacement): zero
                const int4 v = ld4(in, c);
                r[q] = dc ? scale4(v, __ldg(dc + c), D.mod) : v;
            }
            st_block(xs, static_cast<uint32_t>(item), r[0], r[1]);
        } else {
            const long long zq = item - n0;
            const long long src = zq < static_cast<long long>(D.z_cols)
                                      ? cyc::op_col(D.drop0, D.drop1, static_cast<long long>(D.x_cols) + zq)
                                      : static_cast<long long>(D.kept_cols) + (zq - static_cast<long long>(D.z_cols));
            int4 v = make_int4(0, 0, 0, 0);
            if (src >= 0) {
                v = ld4(in, src);
                if (dc) v = scale4(v, __ldg(dc + src), D.mod);
            }
            st4(zs, zq, v);
        }
    }
}

// (m-1)-subset S: its t rows t(S, beta) = (D_m xs)(S, beta), then its y block
//   y(S, a) = sum_kappa B[a,kappa] zs(S, kappa) - sum_beta R[a,beta] t(S, beta).
template <bool SMALL, bool STREAM>
__global__ void __launch_bounds__(kThreads) sub_dm_forward_elim_kernel(SubsetDev D, const uint4* __restrict__ xs,
                                                                       const int32_t* __restrict__ zs,
                                                                       uint4* __restrict__ y) {
    extern __shared__ int32_t sm[];
    const Tables T = stage(D, D.blob_f, sm);
    BW_ITEMS(item, D.n1) {
        const uint32_t s = static_cast<uint32_t>(item);
        const uint32_t d = __ldg(D.m1 + s);
        const int tch = static_cast<int>(d >> 26), ych = T.ych[tch];
        const int ya = T.a0off[ych], ny = T.a0off[ych + 1] - ya;
        int4 out[2] = {make_int4(0, 0, 0, 0), make_int4(0, 0, 0, 0)};
        if (ny > 0) {
            const int tb = T.a1off[tch], nt = T.a1off[tch + 1] - tb;
            int4 t0 = make_int4(0, 0, 0, 0), t1 = t0;
            if (nt > 0) {
                Acc4<SMALL> acc0, acc1;
                gather_block<SMALL, STREAM>(D.inc_dmf, D.n1, s, D.w_dmf, T.coef, D.r, tch, xs, D.n0, acc0, acc1);
                t0 = acc0.reduce(D.mod);
                t1 = acc1.reduce(D.mod);
            }
            const int beta0 = nt > 0 ? T.a1idx[tb] : 0, beta1 = nt > 1 ? T.a1idx[tb + 1] : beta0;
            const int kb = T.koff[ych], nz = T.koff[ych + 1] - kb;
            int4 z0 = make_int4(0, 0, 0, 0), z1 = z0;
            if (nz > 0) {
                const long long zr = d & kLow26;
                z0 = ld4(zs, zr);
                if (nz > 1) z1 = ld4(zs, zr + 1);
            }
            for (int q = 0; q < ny; ++q) {
                const int a = T.a0idx[ya + q];
                Acc4<SMALL> acc;
                if (nz > 0) acc.mac(T.B[a * D.kdim + T.kidx[kb]], z0);
                if (nz > 1) acc.mac(T.B[a * D.kdim + T.kidx[kb + 1]], z1);
                if (nt > 0) acc.mac(-T.R[a * D.n + beta0], t0);
                if (nt > 1) acc.mac(-T.R[a * D.n + beta1], t1);
                out[q] = acc.reduce(D.mod);
            }
        }
        st_block(y, s, out[0], out[1]);
    }
}

// (m-2)-subset S2: its u rows u(S2, beta) = (D_(m-1) y)(S2, beta), plus
// dense_sign * dense zs_extra for the deformation variants (|terms| stay below
// 2^31: a balanced residue plus two products of balanced residues), each
// written to its position u_pos in the row-mixing locality order.
template <bool SMALL, bool STREAM>
__global__ void __launch_bounds__(kThreads) sub_d2_forward_kernel(SubsetDev D, const uint4* __restrict__ y,
                                                                  const int32_t* __restrict__ zs,
                                                                  uint2* __restrict__ u) {
    extern __shared__ int32_t sm[];
    const Tables T = stage(D, D.blob_f, sm);
    BW_ITEMS(item, D.n2) {
        const uint32_t s = static_cast<uint32_t>(item);
        const uint32_t d = __ldg(D.m2 + s);
        const int uch = static_cast<int>(d >> 26);
        const int nu = T.a1off[uch + 1] - T.a1off[uch];
        const long long urow = d & kLow26;
        int4 out[2] = {make_int4(0, 0, 0, 0), make_int4(0, 0, 0, 0)};
        if (nu > 0) {
            Acc4<SMALL> acc0, acc1;
            gather_block<SMALL, STREAM>(D.inc_d2f, D.n2, s, D.w_d2f, T.coef, D.r, uch, y, D.n1, acc0, acc1);
            out[0] = acc0.reduce(D.mod);
            if (nu > 1) out[1] = acc1.reduce(D.mod);
            if (D.n_extra) {
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    if (q >= nu) break;
                    int4 v = out[q];
                    for (int j = 0; j < D.n_extra; ++j) {
                        const int32_t c = D.dense_sign * __ldg(D.dense + (urow + q) * D.n_extra + j);
                        const int4 e = ld4(zs, static_cast<long long>(D.z_cols) + j);
                        v.x += c * e.x;
                        v.y += c * e.y;
                        v.z += c * e.z;
                        v.w += c * e.w;
                    }
                    out[q] = make_int4(reduce_balanced(v.x, D.mod), reduce_balanced(v.y, D.mod),
                                       reduce_balanced(v.z, D.mod), reduce_balanced(v.w, D.mod));
                }
            }
        }
        // rows to their positions in the row-mixing locality order
#pragma unroll
        for (int q = 0; q < 2; ++q)
            if (q < nu) u[__ldg(D.u_pos + urow + q)] = pack_row(out[q]);
    }
}

// u2 = P u for the folded target preconditioner P = T^t Dr T in ELL form
// ([slot][row] over the padded u2 slots, `ell` slots a row, coalesced across
// threads; columns are positions of u in the locality order; empty slots hold
// value 0).  Four slots at a time: their rows are
// gathered together, and the next four slots' words are loaded meanwhile.
template <bool SMALL, bool STREAM>
__global__ void __launch_bounds__(kThreads) sub_ell_kernel(SubsetDev D, const uint2* __restrict__ u,
                                                           uint2* __restrict__ u2) {
    cyc::pdl_trigger();
    cyc::pdl_wait();
    const long long rows = 2 * static_cast<long long>(D.n2);
    BW_ITEMS(row, rows) {
        Acc4<SMALL> acc;
        const uint32_t* c = D.e_col + row;
        const int16_t* v = D.e_val + row;
        uint32_t cc[4];
        int32_t vv[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            cc[q] = ld_table<STREAM>(c + q * rows);
            vv[q] = ld_table<STREAM>(v + q * rows);
        }
        for (uint32_t k = 0; k < D.ell; k += 4) {
            uint2 x[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) x[q] = __ldg(u + cc[q]);
            uint32_t nc[4];
            int32_t nv[4];
            if (k + 4 < D.ell) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    nc[q] = ld_table<STREAM>(c + (k + 4 + q) * rows);
                    nv[q] = ld_table<STREAM>(v + (k + 4 + q) * rows);
                }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) acc.mac(vv[q], unpack_row(x[q].x, x[q].y));
            if (k + 4 < D.ell) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    cc[q] = nc[q];
                    vv[q] = nv[q];
                }
            }
        }
        u2[row] = pack_row(acc.reduce(D.mod));
    }
}

// (m-1)-subset S: its h rows h(S, a) = (D_(m-1)^t u2)(S, a), then
//   t_adj(S, beta) = sum_a R[a,beta] h(S, a)               (padded t block)
//   out_z(S, kappa) = dc * sum_a B[a,kappa] h(S, a)        (compact, through op_col)
// and, with next_zs, the next application's source row dc * out_z (zero for
// a dropped column), so that apply_square needs no source kernel.
template <bool SMALL, bool STREAM>
__global__ void __launch_bounds__(kThreads) sub_d2_transpose_adjoint_kernel(SubsetDev D,
                                                                            const uint4* __restrict__ u2,
                                                                            const int32_t* __restrict__ dc,
                                                                            uint4* __restrict__ t_adj,
                                                                            int32_t* __restrict__ out,
                                                                            int32_t* __restrict__ next_zs) {
    extern __shared__ int32_t sm[];
    const Tables T = stage(D, D.blob_t, sm);
    BW_ITEMS(item, D.n1) {
        const uint32_t s = static_cast<uint32_t>(item);
        const uint32_t d = __ldg(D.m1 + s);
        const int tch = static_cast<int>(d >> 26), ych = T.ych[tch];
        const int ya = T.a0off[ych], ny = T.a0off[ych + 1] - ya;
        const int a0 = ny > 0 ? T.a0idx[ya] : 0, a1 = ny > 1 ? T.a0idx[ya + 1] : a0;
        int4 h0 = make_int4(0, 0, 0, 0), h1 = h0;
        if (ny > 0) {
            Acc4<SMALL> acc0, acc1;
            gather_block<SMALL, STREAM>(D.inc_d2t, D.n1, s, D.w_d2t, T.coef, D.r, ych, u2, D.n2, acc0, acc1);
            h0 = acc0.reduce(D.mod);
            h1 = acc1.reduce(D.mod);
        }
        const int tb = T.a1off[tch], nt = T.a1off[tch + 1] - tb;
        int4 tv[2] = {make_int4(0, 0, 0, 0), make_int4(0, 0, 0, 0)};
        for (int q = 0; q < nt; ++q) {
            const int beta = T.a1idx[tb + q];
            Acc4<SMALL> acc;
            if (ny > 0) acc.mac(T.R[a0 * D.n + beta], h0);
            if (ny > 1) acc.mac(T.R[a1 * D.n + beta], h1);
            tv[q] = acc.reduce(D.mod);
        }
        st_block(t_adj, s, tv[0], tv[1]);
        const int kb = T.koff[ych], nz = T.koff[ych + 1] - kb;
        const long long zq0 = d & kLow26, zfirst = static_cast<long long>(D.x_cols) + zq0;
        for (int q = 0; q < nz; ++q) {
            const long long orow = cyc::op_col(D.drop0, D.drop1, zfirst + q);
            if (orow < 0) {   // dropped base column (replacement)
                if (next_zs) st4(next_zs, zq0 + q, make_int4(0, 0, 0, 0));
                continue;
            }
            const int kap = T.kidx[kb + q];
            Acc4<SMALL> acc;
            if (ny > 0) acc.mac(T.B[a0 * D.kdim + kap], h0);
            if (ny > 1) acc.mac(T.B[a1 * D.kdim + kap], h1);
            const int4 v = acc.reduce(D.mod);
            const int4 o = dc ? scale4(v, __ldg(dc + orow), D.mod) : v;
            st4(out, orow, o);
            if (next_zs) st4(next_zs, zq0 + q, scale4(o, __ldg(dc + orow), D.mod));   // next source row
        }
    }
}

// m-subset S': its x rows out_x(S', a) = -dc * (D_m^t t_adj)(S', a), compact
// through op_col, and, with next_xs, the next application's padded source
// block dc * out_x (as the source kernel would build it from out).
template <bool SMALL, bool STREAM>
__global__ void __launch_bounds__(kThreads) sub_dm_transpose_kernel(SubsetDev D, const uint4* __restrict__ t_adj,
                                                                    const int32_t* __restrict__ dc,
                                                                    int32_t* __restrict__ out,
                                                                    uint4* __restrict__ next_xs) {
    extern __shared__ int32_t sm[];
    const Tables T = stage(D, D.blob_t, sm);
    BW_ITEMS(item, D.n0) {
        const uint32_t s = static_cast<uint32_t>(item);
        const uint32_t d = __ldg(D.m0 + s);
        const int xch = static_cast<int>(d >> 26);
        const int nx = T.a0off[xch + 1] - T.a0off[xch];
        if (nx == 0) continue;
        Acc4<SMALL> acc0, acc1;
        gather_block<SMALL, STREAM>(D.inc_dmt, D.n0, s, D.w_dmt, T.coef, D.r, xch, t_adj, D.n1, acc0, acc1);
        const long long xrow = d & kLow26;
        int4 nxt[2] = {make_int4(0, 0, 0, 0), make_int4(0, 0, 0, 0)};
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            if (q >= nx) break;
            const long long orow = cyc::op_col(D.drop0, D.drop1, xrow + q);
            if (orow < 0) continue;   // dropped base column (replacement): its source slot stays zero
            const int4 v = neg4(q == 0 ? acc0.reduce(D.mod) : acc1.reduce(D.mod));
            const int4 o = dc ? scale4(v, __ldg(dc + orow), D.mod) : v;
            st4(out, orow, o);
            if (next_xs) nxt[q] = scale4(o, __ldg(dc + orow), D.mod);
        }
        if (next_xs) st_block(next_xs, s, nxt[0], nxt[1]);   // next application's source block
    }
}

// Extra source rows of the deformation transpose from the padded u2:
//   out[kept_cols + j][c] = dense_sign * dc[kept_cols + j] * sum_row dense[row][j] u2[row][c]
// Each CTA sums a stripe of padded rows; the CTA sums meet in an 8-entry
// accumulator (cyc::grid_sum) and the last CTA writes the n_extra rows (and,
// with next_zs, their next source rows).
__global__ void __launch_bounds__(kThreads) sub_dense_t_kernel(SubsetDev D, const uint2* __restrict__ u2,
                                                               const int32_t* __restrict__ dc,
                                                               int32_t* __restrict__ out,
                                                               int32_t* __restrict__ partials,
                                                               unsigned int* __restrict__ counter,
                                                               int32_t* __restrict__ next_zs) {
    extern __shared__ int32_t sm[];
    const Tables T = stage(D, D.blob_f, sm);
    int32_t acc[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) acc[e] = 0;
    int cnt = 0;
    BW_ITEMS(row, 2 * static_cast<long long>(D.n2)) {
        const uint32_t d = __ldg(D.m2 + (row >> 1));
        const int uch = static_cast<int>(d >> 26);
        const int q = static_cast<int>(row & 1);
        if (q >= T.a1off[uch + 1] - T.a1off[uch]) continue;   // padding slot
        const long long crow = static_cast<long long>(d & kLow26) + q;
        const uint2 w = __ldg(u2 + row);
        const int4 v = unpack_row(w.x, w.y);
        for (int j = 0; j < D.n_extra; ++j) {
            const int32_t c = __ldg(D.dense + crow * D.n_extra + j);
            acc[4 * j] += c * v.x;
            acc[4 * j + 1] += c * v.y;
            acc[4 * j + 2] += c * v.z;
            acc[4 * j + 3] += c * v.w;
        }
        if (++cnt == 8) {   // 8 products of balanced residues stay below 2^31
            cnt = 0;
#pragma unroll
            for (int e = 0; e < 8; ++e) acc[e] = reduce_partial(acc[e], D.mod);
        }
    }
    __shared__ int32_t red[kThreads / 32][8];
    __shared__ bool am_last;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        int32_t v = reduce_balanced(acc[e], D.mod);
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (lane == 0) red[warp][e] = reduce_balanced(v, D.mod);
    }
    __syncthreads();
    int32_t mine = 0, total = 0;
    if (threadIdx.x < 8) {
        for (int w = 0; w < kThreads / 32; ++w) mine += red[w][threadIdx.x];
        mine = reduce_balanced(mine, D.mod);
    }
    if (!cyc::grid_sum(partials, counter, 8, mine, total, &am_last)) return;
    if (threadIdx.x < 4 * D.n_extra) {
        const int j = threadIdx.x / 4, c = threadIdx.x % 4;
        const long long orow = static_cast<long long>(D.kept_cols) + j;
        int32_t v = D.dense_sign * reduce_balanced(total, D.mod);
        if (dc) v = reduce_balanced(v * __ldg(dc + orow), D.mod);
        out[orow * 4 + c] = v;
        if (next_zs)   // next application's source row of extra column j
            next_zs[(static_cast<long long>(D.z_cols) + j) * 4 + c] = reduce_balanced(v * __ldg(dc + orow), D.mod);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        *counter = 0;
        __threadfence();
    }
}

// Compact int32 rows <-> padded int16 blocks of the (m-2)-subsets: u2 in the
// non-hot entry points (backward / target_precondition on compact vectors).
__global__ void __launch_bounds__(kThreads) sub_u_pack_kernel(SubsetDev D, const int32_t* __restrict__ u32,
                                                              uint4* __restrict__ u16) {
    extern __shared__ int32_t sm[];
    const Tables T = stage(D, D.blob_f, sm);
    BW_ITEMS(item, D.n2) {
        const uint32_t d = __ldg(D.m2 + item);
        const int uch = static_cast<int>(d >> 26);
        const int nu = T.a1off[uch + 1] - T.a1off[uch];
        const long long first = d & kLow26;
        const int4 zero = make_int4(0, 0, 0, 0);
        st_block(u16, static_cast<uint32_t>(item), nu > 0 ? ld4(u32, first) : zero,
                 nu > 1 ? ld4(u32, first + 1) : zero);
    }
}
__global__ void __launch_bounds__(kThreads) sub_u_unpack_kernel(SubsetDev D, const uint4* __restrict__ u16,
                                                                int32_t* __restrict__ u32) {
    extern __shared__ int32_t sm[];
    const Tables T = stage(D, D.blob_f, sm);
    BW_ITEMS(item, D.n2) {
        const uint32_t d = __ldg(D.m2 + item);
        const int uch = static_cast<int>(d >> 26);
        const int nu = T.a1off[uch + 1] - T.a1off[uch];
        const long long first = d & kLow26;
        const uint4 b = __ldg(u16 + item);
        if (nu > 0) st4(u32, first, unpack_row(b.x, b.y));
        if (nu > 1) st4(u32, first + 1, unpack_row(b.z, b.w));
    }
}

// Compact int32 u rows <-> u in the row-mixing locality order (int16 rows).
__global__ void __launch_bounds__(kThreads) sub_u_to_walk_kernel(SubsetDev D, const int32_t* __restrict__ u32,
                                                                 uint2* __restrict__ u, long long rows) {
    BW_ITEMS(q, rows) u[__ldg(D.u_pos + q)] = pack_row(ld4(u32, q));
}
__global__ void __launch_bounds__(kThreads) sub_u_from_walk_kernel(SubsetDev D, const uint2* __restrict__ u,
                                                                   int32_t* __restrict__ u32, long long rows) {
    BW_ITEMS(q, rows) {
        const uint2 w = __ldg(u + __ldg(D.u_pos + q));
        st4(u32, q, unpack_row(w.x, w.y));
    }
}

int32_t balanced_of(uint32_t v, const Mod& m) { return to_balanced(v % static_cast<uint32_t>(m.p), m); }

}  // namespace

// Builds the subset tables, the padded preconditioner and the two
// shared-memory blobs, and allocates the padded int16 vectors; leaves
// subset_path false (and says why in subset_reason) when the sector does not
// fit the format or BW_CYCLIC_GENERIC asks for the generic row kernels.
void CyclicCtx::setup_subset_path() {
    subset_path = false;
    if (const char* env = std::getenv("BW_CYCLIC_GENERIC")) {
        if (*env && std::string(env) != "0") {
            subset_reason = "BW_CYCLIC_GENERIC is set";
            return;
        }
    }
    cyclic::SubsetTables tab;
    // u is kept in an order with row-mixing partners adjacent, so the folded
    // preconditioner's sixteen columns of a row fall within a few sectors
    const std::vector<uint32_t> u_pos = cyclic::rowmix_locality_order(plan);
    subset_reason = cyclic::build_subset_tables(inst, es, precond, u_pos, tab);
    if (!subset_reason.empty()) return;

    const cyclic::CharMap a0 = cyclic::build_char_map(inst.weight_a0, inst.r);
    const cyclic::CharMap a1 = cyclic::build_char_map(inst.weight_a1, inst.r);
    const cyclic::CharMap km = cyclic::build_char_map(inst.kernel_weights, inst.r);
    const int n = static_cast<int>(inst.n), g = static_cast<int>(inst.genus), r = static_cast<int>(inst.r);
    const int kdim = static_cast<int>(inst.kernel_dim());
    SubsetDev& D = S;
    D.mod = mod;
    D.n = n;
    D.g = g;
    D.kdim = kdim;
    D.r = r;
    int w = 8 * n * r;   // coefficients: [2 n codes][r] x int4
    D.o_R = w;
    w += g * n;
    D.o_B = w;
    w += g * kdim;
    D.o_a0off = w;
    w += r + 1;
    D.o_a0idx = w;
    w += g;
    D.o_a1off = w;
    w += r + 1;
    D.o_a1idx = w;
    w += n;
    D.o_koff = w;
    w += r + 1;
    D.o_kidx = w;
    w += kdim;
    D.o_ych = w;
    w += r;
    D.blob_words = w;
    if (static_cast<size_t>(w) * 4 > 48 * 1024) {
        subset_reason = "shared-memory tables above 48 KB";
        return;
    }
    std::vector<int32_t> common(w, 0);
    for (int a = 0; a < g; ++a) {
        for (int b = 0; b < n; ++b) common[D.o_R + a * n + b] = balanced_of(inst.right_inverse[a * n + b], mod);
        for (int k = 0; k < kdim; ++k) common[D.o_B + a * kdim + k] = balanced_of(inst.kernel_basis[a * kdim + k], mod);
    }
    for (int c = 0; c <= r; ++c) {
        common[D.o_a0off + c] = static_cast<int32_t>(a0.offsets[c]);
        common[D.o_a1off + c] = static_cast<int32_t>(a1.offsets[c]);
        common[D.o_koff + c] = static_cast<int32_t>(km.offsets[c]);
    }
    for (int e = 0; e < g; ++e) common[D.o_a0idx + e] = a0.indices[e];
    for (int e = 0; e < n; ++e) common[D.o_a1idx + e] = a1.indices[e];
    for (int e = 0; e < kdim; ++e) common[D.o_kidx + e] = km.indices[e];
    for (int c = 0; c < r; ++c)
        common[D.o_ych + c] = static_cast<int32_t>((c + r - static_cast<int>(inst.w_weight % inst.r)) % r);
    // Coefficients of code (sign, generator i) and own character ch: own rows
    // k = 0, 1 (the first two keys of ch's block), neighbour slots l = 0, 1,
    // at int32 number 2 k + l of the entry.
    auto put = [&](std::vector<int32_t>& blob, int i, int ch, int k, int l, uint32_t mu) {
        const int32_t b = balanced_of(mu, mod);
        for (int neg = 0; neg < 2; ++neg) blob[4 * ((neg * n + i) * r + ch) + 2 * k + l] = neg ? -b : b;
    };
    std::vector<int32_t> blob_f = common, blob_t = common;
    for (int i = 0; i < n; ++i)
        for (int ch = 0; ch < r; ++ch) {
            // forward: own rows beta in the A1 block of ch; neighbour rows a in
            // the A0 block of A1(beta) - V(i) (the same block for both betas)
            for (uint32_t kb = a1.offsets[ch]; kb < a1.offsets[ch + 1]; ++kb) {
                const int beta = a1.indices[kb];
                const uint32_t q = (inst.weight_a1[beta] + inst.r - inst.weight_v[i] % inst.r) % inst.r;
                for (uint32_t lb = a0.offsets[q]; lb < a0.offsets[q + 1]; ++lb)
                    put(blob_f, i, ch, static_cast<int>(kb - a1.offsets[ch]), static_cast<int>(lb - a0.offsets[q]),
                        inst.mu_at(i, beta, a0.indices[lb]));
            }
            // transpose: own rows a in the A0 block of ch; neighbour rows beta
            // in the A1 block of A0(a) + V(i)
            for (uint32_t kb = a0.offsets[ch]; kb < a0.offsets[ch + 1]; ++kb) {
                const int a = a0.indices[kb];
                const uint32_t q = (inst.weight_a0[a] + inst.weight_v[i]) % inst.r;
                for (uint32_t lb = a1.offsets[q]; lb < a1.offsets[q + 1]; ++lb)
                    put(blob_t, i, ch, static_cast<int>(kb - a0.offsets[ch]), static_cast<int>(lb - a1.offsets[q]),
                        inst.mu_at(i, a1.indices[lb], a));
            }
        }

    D.n1 = static_cast<uint32_t>(tab.m1.size());
    D.n2 = static_cast<uint32_t>(tab.m2.size());
    D.n0 = static_cast<uint32_t>(tab.m0.size());
    D.w_dmf = static_cast<uint32_t>(es.dm.row_width);
    D.w_d2f = static_cast<uint32_t>(es.d2.row_width);
    D.w_d2t = static_cast<uint32_t>(es.d2.column_width);
    D.w_dmt = static_cast<uint32_t>(es.dm.column_width);
    D.m1 = upload(tab.m1);
    D.m2 = upload(tab.m2);
    D.m0 = upload(tab.m0);
    D.inc_dmf = upload(tab.inc_dmf);
    D.inc_d2f = upload(tab.inc_d2f);
    D.inc_d2t = upload(tab.inc_d2t);
    D.inc_dmt = upload(tab.inc_dmt);
    D.u_pos = upload(u_pos);
    D.e_col = upload(tab.e_col);
    D.e_val = upload(tab.e_val);
    D.ell = static_cast<uint32_t>(tab.ell);
    D.blob_f = upload(blob_f);
    D.blob_t = upload(blob_t);
    D.x_cols = es.x_cols;
    D.z_cols = es.z_cols;
    D.kept_cols = E.kept_cols;
    D.drop0 = E.drop0;
    D.drop1 = E.drop1;
    D.n_extra = E.n_extra;
    D.dense_sign = E.dense_sign;
    D.dense = E.dense;
    // Tables read once per application: evict-first when they exceed half the L2.
    size_t table_bytes = 4 * (tab.inc_dmf.size() + tab.inc_d2f.size() + tab.inc_d2t.size() + tab.inc_dmt.size());
    table_bytes += 4 * tab.e_col.size() + 2 * tab.e_val.size();
    int l2 = 0;
    BW_CUDA(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, device));
    stream_tables = table_bytes > static_cast<size_t>(l2) / 2;
    if (const char* env = std::getenv("BW_CYCLIC_PDL")) pdl = std::string(env) != "0";
    // BW_CYCLIC_STREAM_TABLES=1 / =0 forces the evict-first (or the cached)
    // table reads at any size, so that small sectors run either instantiation.
    if (const char* env = std::getenv("BW_CYCLIC_STREAM_TABLES")) {
        if (*env) stream_tables = std::string(env) != "0";
    }
    // Gathered vectors carry one more block, all zero, for the empty slots of
    // a partial chunk of incidences (their words point at it).
    d_xs16 = alloc<uint4>(D.n0 + 1);
    d_zs = alloc<int32_t>((es.z_cols + dense.columns) * num_v);
    d_y16 = alloc<uint4>(D.n1 + 1);
    d_t16 = alloc<uint4>(D.n1 + 1);
    d_u16 = alloc<uint4>((es.target_rows + 1) / 2 + 1);   // u rows (int16) in the locality order
    d_u2_16 = alloc<uint4>(D.n2 + 1);
    BW_CUDA(cudaMemsetAsync(d_xs16, 0, (D.n0 + 1) * sizeof(uint4), stream));
    BW_CUDA(cudaMemsetAsync(d_y16, 0, (D.n1 + 1) * sizeof(uint4), stream));
    BW_CUDA(cudaMemsetAsync(d_t16, 0, (D.n1 + 1) * sizeof(uint4), stream));
    BW_CUDA(cudaMemsetAsync(d_u2_16, 0, (D.n2 + 1) * sizeof(uint4), stream));
    subset_path = true;
}

// Kernel template dispatch: SMALL (int32 sums exact) x STREAM (tables above L2).
#define BW_SUBSET_DISPATCH(launch)      \
    do {                                \
        if (small && stream_tables) {   \
            launch(true, true);         \
        } else if (small) {             \
            launch(true, false);        \
        } else if (stream_tables) {     \
            launch(false, true);        \
        } else {                        \
            launch(false, false);       \
        }                               \
    } while (0)

void CyclicCtx::subset_source16(const int32_t* in, const int32_t* dc) {
    const size_t smem = static_cast<size_t>(S.blob_words) * 4;
    const size_t items = static_cast<size_t>(S.n0) + es.z_cols + dense.columns;
    sub_source_kernel<<<grid_for(items), kThreads, smem, stream>>>(S, in, dc, d_xs16, d_zs);
    BW_CHECK_LAUNCH();
    ++launches;
    xs_for = dc == d_dc ? in : nullptr;
}

void CyclicCtx::subset_forward16() {
    const size_t smem = static_cast<size_t>(S.blob_words) * 4;
#define BW_LAUNCH(A, B)                                                                                    \
    launch_pdl(sub_dm_forward_elim_kernel<A, B>, grid_for(S.n1), smem, S, static_cast<const uint4*>(d_xs16), \
               static_cast<const int32_t*>(d_zs), d_y16);                                                  \
    launch_pdl(sub_d2_forward_kernel<A, B>, grid_for(S.n2), smem, S, static_cast<const uint4*>(d_y16),     \
               static_cast<const int32_t*>(d_zs), reinterpret_cast<uint2*>(d_u16))
    BW_SUBSET_DISPATCH(BW_LAUNCH);
#undef BW_LAUNCH
    BW_CHECK_LAUNCH();
    launches += 2;
}

void CyclicCtx::subset_precondition16() {
    const uint2* u = reinterpret_cast<const uint2*>(d_u16);
    uint2* u2 = reinterpret_cast<uint2*>(d_u2_16);
    const unsigned grid = grid_for(2 * static_cast<size_t>(S.n2));
#define BW_LAUNCH(A, B) launch_pdl(sub_ell_kernel<A, B>, grid, 0, S, u, u2)
    BW_SUBSET_DISPATCH(BW_LAUNCH);
#undef BW_LAUNCH
    BW_CHECK_LAUNCH();
    ++launches;
}

void CyclicCtx::subset_backward16(const int32_t* dc, int32_t* out, bool next_source) {
    const size_t smem = static_cast<size_t>(S.blob_words) * 4;
    // next_source (apply_square, dc = the column preconditioner): the kernels
    // also write the next application's source from `out`
    uint4* nxs = next_source ? d_xs16 : nullptr;
    int32_t* nzs = next_source ? d_zs : nullptr;
#define BW_LAUNCH(A, B)                                                                                       \
    launch_pdl(sub_d2_transpose_adjoint_kernel<A, B>, grid_for(S.n1), smem, S,                               \
               static_cast<const uint4*>(d_u2_16), dc, d_t16, out, nzs);                                      \
    launch_pdl(sub_dm_transpose_kernel<A, B>, grid_for(S.n0), smem, S, static_cast<const uint4*>(d_t16), dc, \
               out, nxs)
    BW_SUBSET_DISPATCH(BW_LAUNCH);
#undef BW_LAUNCH
    BW_CHECK_LAUNCH();
    launches += 2;
    if (S.n_extra) {
        launch_pdl(sub_dense_t_kernel, dense_grid, smem, S, reinterpret_cast<const uint2*>(d_u2_16), dc, out,
                   d_dpart, d_dcounter, nzs);
        BW_CHECK_LAUNCH();
        ++launches;
    }
    if (next_source)
        xs_for = out;
    else if (xs_for == out)
        xs_for = nullptr;
}

void CyclicCtx::subset_u_to_walk(const int32_t* u32) {
    const long long rows = static_cast<long long>(es.target_rows);
    sub_u_to_walk_kernel<<<grid_for(es.target_rows), kThreads, 0, stream>>>(S, u32, reinterpret_cast<uint2*>(d_u16),
                                                                            rows);
    BW_CHECK_LAUNCH();
    ++launches;
}

void CyclicCtx::subset_u_from_walk(int32_t* u32) {
    const long long rows = static_cast<long long>(es.target_rows);
    sub_u_from_walk_kernel<<<grid_for(es.target_rows), kThreads, 0, stream>>>(
        S, reinterpret_cast<const uint2*>(d_u16), u32, rows);
    BW_CHECK_LAUNCH();
    ++launches;
}

void CyclicCtx::subset_pack_u(const int32_t* u32, uint4* u16) {
    sub_u_pack_kernel<<<grid_for(S.n2), kThreads, static_cast<size_t>(S.blob_words) * 4, stream>>>(S, u32, u16);
    BW_CHECK_LAUNCH();
    ++launches;
}

void CyclicCtx::subset_unpack_u(const uint4* u16, int32_t* u32) {
    sub_u_unpack_kernel<<<grid_for(S.n2), kThreads, static_cast<size_t>(S.blob_words) * 4, stream>>>(S, u16, u32);
    BW_CHECK_LAUNCH();
    ++launches;
}

}  // namespace bw
