// Subset-major paper-mode gathers: the four Koszul maps of the eliminated
// operator with one thread per subset.
//
// Every character block of the shipped instances has at most two rows (A0
// blocks two, A1 blocks one or two, kernel-weight blocks at most one), and
// the rows of one subset's block read the same neighbour blocks with different
// coefficients.  So one thread takes a subset, loads each incidence word and
// each neighbour block once, and accumulates both rows.  The incidence word
// holds the neighbour block's first row directly (no offset lookup), and the
// signed coefficients of mu sit in a dense [sign][i][key][2] table in shared
// memory, so an incidence costs one coalesced word, two 16-byte loads and
// sixteen multiply-adds.
//
// Two of the reference's kernel pairs are fused, with their intermediates
// kept in registers:
//   * D_m forward (cuda/cyclic_cuda_helpers.h:145-204) with the elimination
//     y = B z - R t (cyclic_elim_z_to_y_kernel, cyclic_elim_subtract_Rt_kernel,
//     :718-791): t never reaches memory;
//   * D_(m-1) transpose (:206-266) with t_adj = R^t h and z_adj = B^t h and the
//     z part of the adjoint assembly (cyclic_elim_RT_h_kernel,
//     cyclic_elim_BT_h_kernel, cyclic_elim_assemble_adjoint_kernel, :793-895):
//     h never reaches memory.
// Results are the same canonical residues as the generic row kernels in
// bw_cyclic.cu, which remain for instances outside this format.
#include "bw_cyclic.cuh"
#include "bw_cyclic_dev.cuh"

#include <algorithm>

namespace bw {

namespace {

constexpr int kThreads = 256;
constexpr uint32_t kOffsetMask = (1u << 26) - 1;

using cyc::Acc4;
using cyc::ld4;
using cyc::neg4;
using cyc::scale4;
using cyc::st4;

// Views of the staged shared-memory tables.
struct Tables {
    const int2* coef;
    const int32_t *R, *B, *a0off, *a0idx, *a1off, *a1idx, *koff, *kidx, *ych;
};

__device__ __forceinline__ Tables stage(const SubsetDev& D, const int32_t* __restrict__ blob, int32_t* sm) {
    for (int w = threadIdx.x; w < D.blob_words; w += blockDim.x) sm[w] = __ldg(blob + w);
    __syncthreads();
    Tables t;
    t.coef = reinterpret_cast<const int2*>(sm);
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

// Both rows (keys k0, k1) of subset s against its `width` neighbour blocks:
//   acc_r += sum_pos sum_{l < 2} coef[sign, i, k_r][l] * in[first row + l].
// A neighbour block with fewer than two rows has zero coefficients beyond its
// end; the row read there is a real row or one of the two padding rows every
// gathered vector carries.
template <bool SMALL>
__device__ __forceinline__ void gather2(const uint32_t* __restrict__ inc, uint32_t nsub, uint32_t s, uint32_t width,
                                        const int2* coef, int n, int K, int k0, int k1,
                                        const int32_t* __restrict__ in, Acc4<SMALL>& acc0, Acc4<SMALL>& acc1) {
    // Four incidences at a time: their words, then their eight rows, then the
    // products, so that eight independent 16-byte loads are in flight.
    constexpr int U = 4;
    uint32_t pos = 0;
    for (; pos + U <= width; pos += U) {
        uint32_t e[U];
        int4 v0[U], v1[U];
#pragma unroll
        for (int u = 0; u < U; ++u) e[u] = __ldg(inc + static_cast<size_t>(pos + u) * nsub + s);
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const long long first = e[u] & kOffsetMask;
            v0[u] = ld4(in, first);
            v1[u] = ld4(in, first + 1);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int ci = (static_cast<int>(e[u] >> 31) * n + static_cast<int>((e[u] >> 26) & 31u)) * K;
            const int2 c0 = coef[ci + k0], c1 = coef[ci + k1];
            acc0.mac(c0.x, v0[u]);
            acc0.mac(c0.y, v1[u]);
            acc1.mac(c1.x, v0[u]);
            acc1.mac(c1.y, v1[u]);
        }
    }
    for (; pos < width; ++pos) {
        const uint32_t e = __ldg(inc + static_cast<size_t>(pos) * nsub + s);
        const long long first = e & kOffsetMask;
        const int4 v0 = ld4(in, first), v1 = ld4(in, first + 1);
        const int ci = (static_cast<int>(e >> 31) * n + static_cast<int>((e >> 26) & 31u)) * K;
        const int2 c0 = coef[ci + k0], c1 = coef[ci + k1];
        acc0.mac(c0.x, v0);
        acc0.mac(c0.y, v1);
        acc1.mac(c1.x, v0);
        acc1.mac(c1.y, v1);
    }
}

#define BW_SUBSETS(var, count)                                                                    \
    for (uint32_t var = blockIdx.x * blockDim.x + threadIdx.x; var < (count); var += gridDim.x * blockDim.x)

// (m-1)-subset S: its t rows t(S, beta) = (D_m xs)(S, beta), then its y rows
//   y(S, a) = sum_kappa B[a,kappa] zs(S, kappa) - sum_beta R[a,beta] t(S, beta).
template <bool SMALL>
__global__ void __launch_bounds__(kThreads) sub_dm_forward_elim_kernel(SubsetDev D, const int32_t* __restrict__ xs,
                                                                       int32_t* __restrict__ y) {
    extern __shared__ int32_t sm[];
    const Tables T = stage(D, D.blob_f, sm);
    BW_SUBSETS(s, D.n1) {
        const uint32_t dt = __ldg(D.m1_t + s);
        const int tch = static_cast<int>(dt >> 26);
        const int ych = T.ych[tch];
        const int ya = T.a0off[ych], ny = T.a0off[ych + 1] - ya;
        if (ny == 0) continue;
        const int tb = T.a1off[tch], nt = T.a1off[tch + 1] - tb;
        int4 t0 = make_int4(0, 0, 0, 0), t1 = t0;
        int beta0 = 0, beta1 = 0;
        if (nt > 0) {
            beta0 = T.a1idx[tb];
            beta1 = nt > 1 ? T.a1idx[tb + 1] : beta0;
            Acc4<SMALL> acc0, acc1;
            gather2<SMALL>(D.inc_dmf, D.n1, s, D.w_dmf, T.coef, D.n, D.K, beta0, beta1, xs, acc0, acc1);
            t0 = acc0.reduce(D.mod);
            t1 = acc1.reduce(D.mod);
        }
        const int kb = T.koff[ych], nz = T.koff[ych + 1] - kb;
        int4 z0 = make_int4(0, 0, 0, 0), z1 = z0;
        if (nz > 0) {
            const long long zr = static_cast<long long>(D.x_cols) + __ldg(D.m1_z + s);
            z0 = ld4(xs, zr);
            if (nz > 1) z1 = ld4(xs, zr + 1);
        }
        const long long yrow = __ldg(D.m1_y + s);
        for (int q = 0; q < ny; ++q) {
            const int a = T.a0idx[ya + q];
            Acc4<SMALL> acc;
            if (nz > 0) acc.mac(T.B[a * D.kdim + T.kidx[kb]], z0);
            if (nz > 1) acc.mac(T.B[a * D.kdim + T.kidx[kb + 1]], z1);
            if (nt > 0) acc.mac(-T.R[a * D.n + beta0], t0);
            if (nt > 1) acc.mac(-T.R[a * D.n + beta1], t1);
            st4(y, yrow + q, acc.reduce(D.mod));
        }
    }
}

// (m-2)-subset S2: its u rows u(S2, beta) = (D_(m-1) y)(S2, beta), plus
// dense_sign * dense xs_extra for the deformation variants.
template <bool SMALL>
__global__ void __launch_bounds__(kThreads) sub_d2_forward_kernel(SubsetDev D, const int32_t* __restrict__ y,
                                                                  const int32_t* __restrict__ xs,
                                                                  int32_t* __restrict__ u) {
    extern __shared__ int32_t sm[];
    const Tables T = stage(D, D.blob_f, sm);
    BW_SUBSETS(s, D.n2) {
        const uint32_t du = __ldg(D.m2_u + s);
        const int uch = static_cast<int>(du >> 26);
        const int ub = T.a1off[uch], nu = T.a1off[uch + 1] - ub;
        if (nu == 0) continue;
        const int beta0 = T.a1idx[ub], beta1 = nu > 1 ? T.a1idx[ub + 1] : beta0;
        Acc4<SMALL> acc0, acc1;
        gather2<SMALL>(D.inc_d2f, D.n2, s, D.w_d2f, T.coef, D.n, D.K, beta0, beta1, y, acc0, acc1);
        const long long urow = du & kOffsetMask;
        for (int q = 0; q < nu; ++q) {
            int4 v = q == 0 ? acc0.reduce(D.mod) : acc1.reduce(D.mod);
            if (D.n_extra) {
                for (int j = 0; j < D.n_extra; ++j) {
                    const int32_t c = D.dense_sign * __ldg(D.dense + (urow + q) * D.n_extra + j);
                    const int4 e = ld4(xs, static_cast<long long>(D.base_cols) + j);
                    v.x += c * e.x;
                    v.y += c * e.y;
                    v.z += c * e.z;
                    v.w += c * e.w;
                }
                v = make_int4(reduce_balanced(v.x, D.mod), reduce_balanced(v.y, D.mod), reduce_balanced(v.z, D.mod),
                              reduce_balanced(v.w, D.mod));
            }
            st4(u, urow + q, v);
        }
    }
}

// (m-1)-subset S: its h rows h(S, a) = (D_(m-1)^t u2)(S, a), then
//   t_adj(S, beta) = sum_a R[a,beta] h(S, a)               (all t rows of S)
//   out_z(S, kappa) = dc * sum_a B[a,kappa] h(S, a)        (z rows, through op_col)
template <bool SMALL>
__global__ void __launch_bounds__(kThreads) sub_d2_transpose_adjoint_kernel(SubsetDev D,
                                                                            const int32_t* __restrict__ u2,
                                                                            const int32_t* __restrict__ dc,
                                                                            int32_t* __restrict__ t_adj,
                                                                            int32_t* __restrict__ out) {
    extern __shared__ int32_t sm[];
    const Tables T = stage(D, D.blob_t, sm);
    BW_SUBSETS(s, D.n1) {
        const uint32_t dt = __ldg(D.m1_t + s);
        const int tch = static_cast<int>(dt >> 26);
        const int ych = T.ych[tch];
        const int ya = T.a0off[ych], ny = T.a0off[ych + 1] - ya;
        const int a0 = ny > 0 ? T.a0idx[ya] : 0, a1 = ny > 1 ? T.a0idx[ya + 1] : a0;
        int4 h0 = make_int4(0, 0, 0, 0), h1 = h0;
        if (ny > 0) {
            Acc4<SMALL> acc0, acc1;
            gather2<SMALL>(D.inc_d2t, D.n1, s, D.w_d2t, T.coef, D.n, D.K, a0, a1, u2, acc0, acc1);
            h0 = acc0.reduce(D.mod);
            h1 = acc1.reduce(D.mod);
        }
        const int tb = T.a1off[tch], nt = T.a1off[tch + 1] - tb;
        const long long trow = dt & kOffsetMask;
        for (int q = 0; q < nt; ++q) {
            const int beta = T.a1idx[tb + q];
            Acc4<SMALL> acc;
            if (ny > 0) acc.mac(T.R[a0 * D.n + beta], h0);
            if (ny > 1) acc.mac(T.R[a1 * D.n + beta], h1);
            st4(t_adj, trow + q, acc.reduce(D.mod));
        }
        const int kb = T.koff[ych], nz = T.koff[ych + 1] - kb;
        if (nz == 0) continue;
        const long long zfirst = static_cast<long long>(D.x_cols) + __ldg(D.m1_z + s);
        for (int q = 0; q < nz; ++q) {
            const long long orow = cyc::op_col(D.drop0, D.drop1, zfirst + q);
            if (orow < 0) continue;   // dropped base column (replacement)
            const int kap = T.kidx[kb + q];
            Acc4<SMALL> acc;
            if (ny > 0) acc.mac(T.B[a0 * D.kdim + kap], h0);
            if (ny > 1) acc.mac(T.B[a1 * D.kdim + kap], h1);
            const int4 v = acc.reduce(D.mod);
            st4(out, orow, dc ? scale4(v, __ldg(dc + orow), D.mod) : v);
        }
    }
}

// m-subset S': its x rows out_x(S', a) = -dc * (D_m^t t_adj)(S', a), through op_col.
template <bool SMALL>
__global__ void __launch_bounds__(kThreads) sub_dm_transpose_kernel(SubsetDev D, const int32_t* __restrict__ t_adj,
                                                                    const int32_t* __restrict__ dc,
                                                                    int32_t* __restrict__ out) {
    extern __shared__ int32_t sm[];
    const Tables T = stage(D, D.blob_t, sm);
    BW_SUBSETS(s, D.n0) {
        const uint32_t dx = __ldg(D.m_x + s);
        const int xch = static_cast<int>(dx >> 26);
        const int xa = T.a0off[xch], nx = T.a0off[xch + 1] - xa;
        if (nx == 0) continue;
        const int a0 = T.a0idx[xa], a1 = nx > 1 ? T.a0idx[xa + 1] : a0;
        Acc4<SMALL> acc0, acc1;
        gather2<SMALL>(D.inc_dmt, D.n0, s, D.w_dmt, T.coef, D.n, D.K, a0, a1, t_adj, acc0, acc1);
        const long long xrow = dx & kOffsetMask;
        for (int q = 0; q < nx; ++q) {
            const long long orow = cyc::op_col(D.drop0, D.drop1, xrow + q);
            if (orow < 0) continue;   // dropped base column (replacement)
            const int4 v = neg4(q == 0 ? acc0.reduce(D.mod) : acc1.reduce(D.mod));
            st4(out, orow, dc ? scale4(v, __ldg(dc + orow), D.mod) : v);
        }
    }
}

int32_t balanced_of(uint32_t v, const Mod& m) { return to_balanced(v % static_cast<uint32_t>(m.p), m); }

}  // namespace

// Builds the subset tables and the two shared-memory blobs; leaves
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
    subset_reason = cyclic::build_subset_tables(inst, es, tab);
    if (!subset_reason.empty()) return;

    const cyclic::CharMap a0 = cyclic::build_char_map(inst.weight_a0, inst.r);
    const cyclic::CharMap a1 = cyclic::build_char_map(inst.weight_a1, inst.r);
    const cyclic::CharMap km = cyclic::build_char_map(inst.kernel_weights, inst.r);
    const int n = static_cast<int>(inst.n), g = static_cast<int>(inst.genus), r = static_cast<int>(inst.r);
    const int kdim = static_cast<int>(inst.kernel_dim()), K = std::max(n, g);
    SubsetDev& D = S;
    D.mod = mod;
    D.n = n;
    D.g = g;
    D.kdim = kdim;
    D.r = r;
    D.K = K;
    int w = 4 * n * K;
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
    std::vector<int32_t> blob_f = common, blob_t = common;
    auto coef_at = [&](std::vector<int32_t>& blob, int neg, int i, int key, int l, uint32_t mu) {
        const int32_t b = balanced_of(mu, mod);
        blob[(((neg * n + i) * K + key) * 2) + l] = neg ? -b : b;
    };
    // forward: (i, beta) -> mu[i, beta, a] over the A0 block of A1(beta) - V(i)
    for (int i = 0; i < n; ++i)
        for (int beta = 0; beta < n; ++beta) {
            const uint32_t q = (inst.weight_a1[beta] + inst.r - inst.weight_v[i] % inst.r) % inst.r;
            for (uint32_t idx = a0.offsets[q]; idx < a0.offsets[q + 1]; ++idx)
                for (int neg = 0; neg < 2; ++neg)
                    coef_at(blob_f, neg, i, beta, static_cast<int>(idx - a0.offsets[q]),
                            inst.mu_at(i, beta, a0.indices[idx]));
        }
    // transpose: (j, a) -> mu[j, beta, a] over the A1 block of A0(a) + V(j)
    for (int j = 0; j < n; ++j)
        for (int a = 0; a < g; ++a) {
            const uint32_t q = (inst.weight_a0[a] + inst.weight_v[j]) % inst.r;
            for (uint32_t idx = a1.offsets[q]; idx < a1.offsets[q + 1]; ++idx)
                for (int neg = 0; neg < 2; ++neg)
                    coef_at(blob_t, neg, j, a, static_cast<int>(idx - a1.offsets[q]),
                            inst.mu_at(j, a1.indices[idx], a));
        }

    D.n1 = static_cast<uint32_t>(tab.m1_t.size());
    D.n2 = static_cast<uint32_t>(tab.m2_u.size());
    D.n0 = static_cast<uint32_t>(tab.m_x.size());
    D.w_dmf = static_cast<uint32_t>(es.dm.row_width);
    D.w_d2f = static_cast<uint32_t>(es.d2.row_width);
    D.w_d2t = static_cast<uint32_t>(es.d2.column_width);
    D.w_dmt = static_cast<uint32_t>(es.dm.column_width);
    D.m1_t = upload(tab.m1_t);
    D.m1_y = upload(tab.m1_y);
    D.m1_z = upload(tab.m1_z);
    D.m2_u = upload(tab.m2_u);
    D.m_x = upload(tab.m_x);
    D.inc_dmf = upload(tab.inc_dmf);
    D.inc_d2f = upload(tab.inc_d2f);
    D.inc_d2t = upload(tab.inc_d2t);
    D.inc_dmt = upload(tab.inc_dmt);
    D.blob_f = upload(blob_f);
    D.blob_t = upload(blob_t);
    D.x_cols = es.x_cols;
    D.base_cols = E.base_cols;
    D.drop0 = E.drop0;
    D.drop1 = E.drop1;
    D.n_extra = E.n_extra;
    D.dense_sign = E.dense_sign;
    D.dense = E.dense;
    subset_path = true;
}

void CyclicCtx::subset_forward(int32_t* u) {
    const size_t smem = static_cast<size_t>(S.blob_words) * 4;
    if (small) {
        sub_dm_forward_elim_kernel<true><<<grid_for(S.n1), kThreads, smem, stream>>>(S, d_xs, d_y);
        sub_d2_forward_kernel<true><<<grid_for(S.n2), kThreads, smem, stream>>>(S, d_y, d_xs, u);
    } else {
        sub_dm_forward_elim_kernel<false><<<grid_for(S.n1), kThreads, smem, stream>>>(S, d_xs, d_y);
        sub_d2_forward_kernel<false><<<grid_for(S.n2), kThreads, smem, stream>>>(S, d_y, d_xs, u);
    }
    BW_CHECK_LAUNCH();
    launches += 2;
}

void CyclicCtx::subset_backward(const int32_t* u2, const int32_t* dc, int32_t* out) {
    const size_t smem = static_cast<size_t>(S.blob_words) * 4;
    if (small) {
        sub_d2_transpose_adjoint_kernel<true><<<grid_for(S.n1), kThreads, smem, stream>>>(S, u2, dc, d_t, out);
        sub_dm_transpose_kernel<true><<<grid_for(S.n0), kThreads, smem, stream>>>(S, d_t, dc, out);
    } else {
        sub_d2_transpose_adjoint_kernel<false><<<grid_for(S.n1), kThreads, smem, stream>>>(S, u2, dc, d_t, out);
        sub_dm_transpose_kernel<false><<<grid_for(S.n0), kThreads, smem, stream>>>(S, d_t, dc, out);
    }
    BW_CHECK_LAUNCH();
    launches += 2;
}

}  // namespace bw
