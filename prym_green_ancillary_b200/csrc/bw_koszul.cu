// Synthetic Koszul operator S = D d^T d and its block-Wiedemann sequence,
// plain CUDA-core form, plus the context / sequence-session plumbing that the
// INT8-limb tensor-core form (bw_koszul_i8.cu) shares.
//
// Data layout in HBM (all row-major, balanced int32 residues inside the
// engine, canonical uint32 at the ABI):
//   Y, W  : n_src x n   row = S_rank * dim_in  + b   (S a k-subset)
//   Z     : n_tgt x n   row = T_rank * dim_out + c   (T a (k-1)-subset)
//   X     : n_src x m
// so one subset's block is one contiguous run of dim * n residues.
//
// Incidence tables (built once on the host):
//   fwd[T][q], q < r-k+1 : the subsets S = T u {i}, i not in T
//   bwd[S][q], q < k     : the subsets T = S \ {i},  i in S
// each entry = subset rank | i << 26 | negative << 31, with the entries of a
// row ordered positive signs first so that a kernel flips its accumulator sign
// at most once per output block.
#include "bw_koszul.cuh"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <cstring>
#include <vector>

namespace bw {

// ----------------------------------------------------------------- kernels

namespace {

// acc[o0 + a][j] += coef[a] * y[j] for the four coefficients of one int4
template <int TO>
__device__ __forceinline__ void mac4(int32_t (&acc)[TO][4], int o0, const int4& a, const int4& y) {
    acc[o0][0] += a.x * y.x; acc[o0][1] += a.x * y.y; acc[o0][2] += a.x * y.z; acc[o0][3] += a.x * y.w;
    acc[o0 + 1][0] += a.y * y.x; acc[o0 + 1][1] += a.y * y.y; acc[o0 + 1][2] += a.y * y.z; acc[o0 + 1][3] += a.y * y.w;
    acc[o0 + 2][0] += a.z * y.x; acc[o0 + 2][1] += a.z * y.y; acc[o0 + 2][2] += a.z * y.z; acc[o0 + 2][3] += a.z * y.w;
    acc[o0 + 3][0] += a.w * y.x; acc[o0 + 3][1] += a.w * y.y; acc[o0 + 3][2] += a.w * y.z; acc[o0 + 3][3] += a.w * y.w;
}

template <int TO>
__device__ __forceinline__ void reduce_tile(int32_t (&acc)[TO][4], const Mod& mod) {
#pragma unroll
    for (int a = 0; a < TO; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = reduce_partial(acc[a][b], mod);
}

template <int TO>
__device__ __forceinline__ void negate_tile(int32_t (&acc)[TO][4]) {
#pragma unroll
    for (int a = 0; a < TO; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = -acc[a][b];
}

// One gather-multiply pass shared by d and d^T.
//
//   out[blk][o][j] = sum_{q < width} sign_q sum_{u < inner} coef[i_q][u][o] * in[sub_q][u][j]
//
// d   : blk = T, o = c (dim_out), u = b (dim_in),  coef = M^T  (i x b x c)
// d^T : blk = S, o = b (dim_in),  u = c (dim_out), coef = M    (i x c x b)
//
// A thread owns a TO (o) x 4 (j) register tile of one output block (TO = 4 or
// 8: an 8-row tile does twice the multiply-adds per gathered 16-byte row); the
// coefficient tiles of all r maps sit in shared memory ([i][u][o], rows of
// `ostride` = outer rounded up to 8, zero-padded), the gathered input rows
// stream from L2 as 16-byte loads.  Sums of 8 balanced products stay inside
// int32 next to a partially reduced value, so the accumulator is reduced every
// 8 u-steps.
template <int NB, int TO>
__global__ void __launch_bounds__(256) gather_mac_kernel(
    const int32_t* __restrict__ in, int32_t* __restrict__ out,
    const uint32_t* __restrict__ inc, const int32_t* __restrict__ coef,
    const int32_t* __restrict__ diag,   // nullptr: no scaling
    long long n_blk, int width, int r, int inner, int outer, int ostride, Mod mod) {
    extern __shared__ int4 smem_raw[];
    int32_t* sm = reinterpret_cast<int32_t*>(smem_raw);
    const int total = r * inner * ostride;
    for (int e = threadIdx.x; e < total; e += blockDim.x) sm[e] = coef[e];
    __syncthreads();

    constexpr int JG = NB / 4;
    constexpr int TQ = TO / 4;                     // int4 coefficient loads per u-step
    const int OG = (outer + TO - 1) / TO;
    const int OS4 = ostride / 4;
    const int tpb = OG * JG;                       // threads per output block
    const int bpc = blockDim.x / tpb;              // output blocks per CTA pass
    const int local = threadIdx.x / tpb;
    const int sub = threadIdx.x - local * tpb;
    const int og = sub / JG;
    const int jg = sub - og * JG;
    if (local >= bpc) return;                      // no barrier below this point

    const int4* sm4 = reinterpret_cast<const int4*>(sm);
    for (long long blk = static_cast<long long>(blockIdx.x) * bpc + local; blk < n_blk;
         blk += static_cast<long long>(gridDim.x) * bpc) {
        int32_t acc[TO][4];
#pragma unroll
        for (int a = 0; a < TO; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] = 0;
        bool neg_state = false;
        const uint32_t* binc = inc + blk * width;
        // The incidence word of the next neighbour is loaded one neighbour
        // ahead, and a chunk's eight input rows are all in flight before its
        // multiply-adds: the gathers' L2 latency overlaps instead of chaining.
        uint32_t e_next = width > 0 ? __ldg(binc) : 0u;
        for (int q = 0; q < width; ++q) {
            const uint32_t e = e_next;
            if (q + 1 < width) e_next = __ldg(binc + q + 1);
            const bool neg = (e >> 31) != 0;
            const int i = static_cast<int>((e >> 26) & 31u);
            const long long s = static_cast<long long>(e & 0x3FFFFFFu);
            if (neg != neg_state) {
                negate_tile<TO>(acc);
                neg_state = neg;
            }
            const int4* irow = reinterpret_cast<const int4*>(in + s * inner * NB) + jg;
            const int4* crow = sm4 + static_cast<size_t>(i) * inner * OS4 + og * TQ;
            for (int u0 = 0; u0 < inner; u0 += 8) {
                int4 y[8];
#pragma unroll
                for (int uu = 0; uu < 8; ++uu)
                    y[uu] = u0 + uu < inner ? __ldg(irow + (u0 + uu) * JG) : make_int4(0, 0, 0, 0);
#pragma unroll
                for (int uu = 0; uu < 8; ++uu) {
                    if (u0 + uu >= inner) break;
#pragma unroll
                    for (int t = 0; t < TQ; ++t) mac4<TO>(acc, 4 * t, crow[(u0 + uu) * OS4 + t], y[uu]);
                }
                reduce_tile<TO>(acc, mod);
            }
        }
        if (neg_state) negate_tile<TO>(acc);
        const int o0 = og * TO;
#pragma unroll
        for (int a = 0; a < TO; ++a) {
            const int o = o0 + a;
            if (o >= outer) break;
            const long long row = blk * outer + o;
            int4 v;
            int32_t s0 = reduce_balanced(acc[a][0], mod), s1 = reduce_balanced(acc[a][1], mod);
            int32_t s2 = reduce_balanced(acc[a][2], mod), s3 = reduce_balanced(acc[a][3], mod);
            if (diag != nullptr) {
                const int32_t dv = __ldg(diag + row);
                s0 = reduce_balanced(s0 * dv, mod);
                s1 = reduce_balanced(s1 * dv, mod);
                s2 = reduce_balanced(s2 * dv, mod);
                s3 = reduce_balanced(s3 * dv, mod);
            }
            v.x = s0; v.y = s1; v.z = s2; v.w = s3;
            reinterpret_cast<int4*>(out + row * NB)[jg] = v;
        }
    }
}

// Projection a = X^T W (m x n) of one block into seq[*seq_index].  Every CTA
// adds its m x n balanced sums into one int32 accumulator with atomics (at
// most 4 * 148 CTAs x (p-1)/2, far below 2^31: exact, and the same whatever
// the order of the additions); the last CTA to finish reads and clears it.
//   partials : m x n int32 accumulator, left at 0 after every launch
//   counter  : arrival counter, left at 0 after every launch
template <int NB>
__global__ void __launch_bounds__(256) project_kernel(
    const int32_t* __restrict__ X, const int32_t* __restrict__ W, long long rows, int m,
    int32_t* __restrict__ partials, unsigned int* __restrict__ counter,
    uint32_t* __restrict__ seq, unsigned long long* __restrict__ seq_index, Mod mod) {
    constexpr int JG = NB / 4;
    const int tps = m * JG;                       // threads per row slice
    const int slices = blockDim.x / tps;
    const int slice = threadIdx.x / tps;
    const int sub = threadIdx.x - slice * tps;
    const int x = sub / JG;
    const int jg = sub - x * JG;
    __shared__ int32_t red[256 * 4];
    __shared__ bool am_last;

    int32_t acc[4] = {0, 0, 0, 0};
    if (slice < slices) {
        // four rows a pass, their loads in flight together; eight products of
        // balanced residues beside a partially reduced value stay inside int32
        const long long stride = static_cast<long long>(gridDim.x) * slices;
        long long row = static_cast<long long>(blockIdx.x) * slices + slice;
        for (; row + 3 * stride < rows; row += 4 * stride) {
            int32_t xv[4];
            int4 w[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                xv[q] = __ldg(X + (row + q * stride) * m + x);
                w[q] = __ldg(reinterpret_cast<const int4*>(W + (row + q * stride) * NB) + jg);
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                acc[0] += xv[q] * w[q].x; acc[1] += xv[q] * w[q].y; acc[2] += xv[q] * w[q].z; acc[3] += xv[q] * w[q].w;
            }
#pragma unroll
            for (int a = 0; a < 4; ++a) acc[a] = reduce_partial(acc[a], mod);
        }
        for (; row < rows; row += stride) {
            const int32_t xv = __ldg(X + row * m + x);
            const int4 w = __ldg(reinterpret_cast<const int4*>(W + row * NB) + jg);
            acc[0] += xv * w.x; acc[1] += xv * w.y; acc[2] += xv * w.z; acc[3] += xv * w.w;
        }
#pragma unroll
        for (int a = 0; a < 4; ++a) acc[a] = reduce_balanced(acc[a], mod);
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) red[threadIdx.x * 4 + a] = acc[a];
    __syncthreads();
    // Fold the slices: thread t < tps sums column t of the slice table.
    if (threadIdx.x < tps) {
        int32_t s[4] = {0, 0, 0, 0};
        for (int sl = 0; sl < slices; ++sl) {
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                s[a] += red[(sl * tps + threadIdx.x) * 4 + a];
                if ((sl & 7) == 7) s[a] = reduce_partial(s[a], mod);
            }
        }
        const int xx = threadIdx.x / JG, jj = threadIdx.x - xx * JG;
        int32_t* dst = partials + (static_cast<size_t>(xx) * NB + jj * 4);
#pragma unroll
        for (int a = 0; a < 4; ++a) atomicAdd(dst + a, reduce_balanced(s[a], mod));
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int ticket = atomicAdd(counter, 1u);
        am_last = (ticket == gridDim.x - 1);
    }
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    const unsigned long long pos = *reinterpret_cast<volatile unsigned long long*>(seq_index);
    const int entries = m * NB;
    for (int e = threadIdx.x; e < entries; e += blockDim.x)
        seq[pos * entries + e] = to_canonical(reduce_balanced(atomicExch(partials + e, 0), mod), mod);
    __syncthreads();
    if (threadIdx.x == 0) {
        *seq_index = pos + 1;
        *counter = 0;
        __threadfence();
    }
}

__global__ void to_balanced_kernel(const uint32_t* __restrict__ in, int32_t* __restrict__ out,
                                   long long count, Mod mod) {
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride)
        out[i] = to_balanced(in[i] % static_cast<uint32_t>(mod.p), mod);
}

__global__ void to_canonical_kernel(const int32_t* __restrict__ in, uint32_t* __restrict__ out,
                                    long long count, Mod mod) {
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride)
        out[i] = to_canonical(in[i], mod);
}

}  // namespace

// ------------------------------------------------------------ host helpers

void KoszulCtx::launch_to_balanced(const uint32_t* in, int32_t* out, uint64_t count, cudaStream_t st) {
    if (count == 0) return;
    unsigned grid = static_cast<unsigned>(std::min<uint64_t>((count + 255) / 256, static_cast<uint64_t>(sms) * 8));
    to_balanced_kernel<<<grid, 256, 0, st>>>(in, out, static_cast<long long>(count), mod);
    BW_CHECK_LAUNCH();
    ++launches;
}

void KoszulCtx::launch_to_canonical(const int32_t* in, uint32_t* out, uint64_t count, cudaStream_t st) {
    if (count == 0) return;
    unsigned grid = static_cast<unsigned>(std::min<uint64_t>((count + 255) / 256, static_cast<uint64_t>(sms) * 8));
    to_canonical_kernel<<<grid, 256, 0, st>>>(in, out, static_cast<long long>(count), mod);
    BW_CHECK_LAUNCH();
    ++launches;
}

namespace {

template <int NB, int TO>
void launch_gather(KoszulCtx& c, const int32_t* in, int32_t* out, const uint32_t* inc, const int32_t* coef,
                   const int32_t* diag, uint64_t n_blk, int width, int inner, int outer, int ostride,
                   cudaStream_t st) {
    const size_t smem = static_cast<size_t>(c.r) * inner * ostride * sizeof(int32_t);
    auto kern = gather_mac_kernel<NB, TO>;
    const int tpb = (outer + TO - 1) / TO * (NB / 4);
    BW_REQUIRE(tpb <= 256, "dimension too large for the plain gather kernel (dim/4 * n/4 > 256)");
    const int bpc = 256 / tpb;
    BW_REQUIRE(static_cast<int>(smem) <= allow_dynamic_smem(kern, c.device),
               "maps too large for shared memory staging");
    int occ = 0;
    BW_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 256, smem));
    BW_REQUIRE(occ > 0, "plain gather kernel does not fit on an SM");
    const uint64_t groups = (n_blk + bpc - 1) / bpc;
    const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(groups, static_cast<uint64_t>(c.sms) * occ));
    kern<<<grid, 256, smem, st>>>(in, out, inc, coef, diag, static_cast<long long>(n_blk), width, c.r,
                                  inner, outer, ostride, c.mod);
    BW_CHECK_LAUNCH();
    ++c.launches;
}

template <int NB>
void launch_project(KoszulCtx& c, const int32_t* W, cudaStream_t st) {
    project_kernel<NB><<<c.proj_grid, 256, 0, st>>>(c.d_xb, W, static_cast<long long>(c.n_src), c.m,
                                                    c.d_partials, c.d_counter, c.d_seq, c.d_seq_index, c.mod);
    BW_CHECK_LAUNCH();
    ++c.launches;
}

template <class F>
void dispatch_nb(int nb, F&& f) {
    switch (nb) {
        case 4: f(std::integral_constant<int, 4>{}); break;
        case 8: f(std::integral_constant<int, 8>{}); break;
        case 16: f(std::integral_constant<int, 16>{}); break;
        case 32: f(std::integral_constant<int, 32>{}); break;
        default: throw Error("block width must be 4, 8, 16 or 32", 1);
    }
}

}  // namespace

void KoszulCtx::plain_forward(const int32_t* y, int32_t* z, cudaStream_t st) {
    dispatch_nb(nb, [&](auto NBc) {
        constexpr int NB = decltype(NBc)::value;
        if (tile_fwd == 8)
            launch_gather<NB, 8>(*this, y, z, d_fwd, d_coef_fwd, nullptr, n_t, r - k + 1, ci, co, co8, st);
        else
            launch_gather<NB, 4>(*this, y, z, d_fwd, d_coef_fwd, nullptr, n_t, r - k + 1, ci, co, co8, st);
    });
}

void KoszulCtx::plain_transpose(const int32_t* z, int32_t* w, bool scale, cudaStream_t st) {
    dispatch_nb(nb, [&](auto NBc) {
        constexpr int NB = decltype(NBc)::value;
        const int32_t* dg = scale ? d_diag : nullptr;
        if (tile_bwd == 8)
            launch_gather<NB, 8>(*this, z, w, d_bwd, d_coef_bwd, dg, n_s, k, co, ci, ci8, st);
        else
            launch_gather<NB, 4>(*this, z, w, d_bwd, d_coef_bwd, dg, n_s, k, co, ci, ci8, st);
    });
}

void KoszulCtx::project(const int32_t* w, cudaStream_t st) {
    dispatch_nb(nb, [&](auto NBc) { launch_project<decltype(NBc)::value>(*this, w, st); });
}

// One step: cur -> other, append a_i.
void KoszulCtx::step_once(cudaStream_t st) {
    if (form == BW_FORM_INT8) {
        i8_step_once(st);
        return;
    }
    int32_t* src = cur_is_a ? d_ya : d_yb;
    int32_t* dst = cur_is_a ? d_yb : d_ya;
    plain_forward(src, d_z, st);
    plain_transpose(d_z, dst, true, st);
    project(dst, st);
    cur_is_a = !cur_is_a;
}

// --------------------------------------------------------------- creation

KoszulCtx::~KoszulCtx() {
    cudaSetDevice(device);
    i8_destroy();
    for (auto& g : graphs)
        if (g) cudaGraphExecDestroy(g);
    for (void* p : allocations) cudaFree(p);
    if (ev_join) cudaEventDestroy(ev_join);
    if (own_stream) cudaStreamDestroy(own_stream);
}

template <class T>
T* KoszulCtx::alloc(uint64_t count) {
    void* p = nullptr;
    const uint64_t bytes = std::max<uint64_t>(count, 1) * sizeof(T);
    BW_CUDA(cudaMalloc(&p, bytes));
    allocations.push_back(p);
    device_bytes += bytes;
    return static_cast<T*>(p);
}

static void build_tables(int r, int k, std::vector<uint32_t>& fwd, std::vector<uint32_t>& bwd) {
    const uint64_t n_t = binom(r, k - 1), n_s = binom(r, k);
    const int fw = r - k + 1;
    fwd.assign(n_t * fw, 0);
    bwd.assign(n_s * k, 0);
    int T[64], S[64];
    for (uint64_t t = 0; t < n_t; ++t) {
        lex_unrank(t, r, k - 1, T);
        uint32_t pos_list[64], neg_list[64];
        int np = 0, nn = 0, pos = 0;
        for (int i = 0; i < r; ++i) {
            if (pos < k - 1 && T[pos] == i) {
                ++pos;
                continue;
            }
            for (int q = 0, w = 0; q < k; ++q) S[q] = (q == pos) ? i : T[w++];
            const uint32_t e = static_cast<uint32_t>(lex_rank(S, r, k)) | (static_cast<uint32_t>(i) << 26);
            if (pos & 1) neg_list[nn++] = e | 0x80000000u;
            else pos_list[np++] = e;
        }
        uint32_t* row = fwd.data() + t * fw;
        std::memcpy(row, pos_list, sizeof(uint32_t) * np);
        std::memcpy(row + np, neg_list, sizeof(uint32_t) * nn);
    }
    for (uint64_t s = 0; s < n_s; ++s) {
        lex_unrank(s, r, k, S);
        uint32_t* row = bwd.data() + s * k;
        int np = 0;
        uint32_t neg_list[64];
        int nn = 0;
        for (int pos = 0; pos < k; ++pos) {
            for (int q = 0, w = 0; q < k; ++q)
                if (q != pos) T[w++] = S[q];
            const uint32_t e = static_cast<uint32_t>(lex_rank(T, r, k - 1)) | (static_cast<uint32_t>(S[pos]) << 26);
            if (pos & 1) neg_list[nn++] = e | 0x80000000u;
            else row[np++] = e;
        }
        std::memcpy(row + np, neg_list, sizeof(uint32_t) * nn);
    }
}

KoszulCtx* KoszulCtx::create(const bw_koszul_desc& d, int dev) {
    BW_REQUIRE(d.r >= 2 && d.r <= 31, "r must be in 2..31");
    BW_REQUIRE(d.k >= 1 && d.k <= d.r, "k must be in 1..r");
    BW_REQUIRE(d.dim_in >= 1 && d.dim_out >= 1 && d.dim_in <= 256 && d.dim_out <= 256,
               "dim_in and dim_out must be in 1..256");
    BW_REQUIRE(d.prime >= 3 && d.prime < 32768 && (d.prime & 1u), "prime must be odd and below 2^15");
    for (uint32_t f = 3; f * f <= d.prime; f += 2)
        BW_REQUIRE(d.prime % f != 0, "modulus is not prime");
    auto ok_w = [](uint32_t w) { return w == 4 || w == 8 || w == 16 || w == 32; };
    BW_REQUIRE(ok_w(d.block_width) && ok_w(d.proj_width), "block and projection widths must be 4, 8, 16 or 32");
    BW_REQUIRE(d.form == BW_FORM_PLAIN || d.form == BW_FORM_INT8, "unknown arithmetic form");
    BW_REQUIRE(d.maps != nullptr && d.diag != nullptr, "maps and diagonal are required");
    BW_REQUIRE(binom(d.r, d.k) < (1ull << 26) && binom(d.r, d.k - 1) < (1ull << 26),
               "subset counts above 2^26 are not supported");

    std::unique_ptr<KoszulCtx> c(new KoszulCtx());
    c->device = dev;
    BW_CUDA(cudaSetDevice(dev));
    c->sms = sm_count(dev);
    c->r = static_cast<int>(d.r);
    c->k = static_cast<int>(d.k);
    c->ci = static_cast<int>(d.dim_in);
    c->co = static_cast<int>(d.dim_out);
    c->ci8 = (c->ci + 7) / 8 * 8;
    c->co8 = (c->co + 7) / 8 * 8;
    c->nb = static_cast<int>(d.block_width);
    c->nbi = d.form == BW_FORM_INT8 ? (c->nb <= 16 ? 16 : 32) : c->nb;
    c->m = static_cast<int>(d.proj_width);
    c->p = d.prime;
    c->mod = make_mod(d.prime);
    c->form = d.form;
    c->n_s = binom(c->r, c->k);
    c->n_t = binom(c->r, c->k - 1);
    c->n_src = c->n_s * c->ci;
    c->n_tgt = c->n_t * c->co;
    BW_CUDA(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
    BW_CUDA(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));

    const size_t smem_fwd = static_cast<size_t>(c->r) * c->ci * c->co8 * sizeof(int32_t);
    const size_t smem_bwd = static_cast<size_t>(c->r) * c->co * c->ci8 * sizeof(int32_t);
    BW_REQUIRE(smem_fwd <= 200 * 1024 && smem_bwd <= 200 * 1024,
               "maps too large for shared memory staging (r * dim_in * dim_out * 4 > 200 KiB)");

    // Coefficient tiles (balanced): forward uses M^T [i][b][c8], transpose M [i][c][b8] (rows zero-padded to 8).
    std::vector<int32_t> coef_fwd(static_cast<size_t>(c->r) * c->ci * c->co8, 0);
    std::vector<int32_t> coef_bwd(static_cast<size_t>(c->r) * c->co * c->ci8, 0);
    c->maps_canonical.assign(d.maps, d.maps + static_cast<size_t>(c->r) * c->co * c->ci);
    for (int i = 0; i < c->r; ++i)
        for (int cc = 0; cc < c->co; ++cc)
            for (int b = 0; b < c->ci; ++b) {
                const uint32_t v = d.maps[(static_cast<size_t>(i) * c->co + cc) * c->ci + b] % c->p;
                const int32_t bal = to_balanced(v, c->mod);
                coef_fwd[(static_cast<size_t>(i) * c->ci + b) * c->co8 + cc] = bal;
                coef_bwd[(static_cast<size_t>(i) * c->co + cc) * c->ci8 + b] = bal;
            }
    std::vector<uint32_t> fwd, bwd;
    build_tables(c->r, c->k, fwd, bwd);

    cudaStream_t st = c->own_stream;
    c->d_coef_fwd = c->alloc<int32_t>(coef_fwd.size());
    c->d_coef_bwd = c->alloc<int32_t>(coef_bwd.size());
    c->d_fwd = c->alloc<uint32_t>(fwd.size());
    c->d_bwd = c->alloc<uint32_t>(bwd.size());
    BW_CUDA(cudaMemcpyAsync(c->d_coef_fwd, coef_fwd.data(), coef_fwd.size() * 4, cudaMemcpyHostToDevice, st));
    BW_CUDA(cudaMemcpyAsync(c->d_coef_bwd, coef_bwd.data(), coef_bwd.size() * 4, cudaMemcpyHostToDevice, st));
    BW_CUDA(cudaMemcpyAsync(c->d_fwd, fwd.data(), fwd.size() * 4, cudaMemcpyHostToDevice, st));
    BW_CUDA(cudaMemcpyAsync(c->d_bwd, bwd.data(), bwd.size() * 4, cudaMemcpyHostToDevice, st));

    c->d_diag = c->alloc<int32_t>(c->n_src);
    if (d.diag_on_device) {
        c->launch_to_balanced(d.diag, c->d_diag, c->n_src, st);
    } else {
        uint32_t* tmp = c->alloc<uint32_t>(c->n_src);
        BW_CUDA(cudaMemcpyAsync(tmp, d.diag, c->n_src * 4, cudaMemcpyHostToDevice, st));
        c->launch_to_balanced(tmp, c->d_diag, c->n_src, st);
        BW_CUDA(cudaStreamSynchronize(st));
        c->release(tmp);
    }
    if (c->form == BW_FORM_PLAIN) {   // the INT8 form keeps its state as limb planes
        c->d_ya = c->alloc<int32_t>(c->n_src * c->nb);
        c->d_yb = c->alloc<int32_t>(c->n_src * c->nb);
        c->d_z = c->alloc<int32_t>(c->n_tgt * c->nb);
        c->d_xb = c->alloc<int32_t>(c->n_src * c->m);
    }
    c->proj_grid = static_cast<unsigned>(std::min<uint64_t>(static_cast<uint64_t>(c->sms) * 4,
                                                            std::max<uint64_t>(1, (c->n_src + 255) / 256)));
    const uint64_t scratch_before = c->device_bytes;
    // per-CTA partial sums: the plain projection's grid, or up to one CTA per SM for the INT8 form
    c->d_partials = c->alloc<int32_t>(std::max<uint64_t>(c->proj_grid, c->sms) * c->m * std::max(c->nb, c->nbi));
    c->d_counter = c->alloc<unsigned int>(1);
    c->d_seq_index = c->alloc<unsigned long long>(1);
    c->scratch_bytes = c->device_bytes - scratch_before;
    BW_CUDA(cudaMemsetAsync(c->d_counter, 0, sizeof(unsigned int), st));
    BW_CUDA(cudaMemsetAsync(c->d_seq_index, 0, sizeof(unsigned long long), st));
    if (c->form == BW_FORM_INT8) c->i8_setup();
    if (c->form == BW_FORM_PLAIN) c->plain_setup();
    BW_CUDA(cudaStreamSynchronize(st));
    return c.release();
}

namespace {
// Plain tile heights chosen per operator shape and device, shared by every
// context of the process.
std::mutex g_plain_mutex;
std::map<std::tuple<int, int, int, int, int, int>, std::pair<int, int>> g_plain_tiles;
}  // namespace

// The plain gathers hold a 4- or 8-row output tile per thread (8 rows: twice
// the multiply-adds per gathered row, more registers, and the rows padded to
// a multiple of 8).  Each direction's height is timed at set-up on the
// context's own buffers (one warm-up and two launches; the kernels' work does
// not depend on the values) and the faster kept; BW_PLAIN_TILE=4 or =8 forces
// one height.
void KoszulCtx::plain_setup() {
    int forced = 0;
    if (const char* e = std::getenv("BW_PLAIN_TILE")) forced = std::atoi(e);
    if (forced == 4 || forced == 8) {
        tile_fwd = tile_bwd = forced;
        plain_plan = "plain: " + std::to_string(forced) + " output rows a thread (forced)";
        return;
    }
    const auto key = std::make_tuple(r, k, ci, co, nb, sms);
    {
        std::lock_guard<std::mutex> lock(g_plain_mutex);
        const auto it = g_plain_tiles.find(key);
        if (it != g_plain_tiles.end()) {
            tile_fwd = it->second.first;
            tile_bwd = it->second.second;
            plain_plan = "plain: d " + std::to_string(tile_fwd) + ", d^T " + std::to_string(tile_bwd) +
                         " output rows a thread (tuned earlier in this process)";
            return;
        }
    }
    cudaStream_t st = own_stream;
    BW_CUDA(cudaMemsetAsync(d_ya, 0, n_src * nb * sizeof(int32_t), st));
    BW_CUDA(cudaMemsetAsync(d_z, 0, n_tgt * nb * sizeof(int32_t), st));
    cudaEvent_t e0, e1;
    BW_CUDA(cudaEventCreate(&e0));
    BW_CUDA(cudaEventCreate(&e1));
    auto time_it = [&](bool fwd, int tile) {
        (fwd ? tile_fwd : tile_bwd) = tile;
        auto run = [&] {
            if (fwd)
                plain_forward(d_ya, d_z, st);
            else
                plain_transpose(d_z, d_yb, true, st);
        };
        run();
        BW_CUDA(cudaEventRecord(e0, st));
        run();
        run();
        BW_CUDA(cudaEventRecord(e1, st));
        BW_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        BW_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        return ms / 2;
    };
    char buf[256];
    const float f4 = time_it(true, 4), f8 = time_it(true, 8);
    const float b4 = time_it(false, 4), b8 = time_it(false, 8);
    BW_CUDA(cudaEventDestroy(e0));
    BW_CUDA(cudaEventDestroy(e1));
    tile_fwd = f8 < f4 ? 8 : 4;
    tile_bwd = b8 < b4 ? 8 : 4;
    std::snprintf(buf, sizeof buf,
                  "plain: d %d, d^T %d output rows a thread (tuned: d 4 rows %.4f ms, 8 rows %.4f ms; d^T 4 rows %.4f "
                  "ms, 8 rows %.4f ms)",
                  tile_fwd, tile_bwd, f4, f8, b4, b8);
    plain_plan = buf;
    std::lock_guard<std::mutex> lock(g_plain_mutex);
    g_plain_tiles[key] = {tile_fwd, tile_bwd};
}

template int8_t* KoszulCtx::alloc<int8_t>(uint64_t);
template int16_t* KoszulCtx::alloc<int16_t>(uint64_t);
template int* KoszulCtx::alloc<int>(uint64_t);
template uint32_t* KoszulCtx::alloc<uint32_t>(uint64_t);
template int4* KoszulCtx::alloc<int4>(uint64_t);

void KoszulCtx::release(void* p) {
    auto it = std::find(allocations.begin(), allocations.end(), p);
    if (it != allocations.end()) {
        cudaFree(p);
        allocations.erase(it);
    }
}

// ------------------------------------------------------- sequence session

void KoszulCtx::seq_start(const uint32_t* x, const uint32_t* y0, uint32_t* seq, uint64_t capacity,
                          cudaStream_t st) {
    BW_ARG(x != nullptr && y0 != nullptr && seq != nullptr, "seq_start: null buffer");
    BW_REQUIRE(capacity >= 1, "seq_start: sequence capacity must be at least 1");
    d_seq = seq;
    seq_capacity = capacity;
    cur_is_a = true;
    BW_CUDA(cudaMemsetAsync(d_seq_index, 0, sizeof(unsigned long long), st));
    BW_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(unsigned int), st));
    BW_CUDA(cudaMemsetAsync(d_partials, 0, static_cast<size_t>(m) * std::max(nb, nbi) * sizeof(int32_t), st));
    if (form == BW_FORM_INT8) {
        i8_load_x(x, st);
        i8_to_limbs(y0, I8_YA, st);
        i8_project(I8_YA, st);
    } else {
        launch_to_balanced(x, d_xb, n_src * m, st);
        launch_to_balanced(y0, d_ya, n_src * nb, st);
        project(d_ya, st);
    }
    seq_len = 1;
    // The step graphs capture device pointers: all are the context's own but
    // the sequence buffer, so a session with another buffer recaptures them.
    if (seq != graph_seq) {
        for (auto& g : graphs)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
        graph_seq = seq;
    }
    in_session = true;
}

void KoszulCtx::seq_step(uint64_t steps, cudaStream_t st) {
    BW_REQUIRE(in_session, "seq_step: no sequence session (call bw_koszul_seq_start)");
    BW_REQUIRE(seq_len + steps <= seq_capacity, "seq_step: sequence buffer capacity exceeded");
    // Pairs of steps run as a captured graph (one graph per starting buffer).
    while (steps >= 2 * kGraphPairs) {
        const int gi = cur_is_a ? 0 : 1;
        if (!graphs[gi]) {
            cudaGraph_t graph;
            const bool a0 = cur_is_a;
            const uint64_t launches0 = launches;   // captured launches do not execute
            BW_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            try {
                for (int s = 0; s < 2 * kGraphPairs; ++s) step_once(st);
            } catch (...) {
                cudaStreamEndCapture(st, &graph);
                throw;
            }
            BW_CUDA(cudaStreamEndCapture(st, &graph));
            cur_is_a = a0;   // capture does not execute
            graph_launch_kernels = launches - launches0;
            launches = launches0;
            BW_CUDA(cudaGraphInstantiate(&graphs[gi], graph, 0));
            cudaGraphDestroy(graph);
        }
        BW_CUDA(cudaGraphLaunch(graphs[gi], st));
        launches += graph_launch_kernels;
        seq_len += 2 * kGraphPairs;
        steps -= 2 * kGraphPairs;
    }
    while (steps > 0) {
        step_once(st);
        ++seq_len;
        --steps;
    }
}

uint64_t KoszulCtx::launches_in_pair_graph() const {
    return static_cast<uint64_t>(2 * kGraphPairs) * kernels_per_step();
}

uint64_t KoszulCtx::kernels_per_step() const { return form == BW_FORM_INT8 ? i8_kernels_per_step() : 3; }

void KoszulCtx::seq_finish(uint32_t* y_out, uint64_t* nlen_out, cudaStream_t st) {
    BW_REQUIRE(in_session, "seq_finish: no sequence session");
    in_session = false;
    if (form == BW_FORM_INT8) {
        if (y_out) i8_from_limbs(cur_is_a ? I8_YA : I8_YB, y_out, st);
        BW_CUDA(cudaStreamSynchronize(st));
        i8_check_error();
    } else if (y_out) {
        launch_to_canonical(cur_is_a ? d_ya : d_yb, y_out, n_src * nb, st);
    }
    if (nlen_out) *nlen_out = seq_len;
}

}  // namespace bw

// ------------------------------------------------------------------ C ABI

using namespace bw;

// A NULL stream means "ordered like the legacy default stream": the call's
// work runs on the context's own stream after everything issued before it on
// the legacy stream, and later legacy-stream work waits for it.
struct StreamScope {
    KoszulCtx& c;
    cudaStream_t st;
    bool joined;
    StreamScope(KoszulCtx& ctx, void* stream)
        : c(ctx), st(stream ? static_cast<cudaStream_t>(stream) : ctx.own_stream), joined(stream == nullptr) {
        if (joined) {
            BW_CUDA(cudaEventRecord(c.ev_join, cudaStreamLegacy));
            BW_CUDA(cudaStreamWaitEvent(st, c.ev_join, 0));
        }
    }
    ~StreamScope() {
        if (joined && cudaEventRecord(c.ev_join, st) == cudaSuccess) cudaStreamWaitEvent(cudaStreamLegacy, c.ev_join, 0);
    }
};

extern "C" int bw_koszul_create(const bw_koszul_desc* desc, int device, bw_koszul** out) {
    return guarded([&] {
        BW_ARG(desc != nullptr && out != nullptr, "bw_koszul_create: null argument");
        *out = nullptr;
        KoszulCtx* impl = KoszulCtx::create(*desc, device);
        *out = new bw_koszul{impl};
    });
}

extern "C" int bw_koszul_info_get(const bw_koszul* ctx, bw_koszul_info* out) {
    return guarded([&] {
        BW_ARG(ctx != nullptr && out != nullptr, "bw_koszul_info_get: null argument");
        const KoszulCtx& c = *ctx->impl;
        out->n_src = c.n_src;
        out->n_tgt = c.n_tgt;
        out->device_bytes = c.device_bytes;
        out->scratch_bytes = c.scratch_bytes;
        out->form = c.form;
        out->sm_count = static_cast<uint32_t>(c.sms);
    });
}

extern "C" void bw_koszul_destroy(bw_koszul* ctx) {
    if (!ctx) return;
    delete ctx->impl;
    delete ctx;
}

extern "C" int bw_koszul_forward(bw_koszul* ctx, const uint32_t* d_y, uint32_t* d_z, void* stream) {
    return guarded([&] {
        BW_ARG(ctx && d_y && d_z, "bw_koszul_forward: null argument");
        KoszulCtx& c = *ctx->impl;
        BW_REQUIRE(!c.in_session, "bw_koszul_forward: a sequence session is open");
        BW_CUDA(cudaSetDevice(c.device));
        StreamScope scope(c, stream);
        cudaStream_t st = scope.st;
        if (c.form == BW_FORM_INT8) {
            c.i8_to_limbs(d_y, KoszulCtx::I8_YA, st);
            c.i8_run(true, KoszulCtx::I8_YA, KoszulCtx::I8_Z, false, st);
            c.i8_from_limbs(KoszulCtx::I8_Z, d_z, st);
            BW_CUDA(cudaStreamSynchronize(st));
            c.i8_check_error();
            return;
        }
        c.launch_to_balanced(d_y, c.d_ya, c.n_src * c.nb, st);
        c.plain_forward(c.d_ya, c.d_z, st);
        c.launch_to_canonical(c.d_z, d_z, c.n_tgt * c.nb, st);
    });
}

extern "C" int bw_koszul_transpose(bw_koszul* ctx, const uint32_t* d_z, uint32_t* d_w, int scale_by_diag,
                                   void* stream) {
    return guarded([&] {
        BW_ARG(ctx && d_z && d_w, "bw_koszul_transpose: null argument");
        KoszulCtx& c = *ctx->impl;
        BW_REQUIRE(!c.in_session, "bw_koszul_transpose: a sequence session is open");
        BW_CUDA(cudaSetDevice(c.device));
        StreamScope scope(c, stream);
        cudaStream_t st = scope.st;
        if (c.form == BW_FORM_INT8) {
            c.i8_to_limbs(d_z, KoszulCtx::I8_Z, st);
            c.i8_run(false, KoszulCtx::I8_Z, KoszulCtx::I8_YA, scale_by_diag != 0, st);
            c.i8_from_limbs(KoszulCtx::I8_YA, d_w, st);
            BW_CUDA(cudaStreamSynchronize(st));
            c.i8_check_error();
            return;
        }
        c.launch_to_balanced(d_z, c.d_z, c.n_tgt * c.nb, st);
        c.plain_transpose(c.d_z, c.d_ya, scale_by_diag != 0, st);
        c.launch_to_canonical(c.d_ya, d_w, c.n_src * c.nb, st);
    });
}

extern "C" int bw_koszul_apply(bw_koszul* ctx, const uint32_t* d_y, uint32_t* d_out, void* stream) {
    return guarded([&] {
        BW_ARG(ctx && d_y && d_out, "bw_koszul_apply: null argument");
        KoszulCtx& c = *ctx->impl;
        BW_REQUIRE(!c.in_session, "bw_koszul_apply: a sequence session is open");
        BW_CUDA(cudaSetDevice(c.device));
        StreamScope scope(c, stream);
        cudaStream_t st = scope.st;
        if (c.form == BW_FORM_INT8) {
            c.i8_to_limbs(d_y, KoszulCtx::I8_YA, st);
            c.i8_run(true, KoszulCtx::I8_YA, KoszulCtx::I8_Z, false, st);
            c.i8_run(false, KoszulCtx::I8_Z, KoszulCtx::I8_YB, true, st);
            c.i8_from_limbs(KoszulCtx::I8_YB, d_out, st);
            BW_CUDA(cudaStreamSynchronize(st));
            c.i8_check_error();
            return;
        }
        c.launch_to_balanced(d_y, c.d_ya, c.n_src * c.nb, st);
        c.plain_forward(c.d_ya, c.d_z, st);
        c.plain_transpose(c.d_z, c.d_yb, true, st);
        c.launch_to_canonical(c.d_yb, d_out, c.n_src * c.nb, st);
    });
}

extern "C" int bw_koszul_seq_start(bw_koszul* ctx, const uint32_t* d_x, const uint32_t* d_y0, uint32_t* d_seq,
                                   uint64_t seq_capacity, void* stream) {
    return guarded([&] {
        BW_REQUIRE(ctx != nullptr, "bw_koszul_seq_start: null context");
        KoszulCtx& c = *ctx->impl;
        BW_CUDA(cudaSetDevice(c.device));
        StreamScope scope(c, stream);
        c.seq_start(d_x, d_y0, d_seq, seq_capacity, scope.st);
    });
}

extern "C" int bw_koszul_seq_step(bw_koszul* ctx, uint64_t steps, void* stream) {
    return guarded([&] {
        BW_REQUIRE(ctx != nullptr, "bw_koszul_seq_step: null context");
        KoszulCtx& c = *ctx->impl;
        BW_CUDA(cudaSetDevice(c.device));
        StreamScope scope(c, stream);
        c.seq_step(steps, scope.st);
    });
}

extern "C" int bw_koszul_seq_finish(bw_koszul* ctx, uint32_t* d_y_out, uint64_t* nlen_out, void* stream) {
    return guarded([&] {
        BW_REQUIRE(ctx != nullptr, "bw_koszul_seq_finish: null context");
        KoszulCtx& c = *ctx->impl;
        BW_CUDA(cudaSetDevice(c.device));
        StreamScope scope(c, stream);
        c.seq_finish(d_y_out, nlen_out, scope.st);
    });
}

extern "C" int bw_koszul_sequence_host(bw_koszul* ctx, const uint32_t* h_x, const uint32_t* h_y0, uint64_t nlen,
                                       uint32_t* h_seq, uint32_t* h_y_final) {
    return guarded([&] {
        BW_ARG(ctx && h_x && h_y0 && h_seq, "bw_koszul_sequence_host: null argument");
        BW_REQUIRE(nlen >= 1, "bw_koszul_sequence_host: nlen must be at least 1");
        KoszulCtx& c = *ctx->impl;
        BW_CUDA(cudaSetDevice(c.device));
        cudaStream_t st = c.own_stream;
        const uint64_t entry = static_cast<uint64_t>(c.m) * c.nb;
        c.ensure_host_staging(nlen);
        BW_CUDA(cudaMemcpyAsync(c.d_stage_x, h_x, c.n_src * c.m * 4, cudaMemcpyHostToDevice, st));
        BW_CUDA(cudaMemcpyAsync(c.d_stage_y, h_y0, c.n_src * c.nb * 4, cudaMemcpyHostToDevice, st));
        c.seq_start(c.d_stage_x, c.d_stage_y, c.d_stage_seq, nlen, st);
        c.seq_step(nlen - 1, st);
        c.seq_finish(h_y_final ? c.d_stage_y : nullptr, nullptr, st);
        BW_CUDA(cudaMemcpyAsync(h_seq, c.d_stage_seq, nlen * entry * 4, cudaMemcpyDeviceToHost, st));
        if (h_y_final)
            BW_CUDA(cudaMemcpyAsync(h_y_final, c.d_stage_y, c.n_src * c.nb * 4, cudaMemcpyDeviceToHost, st));
        BW_CUDA(cudaStreamSynchronize(st));
    });
}

extern "C" int bw_koszul_plan(const bw_koszul* ctx, char* buf, size_t cap) {
    return guarded([&] {
        BW_ARG(ctx && buf && cap > 0, "bw_koszul_plan: null argument");
        const KoszulCtx& c = *ctx->impl;
        const std::string text = c.form == BW_FORM_INT8 ? c.i8_plan_text() : c.plain_plan;
        BW_ARG(text.size() < cap, "bw_koszul_plan: buffer too small");
        std::memcpy(buf, text.c_str(), text.size() + 1);
    });
}

extern "C" int bw_koszul_seq_step_timed(bw_koszul* ctx, uint64_t steps, float* ms_out, void* stream) {
    return guarded([&] {
        BW_ARG(ctx != nullptr && ms_out != nullptr, "bw_koszul_seq_step_timed: null argument");
        KoszulCtx& c = *ctx->impl;
        BW_REQUIRE(c.in_session, "bw_koszul_seq_step_timed: no sequence session");
        BW_REQUIRE(c.seq_len + steps <= c.seq_capacity, "bw_koszul_seq_step_timed: capacity exceeded");
        BW_CUDA(cudaSetDevice(c.device));
        StreamScope scope(c, stream);
        cudaStream_t st = scope.st;
        std::vector<cudaEvent_t> ev(4 * steps);
        for (auto& e : ev) BW_CUDA(cudaEventCreate(&e));
        for (uint64_t s = 0; s < steps; ++s) {
            BW_CUDA(cudaEventRecord(ev[4 * s], st));
            if (c.form == BW_FORM_INT8) {
                const int a = c.cur_is_a ? KoszulCtx::I8_YA : KoszulCtx::I8_YB;
                const int b = c.cur_is_a ? KoszulCtx::I8_YB : KoszulCtx::I8_YA;
                c.i8_run(true, a, KoszulCtx::I8_Z, false, st);
                BW_CUDA(cudaEventRecord(ev[4 * s + 1], st));
                c.i8_run(false, KoszulCtx::I8_Z, b, true, st);
                BW_CUDA(cudaEventRecord(ev[4 * s + 2], st));
                c.i8_project(b, st);
            } else {
                int32_t* src = c.cur_is_a ? c.d_ya : c.d_yb;
                int32_t* dst = c.cur_is_a ? c.d_yb : c.d_ya;
                c.plain_forward(src, c.d_z, st);
                BW_CUDA(cudaEventRecord(ev[4 * s + 1], st));
                c.plain_transpose(c.d_z, dst, true, st);
                BW_CUDA(cudaEventRecord(ev[4 * s + 2], st));
                c.project(dst, st);
            }
            BW_CUDA(cudaEventRecord(ev[4 * s + 3], st));
            c.cur_is_a = !c.cur_is_a;
            ++c.seq_len;
        }
        BW_CUDA(cudaStreamSynchronize(st));
        double acc[3] = {0, 0, 0};
        for (uint64_t s = 0; s < steps; ++s)
            for (int kk = 0; kk < 3; ++kk) {
                float ms = 0;
                BW_CUDA(cudaEventElapsedTime(&ms, ev[4 * s + kk], ev[4 * s + kk + 1]));
                acc[kk] += ms;
            }
        for (auto& e : ev) cudaEventDestroy(e);
        for (int kk = 0; kk < 3; ++kk) ms_out[kk] = steps ? static_cast<float>(acc[kk] / steps) : 0.f;
    });
}

extern "C" uint64_t bw_koszul_launch_count(const bw_koszul* ctx) { return ctx ? ctx->impl->launches : 0; }

void bw::KoszulCtx::ensure_host_staging(uint64_t nlen) {
    const uint64_t entry = static_cast<uint64_t>(m) * nb;
    if (!d_stage_x) d_stage_x = alloc<uint32_t>(n_src * m);
    if (!d_stage_y) d_stage_y = alloc<uint32_t>(n_src * nb);
    if (stage_seq_cap < nlen) {
        if (d_stage_seq) release(d_stage_seq);
        d_stage_seq = alloc<uint32_t>(nlen * entry);
        stage_seq_cap = nlen;
    }
}
