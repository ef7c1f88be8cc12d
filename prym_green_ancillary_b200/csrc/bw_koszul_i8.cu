// INT8-limb tensor-core form of the synthetic Koszul operator (tcgen05 kind::i8).
//
// Every residue x (balanced, |x| <= (p-1)/2 < 2^14) is stored in HBM as two
// signed 8-bit limbs in base 255:  x = 255*hi + lo,  lo in [-127, 127],
// hi in [-64, 64] (|x| <= 16383 = 255 * 64 + 63).  The symmetric range makes negation exact in int8, which
// is how the Koszul signs are applied while operands are staged.
//
// One gather-GEMM kernel serves both d and d^T.  For a tile of 128/n output
// blocks (n = block width) the output is
//   out[blk][o][j] = sum_{i < r} sum_{u < inner} A[(blk, j)][(i, u)] * Bm[o][(i, u)]
// with A[(blk, j)][(i, u)] = sign * in[nbr(blk, i)][u][j] (zero when the
// generator i is not incident to blk) and Bm = the r maps side by side.  The
// tile is an M = 128 GEMM: A = the gathered input blocks (MN-major in shared
// memory: 16 limbs of one input row form one 16-byte core-matrix row),
// B = the maps' lo and hi limbs stacked along N (K-major, resident in shared
// memory for the whole kernel), K = r * inner in steps of 32.  Two MMAs per
// K-step (A = input lo limbs, A = input hi limbs) give four int32 partial
// products per output, recombined exactly mod p in the epilogue:
//   x*m = lo*lo + 255*(lo*hi + hi*lo) + 255^2*hi*hi.
// int32 accumulation is exact: |K * 127 * 127| < 2^24 for K <= 1024.
//
// Limb planes in HBM: four planes per block array (lo, hi, -lo, -hi), each
// laid out [blk][h][u][16 bytes] (h = j / 16), so that every (block, h) is one
// contiguous run of inner * 16 bytes.  The producers fill a stage with 16-byte
// cp.async copies (one per K' row, limb and column group) from the +plane or
// the -plane by the Koszul sign; the rows of an absent generator (about half
// of all rows) are zero-filled by the same copy with source size 0, which
// reads nothing (a common zero source in global memory would funnel that half
// of the traffic through one L2 slice).
// The epilogue writes all four planes of its output.
//
// Warp roles (persistent, one CTA per SM; PW = 8 or 16 producer warps, chosen
// per direction by the set-up autotuner):
//   warps 0..PW-1  producers: each owns one of the tile's output blocks (or,
//               with fewer blocks per tile than producer warps, a share of one
//               block's rows) and keeps their incidence rows in registers (one
//               generator per lane); every thread arrives on the stage barrier
//               through cp.async.mbarrier.arrive.noinc when its copies have
//               landed;
//   warp PW     allocates TMEM and issues tcgen05.mma / tcgen05.commit (after a
//               proxy fence: the stage was written through the generic proxy);
//   the rest    epilogue (eight warps with PW = 8, four with PW = 16), one or two
//               warps per TMEM lane quadrant: tcgen05.ld the four partials,
//               recombine, reduce mod p, scale by D (d^T only), split into
//               limbs, transpose 16 x 16 bytes per half-warp and store one
//               16-byte plane row per lane.
// Stages are tracked with mbarriers; accumulators are double-buffered in TMEM.
// Every wait is bounded and polls only a shared-memory give-up flag: on a
// timeout the kernel records an error code, all roles wind down, in-flight
// copies and MMAs are drained and TMEM is freed.
#include "bw_koszul.cuh"
#include "tc_sm100.cuh"

#include <cuda.h>   // CUtensorMap and cuTensorMapEncodeTiled's types (the function is reached through the runtime)

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

namespace bw {

namespace {

constexpr uint32_t kAbsent = 0xFFFFFFFFu;
constexpr int kEpilogueWarps = 8;                 // hybrid kernel; per TMEM lane quadrant: kEpilogueWarps / 4

// Warp roles of the cp.async gather kernel with PW producer warps: PW = 8
// (eight epilogue warps, 17 in all) or PW = 16 (four epilogue warps, 21 in
// all; more copy streams for the same register budget of 96 a thread).
template <int PW>
struct GatherWarps {
    static_assert(PW == 8 || PW == 16, "8 or 16 producer warps");
    static constexpr int producers = PW;
    static constexpr int mma = PW;                        // allocates TMEM, issues the MMAs
    static constexpr int epilogue0 = PW + 1;
    static constexpr int epilogue = PW == 16 ? 4 : 8;     // per TMEM lane quadrant: epilogue / 4
    static constexpr int threads = (PW + 1 + epilogue) * 32;
};
constexpr int kMaxSmem = 227 * 1024;
constexpr int kMaxRowTable = 2048;    // bytes of the K'-row -> generator table

// Plane index inside a four-plane block array.
enum : int { PL_LO = 0, PL_HI = 1, PL_NLO = 2, PL_NHI = 3 };

struct I8Dir {
    const int8_t* in[4];      // input planes lo, hi, -lo, -hi: [blk][h][inner][16]
    long long in_neg_off;     // bytes from an input +plane to its -plane (they share one allocation)
    int8_t* out[4];           // output planes, same layout with `outer`
    const uint32_t* inc;      // [n_blk][r]: neighbour rank | negative << 31, or kAbsent
    const int8_t* b_tiles;    // B operand, already in its shared-memory layout
    const int32_t* diag;      // nullptr, or [n_blk * outer] balanced (scales the output)
    int* err;
    long long n_blk;
    int r, inner, outer, half;   // N = 2 * half, half = outer rounded up to 16
    int gi;                      // generators per stage
    int stages_per_tile;         // ceil(r / gi)
    int ks_full;                 // K-steps of a full stage (gi * inner rows padded to a multiple of 32)
    int ks_last;                 // K-steps of the last stage
    int slots;                   // pipeline depth
    uint32_t b_bytes, slot_bytes, limb_bytes;
    Mod mod;
    int32_t c1, c2;              // 255 and 255^2 mod p, balanced
    uint32_t wait_limit;         // tries of every pipeline wait (tc::kWaitLimit outside the failure tests)
    int hold_first_stage;        // failure tests only: CTA 0's MMA thread never sees its first stage
    // hybrid producer (i8_gather_hybrid_kernel)
    const int4* rows4;           // [n_blk][groups]: plane rows of the four generators of a group (h = 0)
    int groups;                  // ceil(r / 4)
    int gs;                      // groups per stage
    int inner_pad;               // K' rows of a generator: inner rounded up to even (128-byte aligned groups)
    int32_t row_oob;             // a plane row past the input tensor (2 * input blocks * HG): zero-filled
    int t_tma;                   // hybrid producer: output blocks of a tile gathered by TMA (the rest by cp.async)
    uint32_t tx_full, tx_last;   // bytes a full / the last stage of a tile receives
};

// Position in a ring of pipeline slots: slot index and the parity of its
// current phase, advanced without dividing (a 64-bit division per stage would
// sit on the producers' and the MMA thread's critical paths).
struct SlotRing {
    int slot = 0, n = 1;
    uint32_t phase = 0;
    __device__ explicit SlotRing(int count) : n(count) {}
    __device__ void next() {
        if (++slot == n) {
            slot = 0;
            phase ^= 1u;
        }
    }
};

// ll + 255 (lh + hl) + 255^2 hh mod p (balanced); c1 = 255, c2 = 255^2 mod p, balanced.
__device__ __forceinline__ int32_t combine(int32_t ll, int32_t lhhl, int32_t hh, const Mod& mod, int32_t c1,
                                           int32_t c2) {
    const int32_t a = reduce_partial(ll, mod);
    const int32_t b = reduce_partial(lhhl, mod);
    const int32_t c = reduce_partial(hh, mod);
    return reduce_balanced(a + c1 * b + c2 * c, mod);
}

// The gather-GEMM epilogue's value of one output, balanced: ll + 255 (lh + hl)
// + 255^2 hh, times the diagonal entry dg when scaling (d^T).  The sum before
// the last reduction stays below 1.11e9 in magnitude: |ll| <= 1024 * 127^2
// (at most 1024 K rows), 255 * |lh + hl reduced| < 255 * 2p and
// |c2 * hh reduced| < 16383 * 2p; the scaled product is below 2p * (p - 1) / 2.
// Both are within reduce_balanced_fast's range.
__device__ __forceinline__ int32_t epilogue_value(int32_t ll, int32_t lhhl, int32_t hh, const Mod& mod, int32_t c2,
                                                  bool scale, int32_t dg) {
    const int32_t t = ll + 255 * reduce_partial(lhhl, mod) + c2 * reduce_partial(hh, mod);
    return reduce_balanced_fast(scale ? reduce_partial(t, mod) * dg : t, mod);
}

__host__ __device__ __forceinline__ void split_limbs(int32_t v, int8_t& lo, int8_t& hi) {
    // v in [-16383, 16383]: q = floor((v + 127) / 255), lo = v - 255 q in [-127, 127]
    const int32_t q = static_cast<int32_t>(static_cast<uint32_t>(v + 127 + 255 * 128) / 255u) - 128;
    lo = static_cast<int8_t>(v - 255 * q);
    hi = static_cast<int8_t>(q);
}

// 16 x 16 byte transpose inside each half-warp.  On entry lane L (L = lane & 15)
// holds row L as four words (byte b of word q = element 4q + b); on exit it
// holds column L the same way.  Two butterfly stages exchange words (lane bits
// 2 and 3 against word-index bits), two exchange bytes (lane bits 0 and 1
// against byte-index bits, recombined with byte permutes).
__device__ __forceinline__ void transpose16(uint32_t (&w)[4], int lane) {
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const bool upper = (lane >> (k + 2)) & 1;
        const int step = 1 << k;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (q & step) continue;   // the pair (q, q + step)
            const uint32_t send = upper ? w[q] : w[q + step];
            const uint32_t recv = __shfl_xor_sync(0xffffffffu, send, 4 << k);
            if (upper) w[q] = recv;
            else w[q + step] = recv;
        }
    }
    const bool b0 = lane & 1, b1 = (lane >> 1) & 1;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        uint32_t r = __shfl_xor_sync(0xffffffffu, w[q], 1);
        w[q] = __byte_perm(w[q], r, b0 ? 0x3715 : 0x6240);
        r = __shfl_xor_sync(0xffffffffu, w[q], 2);
        w[q] = __byte_perm(w[q], r, b1 ? 0x3276 : 0x5410);
    }
}

// Byte offset of element (row = blk * dim + u, column j) in a plane of width NB.
__host__ __device__ __forceinline__ long long plane_offset(long long blk, int u, int j, int dim, int NB) {
    return blk * (static_cast<long long>(NB) * dim) + static_cast<long long>(j >> 4) * dim * 16 + u * 16 + (j & 15);
}

template <int NB, int PW>
__global__ void __launch_bounds__(GatherWarps<PW>::threads, 1) i8_gather_gemm_kernel(I8Dir P) {
    using W = GatherWarps<PW>;
    constexpr int kProducerWarps = W::producers, kMmaWarp = W::mma, kEpilogueWarp0 = W::epilogue0;
    constexpr int kGatherEpilogueWarps = W::epilogue;
    extern __shared__ __align__(1024) uint8_t smem[];
    constexpr int BT = 128 / NB;        // output blocks per tile
    constexpr int HG = NB / 16;         // 16-byte column groups per block row
    const int N = 2 * P.half;
    uint8_t* sB = smem;
    uint8_t* sA = smem + P.b_bytes;
    uint64_t* full = reinterpret_cast<uint64_t*>(sA + static_cast<size_t>(P.slots) * P.slot_bytes);
    uint64_t* empty = full + P.slots;
    uint64_t* accfull = empty + P.slots;
    uint64_t* accempty = accfull + 2;
    uint64_t* drained = accempty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drained + 1);
    volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);   // CTA give-up flag
    uint8_t* il_of_row = reinterpret_cast<uint8_t*>(tmem_slot + 4);   // K' row of a slot -> generator slot

    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const long long n_tiles = (P.n_blk + BT - 1) / BT;

    // B operand: global -> shared (generic stores, made visible to the tensor core below)
    for (uint32_t off = threadIdx.x * 16; off < P.b_bytes; off += blockDim.x * 16)
        *reinterpret_cast<int4*>(sB + off) = __ldg(reinterpret_cast<const int4*>(P.b_tiles + off));
    tc::fence_proxy_async_smem();
    if (threadIdx.x == 0) {
        for (int s = 0; s < P.slots; ++s) {
            tc::mbar_init(&full[s], kProducerWarps * 32);   // per thread: its copies have landed
            tc::mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            tc::mbar_init(&accfull[b], 1);
            tc::mbar_init(&accempty[b], kGatherEpilogueWarps * 32);
        }
        tc::mbar_init(drained, 1);
        tc::fence_mbar_init();
        *abort = 0;
    }
    const uint32_t tmem_cols = (4 * N <= 256) ? 256u : 512u;
    if (warp == kMmaWarp) {
        tc::tmem_alloc(tmem_slot, tmem_cols);
        tc::tmem_relinquish();
    }
    const int KS = P.ks_full * 32;                       // K' rows of a slot group (gi * inner, padded)
    for (int w = threadIdx.x; w < KS; w += blockDim.x) il_of_row[w] = static_cast<uint8_t>(w / P.inner);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp < kProducerWarps) {
        // ------------------------------------------------------------ producers
        // Warp w stages the output blocks t = w % GROUPS, + GROUPS, ... of each tile.  Lane
        // i holds, for those blocks, where generator i's neighbour run starts: its offset
        // from the limb's +plane in 16-byte units, the -plane's offset added for a negative
        // sign, or kAbsent (read by shuffle; the next tile's entries are loaded one tile
        // ahead).  The warp's lanes walk the K' rows of every (limb, block, column group):
        // a 16-byte cp.async from the +plane or -plane of the neighbour block,
        // or a zero-filling one (source size 0) for an absent generator.  Each
        // thread arrives on the stage barrier once, through
        // cp.async.mbarrier.arrive.noinc, when its copies have landed.
        // More producer warps than blocks: RPW warps share a block, interleaving its rows.
        constexpr int RPW = kProducerWarps > BT ? kProducerWarps / BT : 1;
        constexpr int GROUPS = kProducerWarps / RPW;                     // distinct block positions
        constexpr int TPW = (BT + GROUPS - 1) / GROUPS;                  // blocks per producer warp
        const int group = warp % GROUPS, sub = warp / GROUPS;
        const uint32_t neg16 = static_cast<uint32_t>(P.in_neg_off >> 4);
        const uint32_t run16 = static_cast<uint32_t>(HG * P.inner);   // 16-byte rows of one neighbour block
        auto load_inc = [&](long long tile, uint32_t (&dst)[TPW]) {
#pragma unroll
            for (int k = 0; k < TPW; ++k) {
                const int t = group + k * GROUPS;
                const long long blk = tile * BT + t;
                const uint32_t e = (tile < n_tiles && t < BT && blk < P.n_blk && lane < P.r)
                                       ? __ldg(P.inc + blk * P.r + lane) : kAbsent;
                dst[k] = e == kAbsent ? kAbsent : ((e >> 31) ? neg16 : 0u) + (e & 0x7FFFFFFFu) * run16;
            }
        };
        const uint32_t sA_u32 = tc::smem_u32(sA);
        SlotRing ring(P.slots);
        bool ok = true;
        uint32_t incr[TPW], incn[TPW];
        load_inc(blockIdx.x, incn);
        for (long long tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
#pragma unroll
            for (int k = 0; k < TPW; ++k) incr[k] = incn[k];
            load_inc(tile + gridDim.x, incn);
            for (int s = 0; s < P.stages_per_tile; ++s, ring.next()) {
                const int slot = ring.slot;
                const uint32_t ph = ring.phase;
                int got = 1;
                if (lane == 0)
                    got = tc::mbar_wait(&empty[slot], ph ^ 1u, abort, P.err, tc::ERR_WAIT_EMPTY, P.wait_limit) ? 1 : 0;
                got = __shfl_sync(0xffffffffu, got, 0);
                if (!got) {
                    ok = false;
                    break;
                }
                // failure tests: the first stage of CTA 0 is never filled, so its consumer's wait runs out
                const int g_s = min(P.gi, P.r - s * P.gi);
                const int rows = g_s * P.inner;             // K' rows filled in this stage
                const uint32_t slotA = sA_u32 + static_cast<uint32_t>(slot) * P.slot_bytes;
#pragma unroll
                for (int k = 0; k < TPW; ++k) {
                    const int t = group + k * GROUPS;
                    if (t >= BT) break;
                    for (int w0 = sub * 32; w0 < rows; w0 += RPW * 32) {
                        const int w = w0 + lane;
                        const int il = il_of_row[min(w, rows - 1)];
                        const uint32_t o16 = __shfl_sync(0xffffffffu, incr[k], s * P.gi + il);
                        if (w >= rows) continue;
                        const int b = w - il * P.inner;
                        const uint32_t dst0 = slotA + static_cast<uint32_t>(t * HG * KS + w) * 16u;
                        // one code path for every lane: an absent generator's rows are zero-filled by
                        // the copy itself (source size 0: nothing is read), so the warp does not diverge
                        const bool present = o16 != kAbsent;
                        const uint32_t src16 = (present ? o16 : 0u) + static_cast<uint32_t>(b);
                        const uint32_t nbytes = present ? 16u : 0u;
#pragma unroll
                        for (int limb = 0; limb < 2; ++limb)
#pragma unroll
                            for (int h = 0; h < HG; ++h)
                                tc::cp_async16_zfill(dst0 + static_cast<uint32_t>(limb) * P.limb_bytes +
                                                         static_cast<uint32_t>(h * KS * 16),
                                                     P.in[limb] + static_cast<size_t>(src16 + h * P.inner) * 16u,
                                                     nbytes);
                    }
                }
                tc::cp_async_arrive_noinc(&full[slot]);   // when this thread's copies have landed
            }
        }
        tc::cp_async_wait_all();   // no copy may still be landing when the CTA exits
    } else if (warp == kMmaWarp) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_i8(128, N, true, false);
            const uint32_t sA0 = tc::smem_u32(sA), sB0 = tc::smem_u32(sB);
            const uint32_t a_hi = tc::desc_hi(static_cast<uint32_t>(KS) * 16u), b_hi = tc::desc_hi(256u);
            const uint32_t b_kstep = static_cast<uint32_t>(N) * 32u;   // bytes of B per K-step
            const uint32_t a_limb = P.limb_bytes >> 4;                 // hi limb of A, in descriptor units
            long long tcount = 0;
            SlotRing ring(P.slots);
            bool ok = true;
            bool held = P.hold_first_stage && blockIdx.x == 0;
            for (long long tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x, ++tcount) {
                const int buf = static_cast<int>(tcount & 1);
                const uint32_t aph = static_cast<uint32_t>((tcount >> 1) & 1);
                if (!tc::mbar_wait(&accempty[buf], aph ^ 1u, abort, P.err, tc::ERR_WAIT_ACCUM_FREE, P.wait_limit)) break;
                tc::tc_fence_after();
                const uint32_t dbase = tmem + static_cast<uint32_t>(buf * 2 * N);
                for (int s = 0; s < P.stages_per_tile; ++s, ring.next()) {
                    const int slot = ring.slot;
                    const uint32_t ph = ring.phase;
                    // failure tests: CTA 0 waits for its first stage on a barrier that
                    // nothing completes before the final drain, so the wait runs out
                    uint64_t* wait_bar = (held && s == 0) ? drained : &full[slot];
                    const uint32_t wait_ph = (held && s == 0) ? 0u : ph;
                    held = false;
                    if (!tc::mbar_wait(wait_bar, wait_ph, abort, P.err, tc::ERR_WAIT_FULL, P.wait_limit)) {
                        ok = false;
                        break;
                    }
                    tc::fence_proxy_async_smem();
                    tc::tc_fence_after();
                    const int ks_n = (s == P.stages_per_tile - 1) ? P.ks_last : P.ks_full;
                    // descriptors advance by adding to their low words: A by one K-step (32 rows of
                    // 16 bytes), B by one K-step of the maps (N x 32 bytes); the two limbs of the
                    // input go to the tile's two accumulators
                    const uint32_t a_lo = tc::desc_lo(sA0 + static_cast<uint32_t>(slot) * P.slot_bytes, 128u);
                    const uint32_t b_lo = tc::desc_lo(sB0 + static_cast<uint32_t>(s * P.ks_full) * b_kstep, 128u);
#pragma unroll 2
                    for (int ks = 0; ks < ks_n; ++ks) {
                        const uint64_t bd = tc::desc_make(b_lo + static_cast<uint32_t>(ks) * (b_kstep >> 4), b_hi);
                        const uint32_t acc = (s > 0 || ks > 0) ? 1u : 0u;
                        const uint32_t a_k = a_lo + static_cast<uint32_t>(ks) * (512u >> 4);
                        tc::mma_i8(dbase, tc::desc_make(a_k, a_hi), bd, idesc, acc);
                        tc::mma_i8(dbase + static_cast<uint32_t>(N), tc::desc_make(a_k + a_limb, a_hi), bd, idesc, acc);
                    }
                    tc::mma_commit(&empty[slot]);
                }
                if (!ok) break;
                tc::mma_commit(&accfull[buf]);
            }
            // drain: every MMA issued above completes before TMEM is released
            // (this wait ignores the give-up flag; issued MMAs always finish)
            tc::mma_commit(drained);
            tc::mbar_wait(drained, 0, nullptr, P.err, tc::ERR_WAIT_FINAL);
        }
        __syncwarp();
    } else {
        // ------------------------------------------------------------ epilogue
        // Warps PW+1 on: warp & 3 is the TMEM lane quadrant a warp may read; the
        // warps of a quadrant (two with PW = 8, one with PW = 16) split the
        // 16-column output chunks between them.
        const int q = warp & 3;
        constexpr int EPQ = kGatherEpilogueWarps / 4;          // epilogue warps per quadrant
        const int half_id = (warp - kEpilogueWarp0) >> 2;      // this warp's part of the chunks
        const int m = q * 32 + lane;               // tile row = (block t, column j)
        const int t = m / NB, j = m % NB;
        const uint32_t lane_off = static_cast<uint32_t>(q * 32) << 16;
        const int chunks = P.half / 16;
        const uint32_t h_off = static_cast<uint32_t>((j >> 4) * P.outer * 16);   // this half-warp's column group
        long long tcount = 0;
        for (long long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x, ++tcount) {
            const int buf = static_cast<int>(tcount & 1);
            const uint32_t aph = static_cast<uint32_t>((tcount >> 1) & 1);
            const long long blk = tile * BT + t;
            const bool valid = blk < P.n_blk;
            // prefetch the diagonal entries of this warp's first chunk before waiting for the accumulator
            int32_t dg[16];
            auto load_diag = [&](int c) {
#pragma unroll
                for (int oo = 0; oo < 16; ++oo) {
                    const int o = c * 16 + oo;
                    dg[oo] = (P.diag && valid && o < P.outer) ? __ldg(P.diag + blk * P.outer + o) : 0;
                }
            };
            load_diag(half_id);
            if (!tc::mbar_wait(&accfull[buf], aph, abort, P.err, tc::ERR_WAIT_ACCUM, P.wait_limit)) break;
            tc::tc_fence_after();
            const uint32_t col0 = tmem + lane_off + static_cast<uint32_t>(buf * 2 * N);
            const long long base = blk * static_cast<long long>(NB) * P.outer;
            int8_t* o_lo = P.out[PL_LO] + base;
            int8_t* o_hi = P.out[PL_HI] + base;
            int8_t* o_nlo = P.out[PL_NLO] + base;
            int8_t* o_nhi = P.out[PL_NHI] + base;
            for (int c = half_id; c < chunks; c += EPQ) {
                const int o0 = c * 16;
                if (c != half_id) load_diag(c);
                // this lane's 16 outputs (o0..o0+15 of its column j) as limb bytes; columns o >= outer
                // hold zeros (zero rows of the maps, zero diagonal entries) and are not stored
                uint32_t lw[4] = {0, 0, 0, 0}, hw[4] = {0, 0, 0, 0};
                // Eight columns at a time (the four partials of eight outputs live together), and only
                // the groups of four columns that reach below outer need arithmetic (the rest stay zero).
                const int live = P.outer - o0;
                const bool scale = P.diag != nullptr;
#pragma unroll
                for (int h8 = 0; h8 < 2; ++h8) {
                    if (h8 * 8 >= live) break;
                    int32_t ll[8], lh[8], hl[8], hh[8];
                    const uint32_t cb = col0 + static_cast<uint32_t>(o0 + h8 * 8);
                    tc::tmem_ld8(cb, ll);
                    tc::tmem_ld8(cb + P.half, lh);
                    tc::tmem_ld8(cb + N, hl);
                    tc::tmem_ld8(cb + N + P.half, hh);
                    tc::tmem_ld_wait();
#pragma unroll
                    for (int q = 0; q < 2; ++q) {
                        if (h8 * 8 + q * 4 >= live) break;
#pragma unroll
                        for (int oi = 0; oi < 4; ++oi) {
                            const int oo = q * 4 + oi;
                            const int32_t v = epilogue_value(ll[oo], lh[oo] + hl[oo], hh[oo], P.mod, P.c2, scale,
                                                             dg[h8 * 8 + oo]);
                            int8_t lo, hi;
                            split_limbs(v, lo, hi);
                            lw[h8 * 2 + q] |= static_cast<uint32_t>(static_cast<uint8_t>(lo)) << (8 * oi);
                            hw[h8 * 2 + q] |= static_cast<uint32_t>(static_cast<uint8_t>(hi)) << (8 * oi);
                        }
                    }
                }
                // transposed, lane L of the half-warp holds output row o0 + L: 16 bytes, one per j
                transpose16(lw, lane);
                transpose16(hw, lane);
                const int o = o0 + (lane & 15);
                if (valid && o < P.outer) {
                    const uint32_t off = h_off + static_cast<uint32_t>(o) * 16u;
                    *reinterpret_cast<uint4*>(o_lo + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
                    *reinterpret_cast<uint4*>(o_hi + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
                    *reinterpret_cast<uint4*>(o_nlo + off) =
                        make_uint4(neg_bytes4(lw[0]), neg_bytes4(lw[1]), neg_bytes4(lw[2]), neg_bytes4(lw[3]));
                    *reinterpret_cast<uint4*>(o_nhi + off) =
                        make_uint4(neg_bytes4(hw[0]), neg_bytes4(hw[1]), neg_bytes4(hw[2]), neg_bytes4(hw[3]));
                }
            }
            tc::tc_fence_before();
            tc::mbar_arrive(&accempty[buf]);
        }
    }

    tc::tc_fence_before();
    __syncthreads();
    if (warp == kMmaWarp) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, tmem_cols);
    }
}

// ---- gather-GEMM with a hybrid producer: TMA gathers beside cp.async warps
//
// Same tile, MMA issue and epilogue as i8_gather_gemm_kernel; a stage holds
// gs groups of four generators, each generator inner_pad (inner rounded up to
// even) K' rows, so that every group starts 128-byte aligned.  The tile's
// output blocks t < t_tma are filled by the tensor-memory accelerator, the
// others by eight cp.async warps, both into the same stage and completing on
// the same barrier (257 arrivals: one per cp.async thread when its copies have
// landed, one from the TMA warp with the stage's TMA byte count), so the two
// copy engines work side by side.
//
// TMA part: the +plane and the -plane of a limb are one 2-D tensor (rows =
// (block, h) runs of inner * 16 bytes, the -plane's rows after the +plane's),
// so one tile::gather4 copies the runs of four neighbour blocks, each from the
// plane its Koszul sign selects: row = neg * n_blk_in * HG + nbr * HG + h,
// precomputed on the host per group of four generators (rows4).  An absent
// generator (or a padding generator past r) has a row beyond the tensor: the
// copy fills its rows with zeros and reads nothing.  The odd padding row of a
// generator is beyond the tensor's row width (zero-filled) and meets zero rows
// of the maps.
//
// cp.async part: as in i8_gather_gemm_kernel (16-byte copies from the +plane
// or -plane, zero-filling ones for absent generators), with the rows of a
// block shared by 8 / (BT - t_tma) warps.
//
// Warp roles: warps 0-7 cp.async producers, warp 8 TMA producer, warp 9 MMA
// issuer (allocates TMEM), warps 10-17 epilogue.  On a give-up every producer
// still waits (bounded) for the copies it issued before the CTA exits.
constexpr int kCpWarps = 8;
constexpr int kTmaWarp = kCpWarps;
constexpr int kHyMmaWarp = kCpWarps + 1;
constexpr int kHyEpi0 = kCpWarps + 2;
constexpr int kHyThreads = (kCpWarps + 2 + kEpilogueWarps) * 32;

template <int NB>
__global__ void __launch_bounds__(kHyThreads, 1)
    i8_gather_hybrid_kernel(const __grid_constant__ CUtensorMap map_lo, const __grid_constant__ CUtensorMap map_hi,
                            I8Dir P) {
    extern __shared__ __align__(1024) uint8_t smem[];
    constexpr int BT = 128 / NB;        // output blocks per tile
    constexpr int HG = NB / 16;         // 16-byte column groups per block row
    constexpr int kMaxSlots = 8;
    const int N = 2 * P.half;
    uint8_t* sB = smem;
    uint8_t* sA = smem + P.b_bytes;
    uint64_t* full = reinterpret_cast<uint64_t*>(sA + static_cast<size_t>(P.slots) * P.slot_bytes);
    uint64_t* empty = full + P.slots;
    uint64_t* accfull = empty + P.slots;
    uint64_t* accempty = accfull + 2;
    uint64_t* drained = accempty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drained + 1);
    volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);   // CTA give-up flag
    uint8_t* il_of_row = reinterpret_cast<uint8_t*>(tmem_slot + 4);        // K' row -> generator in stage (255: pad)

    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const long long n_tiles = (P.n_blk + BT - 1) / BT;
    const int KS = P.ks_full * 32;                    // K' rows of a slot's column (full stage, padded)
    // every TMA destination is 128-byte aligned relative to the base
    if ((tc::smem_u32(smem) & 127u) != 0 || P.slots > kMaxSlots || P.t_tma < 0 || P.t_tma > BT ||
        KS > kMaxRowTable) {
        if (threadIdx.x == 0) atomicCAS(P.err, tc::ERR_NONE, tc::ERR_LAYOUT);
        return;
    }

    for (uint32_t off = threadIdx.x * 16; off < P.b_bytes; off += blockDim.x * 16)
        *reinterpret_cast<int4*>(sB + off) = __ldg(reinterpret_cast<const int4*>(P.b_tiles + off));
    tc::fence_proxy_async_smem();
    for (int w = threadIdx.x; w < KS; w += blockDim.x) {
        const int il = w / P.inner_pad, u = w - il * P.inner_pad;
        il_of_row[w] = static_cast<uint8_t>(u < P.inner ? il : 255);
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < P.slots; ++s) {
            tc::mbar_init(&full[s], kCpWarps * 32 + 1);   // cp.async threads + the TMA warp's expect_tx arrive
            tc::mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            tc::mbar_init(&accfull[b], 1);
            tc::mbar_init(&accempty[b], kEpilogueWarps * 32);
        }
        tc::mbar_init(drained, 1);
        tc::fence_mbar_init();
        *abort = 0;
    }
    const uint32_t tmem_cols = (4 * N <= 256) ? 256u : 512u;
    if (warp == kHyMmaWarp) {
        tc::tmem_alloc(tmem_slot, tmem_cols);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp < kCpWarps) {
        // ------------------------------------------------------------ cp.async producers
        // Blocks t_tma..BT-1 of every tile; a block's stage rows are shared by
        // wpb = 8 / n_cp warps (interleaved by 32 rows); lane i holds the
        // incidence entry of generator i for its warp's block (the next tile's
        // entry is loaded one tile ahead).  Every producer thread arrives once
        // per stage, after waiting for the slot to be free.
        const int n_cp = BT - P.t_tma;
        const int wpb = n_cp > 0 ? kCpWarps / n_cp : 1;
        const bool active = n_cp > 0 && warp < n_cp * wpb;
        const int t = active ? P.t_tma + warp / wpb : 0, sub = active ? warp % wpb : 0;
        // lane i: where generator i's neighbour run starts (16-byte units from the limb's +plane,
        // the -plane's offset added for a negative sign), or kAbsent
        const uint32_t neg16 = static_cast<uint32_t>(P.in_neg_off >> 4);
        const uint32_t run16 = static_cast<uint32_t>(HG * P.inner);
        auto load_inc = [&](long long tile) -> uint32_t {
            const long long blk = tile * BT + t;
            const uint32_t e = (active && tile < n_tiles && blk < P.n_blk && lane < P.r)
                                   ? __ldg(P.inc + blk * P.r + lane) : kAbsent;
            return e == kAbsent ? kAbsent : ((e >> 31) ? neg16 : 0u) + (e & 0x7FFFFFFFu) * run16;
        };
        const uint32_t sA_u32 = tc::smem_u32(sA);
        SlotRing ring(P.slots);
        bool ok = true;
        uint32_t incn = load_inc(blockIdx.x);
        for (long long tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
            const uint32_t incr = incn;
            incn = load_inc(tile + gridDim.x);
            for (int s = 0; s < P.stages_per_tile; ++s, ring.next()) {
                const int slot = ring.slot;
                const uint32_t ph = ring.phase;
                int got = 1;
                if (lane == 0)
                    got = tc::mbar_wait(&empty[slot], ph ^ 1u, abort, P.err, tc::ERR_WAIT_EMPTY, P.wait_limit) ? 1 : 0;
                got = __shfl_sync(0xffffffffu, got, 0);
                if (!got) {
                    ok = false;
                    break;
                }
                if (active) {
                    const bool last = s == P.stages_per_tile - 1;
                    const int rows = (last ? P.groups - s * P.gs : P.gs) * 4 * P.inner_pad;
                    const uint32_t col0 = sA_u32 + static_cast<uint32_t>(slot) * P.slot_bytes +
                                          static_cast<uint32_t>(t * HG * KS) * 16u;
                    for (int w0 = sub * 32; w0 < rows; w0 += wpb * 32) {
                        const int w = w0 + lane;
                        const int il = il_of_row[min(w, rows - 1)];
                        const int gen = s * P.gi + (il == 255 ? 0 : il);
                        const uint32_t o16 = __shfl_sync(0xffffffffu, incr, min(gen, 31));
                        // padding rows and generators past r: their B rows are zero, nothing to copy
                        if (w >= rows || il == 255 || gen >= P.r) continue;
                        const int u = w - il * P.inner_pad;
                        const bool present = o16 != kAbsent;
                        const uint32_t src16 = (present ? o16 : 0u) + static_cast<uint32_t>(u);
                        const uint32_t nbytes = present ? 16u : 0u;
                        const uint32_t dst0 = col0 + static_cast<uint32_t>(w) * 16u;
#pragma unroll
                        for (int limb = 0; limb < 2; ++limb)
#pragma unroll
                            for (int h = 0; h < HG; ++h)
                                tc::cp_async16_zfill(dst0 + static_cast<uint32_t>(limb) * P.limb_bytes +
                                                         static_cast<uint32_t>(h * KS * 16),
                                                     P.in[limb] + static_cast<size_t>(src16 + h * P.inner) * 16u,
                                                     nbytes);
                    }
                }
                tc::cp_async_arrive_noinc(&full[slot]);   // when this thread's copies have landed
            }
        }
        tc::cp_async_wait_all();   // no copy may still be landing when the CTA exits
    } else if (warp == kTmaWarp) {
        // ------------------------------------------------------------ TMA producer
        // Blocks 0..t_tma-1: stage s holds groups s * gs .. of every (block,
        // limb, h): 2 * t_tma * HG * g_n gathers; lane j issues j, j + 32, ...
        // Lane 0 posts the stage's TMA byte count first (an arrive with zero
        // bytes when t_tma = 0).
        tc::prefetch_tmap(&map_lo);
        tc::prefetch_tmap(&map_hi);
        const int32_t oob = P.row_oob;   // beyond the input tensor: zero rows, nothing read
        const uint32_t gbytes = static_cast<uint32_t>(P.inner_pad) * 64;   // one group: 4 generators x inner_pad rows
        SlotRing ring(P.slots);
        uint32_t issued_phase[kMaxSlots];
        bool issued[kMaxSlots];
#pragma unroll
        for (int q = 0; q < kMaxSlots; ++q) issued[q] = false, issued_phase[q] = 0;
        bool ok = true;
        for (long long tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
            for (int s = 0; s < P.stages_per_tile; ++s, ring.next()) {
                const int slot = ring.slot;
                const uint32_t ph = ring.phase;
                int got = 1;
                if (lane == 0)
                    got = tc::mbar_wait(&empty[slot], ph ^ 1u, abort, P.err, tc::ERR_WAIT_EMPTY, P.wait_limit) ? 1 : 0;
                got = __shfl_sync(0xffffffffu, got, 0);
                if (!got) {
                    ok = false;
                    break;
                }
                const bool last = s == P.stages_per_tile - 1;
                const int g_n = last ? P.groups - s * P.gs : P.gs;   // groups in this stage
                const int n_g = 2 * P.t_tma * HG * g_n;
                if (lane == 0) tc::mbar_arrive_expect_tx(&full[slot], static_cast<uint32_t>(n_g) * gbytes);
                __syncwarp();
                uint8_t* slotA = sA + static_cast<size_t>(slot) * P.slot_bytes;
                for (int j = lane; j < n_g; j += 32) {
                    const int gl = j % g_n;                 // group within the stage
                    const int rest = j / g_n;
                    const int limb = rest & 1;
                    const int col = rest >> 1;              // t * HG + h, t < t_tma
                    const int tt = col / HG, h = col - (col / HG) * HG;
                    const long long blk = tile * BT + tt;
                    int4 rr = make_int4(oob, oob, oob, oob);
                    if (blk < P.n_blk) rr = __ldg(P.rows4 + blk * P.groups + s * P.gs + gl);
                    uint8_t* dst = slotA + static_cast<size_t>(limb) * P.limb_bytes +
                                   static_cast<size_t>(col) * KS * 16 + static_cast<size_t>(gl) * gbytes;
                    tc::tma_gather4(dst, limb ? static_cast<const void*>(&map_hi) : static_cast<const void*>(&map_lo),
                                    0, rr.x + h, rr.y + h, rr.z + h, rr.w + h, &full[slot]);
                }
                if (n_g > 0) {
                    issued[slot] = true;
                    issued_phase[slot] = ph;
                }
            }
        }
        // no copy may still be landing when the CTA exits: wait (bounded) for
        // the last stage with gathers in every slot (a consumed stage has completed)
        if (lane == 0) {
#pragma unroll
            for (int q = 0; q < kMaxSlots; ++q)
                if (q < P.slots && issued[q]) tc::mbar_wait(&full[q], issued_phase[q], nullptr, P.err, tc::ERR_WAIT_FINAL);
        }
        __syncwarp();
    } else if (warp == kHyMmaWarp) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_i8(128, N, true, false);
            const uint32_t sA0 = tc::smem_u32(sA), sB0 = tc::smem_u32(sB);
            const uint32_t a_hi = tc::desc_hi(static_cast<uint32_t>(KS) * 16u), b_hi = tc::desc_hi(256u);
            const uint32_t b_kstep = static_cast<uint32_t>(N) * 32u;   // bytes of B per K-step
            const uint32_t a_limb = P.limb_bytes >> 4;                 // hi limb of A, in descriptor units
            long long tcount = 0;
            SlotRing ring(P.slots);
            bool ok = true;
            bool held = P.hold_first_stage && blockIdx.x == 0;
            for (long long tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x, ++tcount) {
                const int buf = static_cast<int>(tcount & 1);
                const uint32_t aph = static_cast<uint32_t>((tcount >> 1) & 1);
                if (!tc::mbar_wait(&accempty[buf], aph ^ 1u, abort, P.err, tc::ERR_WAIT_ACCUM_FREE, P.wait_limit)) break;
                tc::tc_fence_after();
                const uint32_t dbase = tmem + static_cast<uint32_t>(buf * 2 * N);
                for (int s = 0; s < P.stages_per_tile; ++s, ring.next()) {
                    const int slot = ring.slot;
                    const uint32_t ph = ring.phase;
                    // failure tests: CTA 0 waits for its first stage on a barrier that
                    // nothing completes before the final drain, so the wait runs out
                    uint64_t* wait_bar = (held && s == 0) ? drained : &full[slot];
                    const uint32_t wait_ph = (held && s == 0) ? 0u : ph;
                    held = false;
                    if (!tc::mbar_wait(wait_bar, wait_ph, abort, P.err, tc::ERR_WAIT_FULL, P.wait_limit)) {
                        ok = false;
                        break;
                    }
                    // the cp.async part was written through the generic proxy
                    tc::fence_proxy_async_smem();
                    tc::tc_fence_after();
                    const int ks_n = (s == P.stages_per_tile - 1) ? P.ks_last : P.ks_full;
                    // descriptors advance by adding to their low words: A by one K-step (32 rows of
                    // 16 bytes), B by one K-step of the maps (N x 32 bytes); the two limbs of the
                    // input go to the tile's two accumulators
                    const uint32_t a_lo = tc::desc_lo(sA0 + static_cast<uint32_t>(slot) * P.slot_bytes, 128u);
                    const uint32_t b_lo = tc::desc_lo(sB0 + static_cast<uint32_t>(s * P.ks_full) * b_kstep, 128u);
#pragma unroll 2
                    for (int ks = 0; ks < ks_n; ++ks) {
                        const uint64_t bd = tc::desc_make(b_lo + static_cast<uint32_t>(ks) * (b_kstep >> 4), b_hi);
                        const uint32_t acc = (s > 0 || ks > 0) ? 1u : 0u;
                        const uint32_t a_k = a_lo + static_cast<uint32_t>(ks) * (512u >> 4);
                        tc::mma_i8(dbase, tc::desc_make(a_k, a_hi), bd, idesc, acc);
                        tc::mma_i8(dbase + static_cast<uint32_t>(N), tc::desc_make(a_k + a_limb, a_hi), bd, idesc, acc);
                    }
                    tc::mma_commit(&empty[slot]);
                }
                if (!ok) break;
                tc::mma_commit(&accfull[buf]);
            }
            // drain: every MMA issued above completes before TMEM is released
            tc::mma_commit(drained);
            tc::mbar_wait(drained, 0, nullptr, P.err, tc::ERR_WAIT_FINAL);
        }
        __syncwarp();
    } else {
        // ------------------------------------------------------------ epilogue
        // Warps 10..17: warp & 3 is the TMEM lane quadrant it may read; the two
        // warps of a quadrant split the 16-column output chunks between them.
        const int q = warp & 3;
        constexpr int EPQ = kEpilogueWarps / 4;
        const int half_id = (warp - kHyEpi0) >> 2;
        const int m = q * 32 + lane;               // tile row = (block t, column j)
        const int t = m / NB, j = m % NB;
        const uint32_t lane_off = static_cast<uint32_t>(q * 32) << 16;
        const int chunks = P.half / 16;
        const uint32_t h_off = static_cast<uint32_t>((j >> 4) * P.outer * 16);
        long long tcount = 0;
        for (long long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x, ++tcount) {
            const int buf = static_cast<int>(tcount & 1);
            const uint32_t aph = static_cast<uint32_t>((tcount >> 1) & 1);
            const long long blk = tile * BT + t;
            const bool valid = blk < P.n_blk;
            int32_t dg[16];
            auto load_diag = [&](int c) {
#pragma unroll
                for (int oo = 0; oo < 16; ++oo) {
                    const int o = c * 16 + oo;
                    dg[oo] = (P.diag && valid && o < P.outer) ? __ldg(P.diag + blk * P.outer + o) : 0;
                }
            };
            load_diag(half_id);
            if (!tc::mbar_wait(&accfull[buf], aph, abort, P.err, tc::ERR_WAIT_ACCUM, P.wait_limit)) break;
            tc::tc_fence_after();
            const uint32_t col0 = tmem + lane_off + static_cast<uint32_t>(buf * 2 * N);
            const long long base = blk * static_cast<long long>(NB) * P.outer;
            int8_t* o_lo = P.out[PL_LO] + base;
            int8_t* o_hi = P.out[PL_HI] + base;
            int8_t* o_nlo = P.out[PL_NLO] + base;
            int8_t* o_nhi = P.out[PL_NHI] + base;
            for (int c = half_id; c < chunks; c += EPQ) {
                const int o0 = c * 16;
                if (c != half_id) load_diag(c);
                uint32_t lw[4] = {0, 0, 0, 0}, hw[4] = {0, 0, 0, 0};
                // Eight columns at a time (the four partials of eight outputs live together), and only
                // the groups of four columns that reach below outer need arithmetic (the rest stay zero).
                const int live = P.outer - o0;
                const bool scale = P.diag != nullptr;
#pragma unroll
                for (int h8 = 0; h8 < 2; ++h8) {
                    if (h8 * 8 >= live) break;
                    int32_t ll[8], lh[8], hl[8], hh[8];
                    const uint32_t cb = col0 + static_cast<uint32_t>(o0 + h8 * 8);
                    tc::tmem_ld8(cb, ll);
                    tc::tmem_ld8(cb + P.half, lh);
                    tc::tmem_ld8(cb + N, hl);
                    tc::tmem_ld8(cb + N + P.half, hh);
                    tc::tmem_ld_wait();
#pragma unroll
                    for (int q = 0; q < 2; ++q) {
                        if (h8 * 8 + q * 4 >= live) break;
#pragma unroll
                        for (int oi = 0; oi < 4; ++oi) {
                            const int oo = q * 4 + oi;
                            const int32_t v = epilogue_value(ll[oo], lh[oo] + hl[oo], hh[oo], P.mod, P.c2, scale,
                                                             dg[h8 * 8 + oo]);
                            int8_t lo, hi;
                            split_limbs(v, lo, hi);
                            lw[h8 * 2 + q] |= static_cast<uint32_t>(static_cast<uint8_t>(lo)) << (8 * oi);
                            hw[h8 * 2 + q] |= static_cast<uint32_t>(static_cast<uint8_t>(hi)) << (8 * oi);
                        }
                    }
                }
                transpose16(lw, lane);
                transpose16(hw, lane);
                const int o = o0 + (lane & 15);
                if (valid && o < P.outer) {
                    const uint32_t off = h_off + static_cast<uint32_t>(o) * 16u;
                    *reinterpret_cast<uint4*>(o_lo + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
                    *reinterpret_cast<uint4*>(o_hi + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
                    *reinterpret_cast<uint4*>(o_nlo + off) =
                        make_uint4(neg_bytes4(lw[0]), neg_bytes4(lw[1]), neg_bytes4(lw[2]), neg_bytes4(lw[3]));
                    *reinterpret_cast<uint4*>(o_nhi + off) =
                        make_uint4(neg_bytes4(hw[0]), neg_bytes4(hw[1]), neg_bytes4(hw[2]), neg_bytes4(hw[3]));
                }
            }
            tc::tc_fence_before();
            tc::mbar_arrive(&accempty[buf]);
        }
    }

    tc::tc_fence_before();
    __syncthreads();
    if (warp == kHyMmaWarp) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, tmem_cols);
    }
}

// ---- limb conversions and the projection on limb planes

// canonical row-major (rows = n_blk * dim, w_in columns) -> four planes of NB
// columns (columns w_in..NB-1 are zero)
template <int NB>
__global__ void to_limbs_kernel(const uint32_t* __restrict__ in, int8_t* __restrict__ lo, int8_t* __restrict__ hi,
                                int8_t* __restrict__ nlo, int8_t* __restrict__ nhi, long long count, int dim,
                                int w_in, Mod mod) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long row = i / NB;
        const int j = static_cast<int>(i - row * NB);
        int8_t a = 0, b = 0;
        if (j < w_in) split_limbs(to_balanced(in[row * w_in + j] % static_cast<uint32_t>(mod.p), mod), a, b);
        const long long blk = row / dim;
        const long long off = plane_offset(blk, static_cast<int>(row - blk * dim), j, dim, NB);
        lo[off] = a;
        hi[off] = b;
        nlo[off] = static_cast<int8_t>(-a);
        nhi[off] = static_cast<int8_t>(-b);
    }
}

// four planes of NB columns -> canonical row-major with the first w_out columns
template <int NB>
__global__ void from_limbs_kernel(const int8_t* __restrict__ lo, const int8_t* __restrict__ hi,
                                  uint32_t* __restrict__ out, long long count, int dim, int w_out, Mod mod) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long row = i / w_out;
        const int j = static_cast<int>(i - row * w_out);
        const long long blk = row / dim;
        const long long off = plane_offset(blk, static_cast<int>(row - blk * dim), j, dim, NB);
        out[i] = to_canonical(255 * static_cast<int32_t>(hi[off]) + lo[off], mod);
    }
}

// ---- projection a = X^T W on the tensor cores
//
// K = the source rows.  A = X in limbs: M rows = the lo limbs of the m
// projection columns in groups of 16, then their hi limbs (MN-major; laid out
// once per session as one contiguous tile per stage).  B = the lo and hi
// planes of W side by side (N = 2 NB, MN-major: one 16-byte plane row is one
// core-matrix row, so a block's rows copy straight from HBM).  A stage is SB
// whole source blocks, SB * dim rows padded to KP (a multiple of 32); the
// padding rows of the X tile are zero, so whatever the stage buffer holds
// there adds nothing.  The M = 128 descriptor also reads past the X tile: the
// TMEM rows at and above 32 * MG are never read back.
//   D[lo x][j]      = sum lo(X) lo(W),   D[lo x][NB + j] = sum lo(X) hi(W),
//   D[hi x][j]      = sum hi(X) lo(W),   D[hi x][NB + j] = sum hi(X) hi(W)
// int32 accumulation is exact for at most 2^31 / 127^2 > 131072 rows, so the
// accumulator is drained (double-buffered) every `drain` stages.
//
// Warps: 0 producer (bulk copies: the stage's X tile and W block runs), 1 MMA
// issuer (allocates TMEM), 2-5 epilogue (tcgen05.ld + reduction mod p).  The
// CTA's combined sums are added into an m x n int32 accumulator; the last CTA
// to finish writes them to seq[*seq_index], clears them and advances the index.
constexpr int kProjThreads = 6 * 32;
constexpr int kProjStageTarget = 32 * 1024;   // bytes of X tile + W runs per stage

struct I8Proj {
    const int8_t* xt;           // [stage][2 MG][KP][16]
    const int8_t* w[2];         // W lo, hi planes: [blk][h][u][16]
    int32_t* partials;          // [m][NB] accumulator, zero between launches
    unsigned int* counter;
    uint32_t* seq;
    unsigned long long* seq_index;
    int* err;
    long long n_blk;
    int dim, m, mg, sb, kp, n_stages, slots, drain;
    int n_out;                  // columns of W that are the caller's (the rest are zero padding)
    uint32_t a_bytes, slot_bytes, pad_bytes;
    Mod mod;
    int32_t c1, c2;
    uint32_t wait_limit;        // tries of every pipeline wait (tc::kWaitLimit outside the failure tests)
};

template <int NB>
__global__ void __launch_bounds__(kProjThreads, 1) i8_project_tc_kernel(I8Proj P) {
    extern __shared__ __align__(1024) uint8_t smem[];
    constexpr int HG = NB / 16;
    constexpr int N = 2 * NB;
    int32_t* red = reinterpret_cast<int32_t*>(smem + static_cast<size_t>(P.slots) * P.slot_bytes + P.pad_bytes);
    uint64_t* full = reinterpret_cast<uint64_t*>(red + 32 * P.mg * N);
    uint64_t* empty = full + P.slots;
    uint64_t* accfull = empty + P.slots;
    uint64_t* accempty = accfull + 2;
    uint64_t* drained = accempty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drained + 1);
    volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);
    __shared__ bool am_last;

    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const long long n_my = blockIdx.x < P.n_stages ? (P.n_stages - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    const long long n_chunks = (n_my + P.drain - 1) / P.drain;
    const uint32_t tmem_cols = 2 * N;   // two accumulators (64 or 128 columns)
    if (threadIdx.x == 0) {
        for (int s = 0; s < P.slots; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            tc::mbar_init(&accfull[b], 1);
            tc::mbar_init(&accempty[b], 4 * 32);
        }
        tc::mbar_init(drained, 1);
        tc::fence_mbar_init();
        *abort = 0;
    }
    if (warp == 1) {
        tc::tmem_alloc(tmem_slot, tmem_cols);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t run_bytes = static_cast<uint32_t>(P.dim) * 16;   // one (block, h) run of a plane

    if (warp == 0) {
        // ------------------------------------------------------------ producer
        SlotRing ring(P.slots);
        for (long long i = 0; i < n_my; ++i, ring.next()) {
            const int slot = ring.slot;
            const uint32_t ph = ring.phase;
            const long long st = blockIdx.x + i * gridDim.x;
            const long long blk0 = st * P.sb;
            const int nbh = static_cast<int>(min(static_cast<long long>(P.sb), P.n_blk - blk0));
            int got = 1;
            if (lane == 0) {
                got = tc::mbar_wait(&empty[slot], ph ^ 1u, abort, P.err, tc::ERR_WAIT_EMPTY, P.wait_limit) ? 1 : 0;
                if (got)
                    tc::mbar_arrive_expect_tx(&full[slot], P.a_bytes + 2u * HG * nbh * run_bytes);
            }
            got = __shfl_sync(0xffffffffu, got, 0);
            if (!got) break;
            uint8_t* sA = smem + static_cast<size_t>(slot) * P.slot_bytes;
            uint8_t* sB = sA + P.a_bytes;
            const uint32_t group_bytes = static_cast<uint32_t>(P.kp) * 16;
            if (lane == 0) tc::bulk_g2s(sA, P.xt + st * P.a_bytes, P.a_bytes, &full[slot]);
            if (HG == 1) {
                // consecutive blocks are consecutive rows of a 16-column plane
                if (lane < 2)
                    tc::bulk_g2s(sB + lane * group_bytes, P.w[lane] + blk0 * run_bytes, nbh * run_bytes, &full[slot]);
            } else {
                for (int q = lane; q < nbh * 2 * HG; q += 32) {
                    const int b = q / (2 * HG), limb = (q / HG) % 2, h = q % HG;
                    tc::bulk_g2s(sB + (limb * HG + h) * group_bytes + b * run_bytes,
                                 P.w[limb] + ((blk0 + b) * HG + h) * static_cast<long long>(run_bytes), run_bytes,
                                 &full[slot]);
                }
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_i8(128, N, true, true);
            const uint32_t s0 = tc::smem_u32(smem);
            const uint32_t gb = static_cast<uint32_t>(P.kp) * 16;
            const int ksteps = P.kp / 32;
            long long i = 0;
            SlotRing ring(P.slots);
            bool ok = true;
            for (long long c = 0; c < n_chunks && ok; ++c) {
                const int buf = static_cast<int>(c & 1);
                const uint32_t aph = static_cast<uint32_t>((c >> 1) & 1);
                if (!tc::mbar_wait(&accempty[buf], aph ^ 1u, abort, P.err, tc::ERR_WAIT_ACCUM_FREE, P.wait_limit)) break;
                tc::tc_fence_after();
                const uint32_t dcol = tmem + static_cast<uint32_t>(buf * N);
                const long long i_end = min(n_my, (c + 1) * P.drain);
                for (bool first = true; i < i_end; ++i, first = false, ring.next()) {
                    const int slot = ring.slot;
                    const uint32_t ph = ring.phase;
                    if (!tc::mbar_wait(&full[slot], ph, abort, P.err, tc::ERR_WAIT_FULL, P.wait_limit)) {
                        ok = false;
                        break;
                    }
                    tc::tc_fence_after();
                    const uint32_t a0 = s0 + static_cast<uint32_t>(slot) * P.slot_bytes;
                    const uint32_t b0 = a0 + P.a_bytes;
                    for (int ks = 0; ks < ksteps; ++ks)
                        tc::mma_i8(dcol, tc::smem_desc(a0 + ks * 512u, 128u, gb), tc::smem_desc(b0 + ks * 512u, 128u, gb),
                                   idesc, (!first || ks > 0) ? 1u : 0u);
                    tc::mma_commit(&empty[slot]);
                }
                if (!ok) break;
                tc::mma_commit(&accfull[buf]);
            }
            tc::mma_commit(drained);
            tc::mbar_wait(drained, 0, nullptr, P.err, tc::ERR_WAIT_FINAL);
        }
        __syncwarp();
    } else {
        // ------------------------------------------------------------ epilogue
        const int q = warp & 3;                  // TMEM lane quadrant of this warp
        const int row = q * 32 + lane;           // D row
        const bool active = q < P.mg;            // rows below 32 * MG carry the X limbs
        int32_t acc[N];
#pragma unroll
        for (int c = 0; c < N; ++c) acc[c] = 0;
        for (long long c = 0; c < n_chunks; ++c) {
            const int buf = static_cast<int>(c & 1);
            const uint32_t aph = static_cast<uint32_t>((c >> 1) & 1);
            if (!tc::mbar_wait(&accfull[buf], aph, abort, P.err, tc::ERR_WAIT_ACCUM, P.wait_limit)) break;
            tc::tc_fence_after();
            if (active) {
                const uint32_t col0 = tmem + (static_cast<uint32_t>(q * 32) << 16) + static_cast<uint32_t>(buf * N);
#pragma unroll
                for (int c0 = 0; c0 < N; c0 += 16) {
                    int32_t v[16];
                    tc::tmem_ld16(col0 + c0, v);
                    tc::tmem_ld_wait();
#pragma unroll
                    for (int cc = 0; cc < 16; ++cc) acc[c0 + cc] = reduce_balanced(acc[c0 + cc] + reduce_partial(v[cc], P.mod), P.mod);
                }
            }
            tc::tc_fence_before();
            tc::mbar_arrive(&accempty[buf]);
        }
        if (active)
#pragma unroll
            for (int c = 0; c < N; ++c) red[row * N + c] = acc[c];
    }

    tc::tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, tmem_cols);
    }
    // x * w = lo*lo + 255 (lo*hi + hi*lo) + 255^2 hi*hi, per (x, j); the
    // CTA's balanced sums meet in one int32 accumulator by atomics (148 CTAs x
    // (p-1)/2 stay far below 2^31: exact and order-independent), which the
    // last CTA reads and clears
    const int entries = P.m * NB;
    const int hi_row = 16 * P.mg;
    for (int e = threadIdx.x; e < entries; e += blockDim.x) {
        const int x = e / NB, j = e - (e / NB) * NB;
        const int32_t ll = red[x * N + j], lh = red[x * N + NB + j];
        const int32_t hl = red[(hi_row + x) * N + j], hh = red[(hi_row + x) * N + NB + j];
        atomicAdd(P.partials + e, combine(ll, lh + hl, hh, P.mod, P.c1, P.c2));
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) am_last = (atomicAdd(P.counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    const unsigned long long pos = *reinterpret_cast<volatile unsigned long long*>(P.seq_index);
    for (int e = threadIdx.x; e < entries; e += blockDim.x) {
        const int x = e / NB, j = e - (e / NB) * NB;
        const int32_t sum = atomicExch(P.partials + e, 0);
        if (j >= P.n_out) continue;
        P.seq[pos * (static_cast<unsigned long long>(P.m) * P.n_out) + x * P.n_out + j] =
            to_canonical(reduce_balanced(sum, P.mod), P.mod);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        *P.seq_index = pos + 1;
        *P.counter = 0;
        __threadfence();
    }
}

// X (canonical, rows x m) -> the projection's A tiles [stage][2 MG][KP][16]:
// group g < MG holds the lo limbs of columns 16 g .. 16 g + 15, group MG + g
// their hi limbs; rows past the stage's SB * dim, past the last row or columns
// past m are zero.
__global__ void x_tiles_kernel(const uint32_t* __restrict__ X, int8_t* __restrict__ xt, long long rows, int m,
                               int mg, int dim, int sb, int kp, long long n_units, Mod mod) {
    for (long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; q < n_units;
         q += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long per_stage = 2LL * mg * kp;
        const long long st = q / per_stage;
        const int rem = static_cast<int>(q - st * per_stage);
        const int g = rem / kp, kr = rem - (rem / kp) * kp;
        const long long row = st * sb * dim + kr;
        const bool valid = kr < sb * dim && row < rows;
        const int limb = g / mg, x0 = (g % mg) * 16;
        uint32_t packed[4] = {0, 0, 0, 0};
#pragma unroll
        for (int xi = 0; xi < 16; ++xi) {
            const int x = x0 + xi;
            int8_t lo = 0, hi = 0;
            if (valid && x < m) split_limbs(to_balanced(X[row * m + x] % static_cast<uint32_t>(mod.p), mod), lo, hi);
            packed[xi / 4] |= static_cast<uint32_t>(static_cast<uint8_t>(limb ? hi : lo)) << (8 * (xi % 4));
        }
        *reinterpret_cast<uint4*>(xt + q * 16) = make_uint4(packed[0], packed[1], packed[2], packed[3]);
    }
}

template <class F>
void dispatch_i8_nb(int nb, F&& f) {
    switch (nb) {
        case 16: f(std::integral_constant<int, 16>{}); break;
        case 32: f(std::integral_constant<int, 32>{}); break;
        default: throw Error("INT8 form supports block widths 16 and 32", 1);
    }
}

}  // namespace

// Host-side state of the INT8 form.
struct KoszulCtx::I8State {
    struct Dir {
        I8Dir p{};
        int8_t* b_tiles = nullptr;
        uint32_t* inc = nullptr;
        int4* rows4 = nullptr;     // TMA gather rows per group of four generators
        bool gather4 = false;      // hybrid producer (TMA gathers beside cp.async warps), else cp.async only
        int pw = 8;                // cp.async producer warps (8 or 16)
        size_t smem = 0;
        unsigned grid = 0;
    } fwd, bwd;
    // Y_a, Y_b, Z: lo, hi, -lo, -hi; each -plane directly follows its +plane in
    // memory, so that one tensor map covers both signs of a limb
    int8_t* planes[3][4] = {};
    CUtensorMap maps[3][2];        // [block array][limb]: rows = (sign, block, h) runs
    std::string plan_text;         // the chosen stage plans and the autotuner's timings
    I8Proj proj{};             // projection plan (X tiles, stage shape, grid)
    int8_t* xt = nullptr;
    size_t proj_smem = 0;
    unsigned proj_grid = 0;
    int* err = nullptr;
};

namespace {

// Autotuner cache: the chosen producer and stage size per operator shape and
// device, shared by every context of the process.
struct TuneKey {
    int r, k, inner, outer, nbi, dir, sms, allowed;
    bool operator<(const TuneKey& o) const {
        return std::tie(r, k, inner, outer, nbi, dir, sms, allowed) <
               std::tie(o.r, o.k, o.inner, o.outer, o.nbi, o.dir, o.sms, o.allowed);
    }
};
struct TuneChoice {
    bool gather4 = false;   // the hybrid producer
    int pw = 8;             // cp.async producer warps
    int gps = 0;            // generators per stage
    int t_tma = 0;          // hybrid: blocks of a tile gathered by TMA
    double ms = 0;
};
std::mutex g_tune_mutex;
std::map<TuneKey, TuneChoice> g_tune_cache;

bool tune_lookup(const TuneKey& k, TuneChoice& out) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    const auto it = g_tune_cache.find(k);
    if (it == g_tune_cache.end()) return false;
    out = it->second;
    return true;
}

void tune_store(const TuneKey& k, const TuneChoice& c) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune_cache[k] = c;
}

// Plans one direction: stage size, pipeline depth, B operand (host layout).
//
// A generator spans `inner_pad` K' rows (inner, rounded up to even for the TMA
// gather producer so that every group of four generators starts 128-byte
// aligned).  A stage holds `gps` generators (gather producer: gs groups of
// four), padded to whole K-steps of 32 rows; B is zero in every padding row
// and for every generator past r, so the A rows there may hold anything.
// Returns false when the maps and stages do not fit in shared memory.
bool plan_direction(KoszulCtx& c, KoszulCtx::I8State::Dir& D, int inner, int outer, bool transpose_maps,
                    bool gather4, int gps_forced = 0) {
    I8Dir& P = D.p;
    P.r = c.r;
    P.inner = inner;
    P.outer = outer;
    P.half = (outer + 15) / 16 * 16;
    const int N = 2 * P.half;
    BW_REQUIRE(N <= 256, "INT8 form: output dimension above 128 is not supported");
    const size_t extra = (2 * 8 + 2 * 2 + 1) * 8 + 16 + kMaxRowTable;
    const int inner_pad = gather4 ? inner + (inner & 1) : inner;
    auto b_bytes_of = [&](int gps) {
        const int stages = (c.r + gps - 1) / gps;
        const int ks_full = (gps * inner_pad + 31) / 32;
        const int last = c.r - (stages - 1) * gps;
        const int last_rows = gather4 ? (last + 3) / 4 * 4 * inner_pad : last * inner_pad;
        return static_cast<size_t>((stages - 1) * ks_full + (last_rows + 31) / 32) * N * 32;
    };
    int gps = 0;
    if (gps_forced > 0) {
        // a stage size chosen by the autotuner (checked below against shared memory)
        if (gather4 && gps_forced % 4 != 0) return false;
        gps = std::min(gps_forced, gather4 ? (c.r + 3) / 4 * 4 : c.r);
        if (gather4) {
            P.groups = (c.r + 3) / 4;
            P.gs = gps / 4;
        } else if (gps * inner > kMaxRowTable) {
            return false;
        }
    } else if (gather4) {
        // groups of four generators per stage: the best-filled choice that
        // leaves at least three pipeline slots, the fewer stages on ties
        P.groups = (c.r + 3) / 4;
        double best = -1;
        for (int gs = 1; gs <= P.groups; ++gs) {
            const int rows = gs * 4 * inner_pad, padded = (rows + 31) / 32 * 32;
            const size_t slot = static_cast<size_t>(2) * 8 * padded * 16;
            const size_t bb = b_bytes_of(4 * gs);
            if (bb + 3 * slot + extra > static_cast<size_t>(kMaxSmem)) break;
            const double fill = static_cast<double>(rows) / padded;
            if (fill > best + 1e-9) {
                best = fill;
                gps = 4 * gs;
            }
        }
        if (gps == 0) return false;
        P.gs = gps / 4;
    } else {
        // the best-filled stage of at most 56 KB of A per slot, the largest such on ties
        double best_fill = -1;
        for (int g = 1; g <= c.r; ++g) {
            const int rows = g * inner, padded = (rows + 31) / 32 * 32;
            if (g > 1 && static_cast<size_t>(2) * 8 * padded * 16 > 56 * 1024) break;
            const double fill = static_cast<double>(rows) / padded;
            if (fill > best_fill - 1e-9) {
                best_fill = std::max(best_fill, fill);
                gps = g;
            }
        }
        BW_REQUIRE(gps * inner <= kMaxRowTable, "INT8 form: stage too deep for the row table");
    }
    P.inner_pad = inner_pad;
    P.gi = gps;
    P.stages_per_tile = (c.r + gps - 1) / gps;
    P.ks_full = (gps * inner_pad + 31) / 32;
    const int last_g = c.r - (P.stages_per_tile - 1) * gps;
    const int last_rows = gather4 ? (last_g + 3) / 4 * 4 * inner_pad : last_g * inner_pad;
    P.ks_last = (last_rows + 31) / 32;
    const int total_ks = (P.stages_per_tile - 1) * P.ks_full + P.ks_last;
    P.b_bytes = static_cast<uint32_t>(total_ks) * N * 32;
    P.limb_bytes = static_cast<uint32_t>(8 * P.ks_full * 32 * 16);
    P.slot_bytes = 2 * P.limb_bytes;
    P.tx_full = static_cast<uint32_t>(16 * gps * inner_pad * 16);              // 2 limbs x 8 columns x rows x 16 B
    P.tx_last = static_cast<uint32_t>(16 * ((last_g + 3) / 4 * 4) * inner_pad * 16);
    int slots = 8;
    while (slots > 1 && P.b_bytes + static_cast<size_t>(slots) * P.slot_bytes + extra > static_cast<size_t>(kMaxSmem))
        --slots;
    if (P.b_bytes + static_cast<size_t>(slots) * P.slot_bytes + extra > static_cast<size_t>(kMaxSmem)) return false;
    if (gather4 && P.ks_full * 32 > kMaxRowTable) return false;
    P.slots = slots;
    D.smem = P.b_bytes + static_cast<size_t>(slots) * P.slot_bytes + extra;
    D.gather4 = gather4;
    P.mod = c.mod;
    P.c1 = to_balanced(255u % c.p, c.mod);
    P.c2 = to_balanced(static_cast<uint32_t>((255ull * 255ull) % c.p), c.mod);

    // B: row n < half -> lo limb, n >= half -> hi limb of map coefficient (o = n mod half),
    // column K' = stage row base + (generator in stage) * inner_pad + u; K-major,
    // 8x16-byte core matrices, LBO 128, SBO 256.
    std::vector<int8_t> B(P.b_bytes, 0);
    const int kp_total = total_ks * 32;
    for (int kp = 0; kp < kp_total; ++kp) {
        const int s = std::min(kp / (P.ks_full * 32), P.stages_per_tile - 1);
        const int local = kp - s * P.ks_full * 32;
        const int gen_local = local / inner_pad, u = local % inner_pad;
        const int i = s * gps + gen_local;
        if (u >= inner || gen_local >= (s == P.stages_per_tile - 1 ? last_g : gps) || i >= c.r) continue;   // padding
        for (int n = 0; n < N; ++n) {
            const int o = n % P.half;
            if (o >= outer) continue;
            // forward: coefficient M_i[o = c][u = b]; transpose: M_i[u = c][o = b]
            const uint32_t raw = transpose_maps
                                     ? c.maps_canonical[(static_cast<size_t>(i) * c.co + u) * c.ci + o]
                                     : c.maps_canonical[(static_cast<size_t>(i) * c.co + o) * c.ci + u];
            int8_t lo, hi;
            split_limbs(to_balanced(raw % c.p, c.mod), lo, hi);
            const int ks = kp / 32, kk = kp % 32;
            const size_t off = static_cast<size_t>(ks) * N * 32 + (n / 8) * 256 + (kk / 16) * 128 + (n % 8) * 16 + (kk % 16);
            B[off] = n < P.half ? lo : hi;
        }
    }
    D.b_tiles = c.alloc<int8_t>(P.b_bytes);
    BW_CUDA(cudaMemcpyAsync(D.b_tiles, B.data(), B.size(), cudaMemcpyHostToDevice, c.own_stream));
    BW_CUDA(cudaStreamSynchronize(c.own_stream));
    P.b_tiles = D.b_tiles;
    return true;
}

// Rows of the TMA gathers: for output block blk and group g (generators
// 4g..4g+3), the plane row of each generator's neighbour run at h = 0:
// neg * n_blk_in * HG + nbr * HG, or one past the last row (zero-filled) for an
// absent generator or one past r.
std::vector<int4> gather_rows(const std::vector<uint32_t>& inc, uint64_t n_blk, int r, uint64_t n_blk_in, int hg) {
    const int groups = (r + 3) / 4;
    const int64_t oob = static_cast<int64_t>(2 * n_blk_in * hg);
    BW_REQUIRE(oob + hg < (1ll << 31), "INT8 form: plane rows above the TMA coordinate range");
    std::vector<int4> out(n_blk * groups);
    for (uint64_t b = 0; b < n_blk; ++b)
        for (int g = 0; g < groups; ++g) {
            int32_t v[4];
            for (int q = 0; q < 4; ++q) {
                const int i = 4 * g + q;
                const uint32_t e = i < r ? inc[b * r + i] : kAbsent;
                v[q] = static_cast<int32_t>(e == kAbsent ? oob
                                                         : static_cast<int64_t>(e >> 31) * n_blk_in * hg +
                                                               static_cast<int64_t>(e & 0x7FFFFFFFu) * hg);
            }
            out[b * groups + g] = make_int4(v[0], v[1], v[2], v[3]);
        }
    return out;
}

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// One limb of a block array as a 2-D tensor for the gathers: rows = the
// (sign, block, h) runs of dim * 16 bytes (the -plane's rows after the
// +plane's), 8-byte elements; box = one run of dim_pad * 16 bytes.
void encode_plane_map(CUtensorMap* map, const int8_t* base, uint64_t n_blk, int dim, int dim_pad, int hg) {
    static const EncodeTiledFn encode = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<EncodeTiledFn>(f);
    }();
    BW_REQUIRE(encode != nullptr, "INT8 form: cuTensorMapEncodeTiled is not available from the driver");
    BW_REQUIRE(reinterpret_cast<uintptr_t>(base) % 16 == 0, "INT8 form: plane not 16-byte aligned");
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(2 * dim), static_cast<cuuint64_t>(2 * n_blk * hg)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(dim) * 16};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(2 * dim_pad), 1};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult rc = encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, const_cast<int8_t*>(base), dims, strides, box,
                               estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    BW_REQUIRE(rc == CUDA_SUCCESS, "INT8 form: cuTensorMapEncodeTiled failed (code " + std::to_string(rc) + ")");
}

// Projection stage shape: SB whole source blocks per stage, KP = SB * dim
// rounded up to 32, about kProjStageTarget bytes of X tile and W runs, the
// least padding first.  Allocates the X tiles.
void plan_projection(KoszulCtx& c, KoszulCtx::I8State& S) {
    I8Proj& P = S.proj;
    BW_REQUIRE(c.m >= 1 && c.m <= 64, "INT8 form: projection width must be 1..64");
    P.m = c.m;
    P.n_out = c.nb;
    P.mg = (c.m + 15) / 16;
    P.dim = c.ci;
    P.n_blk = static_cast<long long>(c.n_s);
    const int row_bytes = (2 * P.mg + 2 * (c.nbi / 16)) * 16;
    int best_sb = 1;
    double best_fill = 0;
    for (int sb = 1; sb <= 4096; ++sb) {
        const int kp = (sb * P.dim + 31) / 32 * 32;
        if (sb > 1 && kp * row_bytes > kProjStageTarget) break;
        const double fill = static_cast<double>(sb * P.dim) / kp;
        if (fill >= best_fill) {
            best_fill = fill;
            best_sb = sb;
        }
    }
    P.sb = best_sb;
    P.kp = (best_sb * P.dim + 31) / 32 * 32;
    P.n_stages = static_cast<int>((P.n_blk + P.sb - 1) / P.sb);
    P.drain = std::max(1, 131072 / P.kp);
    const uint32_t group_bytes = static_cast<uint32_t>(P.kp) * 16;
    P.a_bytes = 2 * P.mg * group_bytes;
    P.slot_bytes = P.a_bytes + 2 * (c.nbi / 16) * group_bytes;
    // the M = 128 A descriptor spans 8 groups from the tile start
    const uint32_t reach = 8 * group_bytes;
    P.pad_bytes = reach > P.slot_bytes ? reach - P.slot_bytes : 0;
    const size_t extra = static_cast<size_t>(32) * P.mg * 2 * c.nbi * 4 + (2 * 8 + 2 * 2 + 1) * 8 + 16;
    const size_t limit = static_cast<size_t>(kMaxSmem) - 1024;   // headroom for the kernel's static flag
    int slots = 4;
    while (slots > 2 && static_cast<size_t>(slots) * P.slot_bytes + P.pad_bytes + extra > limit) --slots;
    BW_REQUIRE(static_cast<size_t>(slots) * P.slot_bytes + P.pad_bytes + extra <= limit,
               "INT8 form: projection stage does not fit in shared memory");
    P.slots = slots;
    S.proj_smem = static_cast<size_t>(slots) * P.slot_bytes + P.pad_bytes + extra;
    P.mod = c.mod;
    P.c1 = to_balanced(255u % c.p, c.mod);
    P.c2 = to_balanced(static_cast<uint32_t>((255ull * 255ull) % c.p), c.mod);
    P.err = S.err;
    S.proj_grid = static_cast<unsigned>(std::max(1, std::min(P.n_stages, c.sms)));
    BW_REQUIRE(S.proj_grid <= std::max<unsigned>(c.proj_grid, static_cast<unsigned>(c.sms)),
               "INT8 form: projection grid above the partials buffer");
    S.xt = c.alloc<int8_t>(static_cast<uint64_t>(P.n_stages) * P.a_bytes);
    P.xt = S.xt;
}

template <int NB>
void launch_i8(KoszulCtx& c, KoszulCtx::I8State::Dir& D, const CUtensorMap* maps, cudaStream_t st) {
    BW_REQUIRE(D.p.inc != nullptr && (!D.gather4 || D.p.rows4 != nullptr) && D.p.b_tiles != nullptr,
               "internal: INT8 gather tables missing for the chosen producer");
    if (D.gather4)
        i8_gather_hybrid_kernel<NB><<<D.grid, kHyThreads, D.smem, st>>>(maps[0], maps[1], D.p);
    else if (D.pw == 16)
        i8_gather_gemm_kernel<NB, 16><<<D.grid, GatherWarps<16>::threads, D.smem, st>>>(D.p);
    else
        i8_gather_gemm_kernel<NB, 8><<<D.grid, GatherWarps<8>::threads, D.smem, st>>>(D.p);
    BW_CHECK_LAUNCH();
    ++c.launches;
}

}  // namespace

void KoszulCtx::i8_destroy() {
    delete i8;
    i8 = nullptr;
}

void KoszulCtx::i8_setup() {
    BW_REQUIRE(nbi == 16 || nbi == 32, "INT8 form: internal block width must be 16 or 32");
    // two double-buffered accumulators of 2 N <= 256 columns each fill the 512 TMEM columns
    BW_REQUIRE(ci <= 64 && co <= 64, "INT8 form: dim_in and dim_out must be at most 64");
    BW_REQUIRE(static_cast<long long>(r) * std::max(ci, co) <= 1024, "INT8 form: r * dim above 1024 (int32 bound)");
    BW_REQUIRE(r <= 32, "INT8 form: at most 32 generators (one per lane)");
    int major = 0;
    BW_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
    BW_REQUIRE(major == 10, "INT8 form needs an sm_100 GPU (tcgen05)");
    i8 = new I8State();
    I8State& S = *i8;
    // dense incidence tables: fwd[T][i] (S = T u i), bwd[S][i] (T = S \ i)
    std::vector<uint32_t> fwd(n_t * r, kAbsent), bwd(n_s * r, kAbsent);
    int T[64], Sx[64];
    for (uint64_t t = 0; t < n_t; ++t) {
        lex_unrank(t, r, k - 1, T);
        int pos = 0;
        for (int i = 0; i < r; ++i) {
            if (pos < k - 1 && T[pos] == i) {
                ++pos;
                continue;
            }
            for (int qq = 0, w = 0; qq < k; ++qq) Sx[qq] = (qq == pos) ? i : T[w++];
            fwd[t * r + i] = static_cast<uint32_t>(lex_rank(Sx, r, k)) | ((pos & 1) ? 0x80000000u : 0u);
        }
    }
    for (uint64_t s = 0; s < n_s; ++s) {
        lex_unrank(s, r, k, Sx);
        for (int pos = 0; pos < k; ++pos) {
            for (int qq = 0, w = 0; qq < k; ++qq)
                if (qq != pos) T[w++] = Sx[qq];
            bwd[s * r + Sx[pos]] = static_cast<uint32_t>(lex_rank(T, r, k - 1)) | ((pos & 1) ? 0x80000000u : 0u);
        }
    }
    // each limb's -plane directly after its +plane (one tensor map covers both signs)
    for (int b = 0; b < 3; ++b) {
        const uint64_t plane = (b < 2 ? n_src : n_tgt) * nbi;
        // the gather producers address a +plane and its -plane in 16-byte units below 2^32 - 1
        BW_REQUIRE(2 * plane / 16 < 0xFFFFFFFFull, "INT8 form: limb planes above the 16-byte offset range");
        for (int limb = 0; limb < 2; ++limb) {
            int8_t* pair = alloc<int8_t>(2 * plane);
            S.planes[b][limb] = pair;
            S.planes[b][limb + 2] = pair + plane;
        }
    }
    S.err = alloc<int>(1);
    BW_CUDA(cudaMemsetAsync(S.err, 0, sizeof(int), own_stream));
    plan_projection(*this, S);
    const int hg = nbi / 16;
    // Both gather tables (TMA rows per group of four generators, and the
    // per-generator words of the cp.async producer) until the plans are chosen.
    auto upload_rows = [&](const std::vector<uint32_t>& inc, uint64_t n_out, uint64_t n_in) {
        const std::vector<int4> rows = gather_rows(inc, n_out, r, n_in, hg);
        int4* d = alloc<int4>(rows.size());
        BW_CUDA(cudaMemcpyAsync(d, rows.data(), rows.size() * sizeof(int4), cudaMemcpyHostToDevice, own_stream));
        BW_CUDA(cudaStreamSynchronize(own_stream));
        return d;
    };
    auto upload_inc = [&](const std::vector<uint32_t>& inc) {
        uint32_t* d = alloc<uint32_t>(inc.size());
        BW_CUDA(cudaMemcpyAsync(d, inc.data(), inc.size() * 4, cudaMemcpyHostToDevice, own_stream));
        BW_CUDA(cudaStreamSynchronize(own_stream));
        return d;
    };
    S.fwd.rows4 = upload_rows(fwd, n_t, n_s);
    S.bwd.rows4 = upload_rows(bwd, n_s, n_t);
    S.fwd.inc = upload_inc(fwd);
    S.bwd.inc = upload_inc(bwd);
    for (int b = 0; b < 3; ++b) {
        const uint64_t n_blk = b < 2 ? n_s : n_t;
        const int dim = b < 2 ? ci : co;
        for (int limb = 0; limb < 2; ++limb)
            encode_plane_map(&S.maps[b][limb], S.planes[b][limb], n_blk, dim, dim + (dim & 1), hg);
    }
    // Failure tests only (the environment of the creating process): a short
    // limit on every pipeline wait, and a first stage that CTA 0 of the d/d^T
    // kernel never fills, so that its consumer's wait runs out and the kernel
    // gives up, frees its TMEM and returns; the host then reports status 2.
    // (The hold starts after the set-up's own timing launches.)
    uint32_t wait_limit = tc::kWaitLimit;
    if (const char* e = std::getenv("BW_TEST_WAIT_LIMIT")) {
        const unsigned long v = std::strtoul(e, nullptr, 10);
        if (v >= 1 && v < tc::kWaitLimit) wait_limit = static_cast<uint32_t>(v);
    }
    int hold = 0;
    if (const char* e = std::getenv("BW_TEST_HOLD_FIRST_STAGE")) hold = (*e && std::string(e) != "0") ? 1 : 0;
    S.proj.wait_limit = wait_limit;
    int cap_g = 0, cap_4 = 0;
    dispatch_i8_nb(nbi, [&](auto NBc) {
        cap_g = std::min(allow_dynamic_smem(i8_gather_gemm_kernel<decltype(NBc)::value, 8>, device),
                         allow_dynamic_smem(i8_gather_gemm_kernel<decltype(NBc)::value, 16>, device));
        cap_4 = allow_dynamic_smem(i8_gather_hybrid_kernel<decltype(NBc)::value>, device);
        const int cap_p = allow_dynamic_smem(i8_project_tc_kernel<decltype(NBc)::value>, device);
        BW_REQUIRE(static_cast<int>(S.proj_smem) <= cap_p, "INT8 form: shared-memory plan above the device limit");
    });
    const int bt = 128 / nbi;
    S.fwd.p.n_blk = static_cast<long long>(n_t);
    S.bwd.p.n_blk = static_cast<long long>(n_s);
    S.fwd.p.row_oob = static_cast<int32_t>(2 * n_s * hg);   // the forward gathers Y (source blocks)
    S.bwd.p.row_oob = static_cast<int32_t>(2 * n_t * hg);   // d^T gathers Z (target blocks)
    S.fwd.grid = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>((n_t + bt - 1) / bt, sms)));
    S.bwd.grid = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>((n_s + bt - 1) / bt, sms)));

    // Stage plans.  Each direction's producer (TMA gathers or cp.async warps)
    // and stage size are chosen by timing every candidate that fits in shared
    // memory on this device, at set-up, on the context's own buffers (the
    // kernels' work does not depend on the values); the choice is cached per
    // shape for the life of the process.  BW_I8_TUNE=0 takes the fill
    // heuristic instead; BW_I8_PRODUCER=cpasync or =hybrid restricts the
    // producer.
    bool allow_g4 = true, allow_cp = true, tune = true;
    if (const char* e = std::getenv("BW_I8_PRODUCER")) {
        allow_g4 = std::string(e) != "cpasync";
        allow_cp = std::string(e) != "hybrid";
    }
    if (const char* e = std::getenv("BW_I8_TUNE")) tune = std::string(e) != "0";
    // BW_I8_PRODUCER_WARPS=8 or =16 restricts the cp.async producer's warp count
    std::vector<int> pws{8, 16};
    if (const char* e = std::getenv("BW_I8_PRODUCER_WARPS")) {
        const int v = std::atoi(e);
        if (v == 8 || v == 16) pws = {v};
    }
    std::string text;
    for (int dir = 0; dir < 2; ++dir) {
        I8State::Dir& D = dir == 0 ? S.fwd : S.bwd;
        const int inner = dir == 0 ? ci : co, outer = dir == 0 ? co : ci;
        const int in_buf = dir == 0 ? I8_YA : I8_Z, out_buf = dir == 0 ? I8_Z : I8_YB;
        auto plan = [&](bool g4, int gps, int t_tma, int pw) {
            if (D.b_tiles) release(D.b_tiles);
            D.b_tiles = nullptr;
            if (!plan_direction(*this, D, inner, outer, dir == 1, g4, gps)) return false;
            if (static_cast<int>(D.smem) > (g4 ? cap_4 : cap_g)) return false;
            D.pw = g4 ? 8 : pw;
            D.p.t_tma = g4 ? t_tma : 0;
            D.p.err = S.err;
            D.p.wait_limit = wait_limit;
            D.p.hold_first_stage = 0;
            D.p.inc = D.inc;
            D.p.rows4 = D.rows4;
            return true;
        };
        const TuneKey key{r, k, inner, outer, nbi, dir, sms,
                          (allow_g4 ? 1 : 0) | (allow_cp ? 2 : 0) | (pws.size() == 1 ? pws[0] * 4 : 0)};
        TuneChoice choice{};
        bool have = tune && tune_lookup(key, choice);
        std::string tried;
        if (!have && tune) {
            // candidates: the cp.async producer with its heuristic stage; the
            // hybrid producer with 1..3 groups of four generators a stage and a
            // quarter, half or three quarters of a tile's blocks gathered by TMA
            struct Cand {
                bool g4;
                int gps, t_tma, pw;
            };
            std::vector<Cand> cands;
            if (allow_cp) {
                // the fill heuristic's stage, and fewer or more generators a stage
                // (smaller stages leave room for more pipeline slots), each with 8
                // and with 16 producer warps
                for (int pw : pws) {
                    cands.push_back({false, 0, 0, pw});
                    for (int g : {4, 6, 8, 12})
                        if (g < r) cands.push_back({false, g, 0, pw});
                }
            }
            if (allow_g4)
                for (int gs = 1; gs <= std::min(3, (r + 3) / 4); ++gs)
                    for (int qt = 1; qt <= 3; ++qt) cands.push_back({true, 4 * gs, qt * bt / 4, 8});
            double best = 1e30;
            for (const Cand& cand : cands) {
                if (!plan(cand.g4, cand.gps, cand.t_tma, cand.pw)) continue;
                const double ms = i8_time_direction(dir == 0, in_buf, out_buf);
                char buf[96];
                if (cand.g4)
                    std::snprintf(buf, sizeof buf, "%shybrid stage=%d tma=%d/%d: %.4f ms", tried.empty() ? "" : ", ",
                                  D.p.gi, cand.t_tma, bt, ms);
                else
                    std::snprintf(buf, sizeof buf, "%scp.async stage=%d warps=%d: %.4f ms", tried.empty() ? "" : ", ",
                                  D.p.gi, cand.pw, ms);
                tried += buf;
                if (ms < best) {
                    best = ms;
                    choice = TuneChoice{cand.g4, cand.pw, D.p.gi, cand.t_tma, ms};
                }
            }
            BW_REQUIRE(best < 1e30, "INT8 form: no stage plan fits in shared memory");
            tune_store(key, choice);
            have = true;
        }
        bool ok = false;
        if (have) ok = plan(choice.gather4, choice.gps, choice.t_tma, choice.pw);
        if (!ok) ok = (allow_cp && plan(false, 0, 0, pws[0])) || (allow_g4 && plan(true, 0, bt / 2, 8));
        BW_REQUIRE(ok, "INT8 form: maps too large for shared memory");
        char buf[192];
        if (D.gather4)
            std::snprintf(buf, sizeof buf, "%s: hybrid (TMA gathers for %d of %d blocks) stage=%d generators, %d slots, "
                          "%zu B shared", dir == 0 ? "d" : "d^T", D.p.t_tma, bt, D.p.gi, D.p.slots, D.smem);
        else
            std::snprintf(buf, sizeof buf, "%s: cp.async stage=%d generators, %d producer warps, %d slots, %zu B shared",
                          dir == 0 ? "d" : "d^T", D.p.gi, D.pw, D.p.slots, D.smem);
        text += (text.empty() ? "" : "; ") + std::string(buf);
        if (!tried.empty()) text += " (tuned: " + tried + ")";
    }
    // the TMA rows are freed when the cp.async producer alone was chosen (the
    // hybrid producer reads both tables)
    for (I8State::Dir* D : {&S.fwd, &S.bwd}) {
        if (!D->gather4) {
            release(D->rows4);
            D->rows4 = nullptr;
        }
        D->p.inc = D->inc;
        D->p.rows4 = D->rows4;
        D->p.hold_first_stage = hold;
    }
    char pbuf[160];
    std::snprintf(pbuf, sizeof pbuf, "; projection: %d blocks a stage (%d rows), %d slots", S.proj.sb, S.proj.kp,
                  S.proj.slots);
    S.plan_text = text + pbuf;
    BW_CUDA(cudaStreamSynchronize(own_stream));
}

const std::string& KoszulCtx::i8_plan_text() const { return i8->plan_text; }

// Device time of one direction's gather-GEMM on the context's buffers: one
// warm-up launch, then the mean of three (CUDA events on the own stream).
double KoszulCtx::i8_time_direction(bool forward_dir, int in_buf, int out_buf) {
    cudaEvent_t e0, e1;
    BW_CUDA(cudaEventCreate(&e0));
    BW_CUDA(cudaEventCreate(&e1));
    i8_run(forward_dir, in_buf, out_buf, !forward_dir, own_stream);
    BW_CUDA(cudaEventRecord(e0, own_stream));
    for (int i = 0; i < 3; ++i) i8_run(forward_dir, in_buf, out_buf, !forward_dir, own_stream);
    BW_CUDA(cudaEventRecord(e1, own_stream));
    BW_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    BW_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    i8_check_error();
    return ms / 3.0;
}

uint64_t KoszulCtx::i8_kernels_per_step() const { return 3; }

void KoszulCtx::i8_run(bool forward_dir, int in_buf, int out_buf, bool scale, cudaStream_t st) {
    I8State::Dir& D = forward_dir ? i8->fwd : i8->bwd;
    for (int pl = 0; pl < 4; ++pl) {
        D.p.in[pl] = i8->planes[in_buf][pl];
        D.p.out[pl] = i8->planes[out_buf][pl];
    }
    D.p.in_neg_off = i8->planes[in_buf][PL_NLO] - i8->planes[in_buf][PL_LO];
    D.p.diag = (!forward_dir && scale) ? d_diag : nullptr;
    dispatch_i8_nb(nbi, [&](auto NBc) { launch_i8<decltype(NBc)::value>(*this, D, i8->maps[in_buf], st); });
}

void KoszulCtx::i8_check_error() {
    int err = 0;
    BW_CUDA(cudaMemcpy(&err, i8->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err != 0) {
        cudaMemset(i8->err, 0, sizeof(int));
        static const char* const names[] = {"", "ERR_WAIT_FULL: consumer waited for a loaded stage",
                                            "ERR_WAIT_EMPTY: producer waited for a free stage",
                                            "ERR_WAIT_ACCUM: epilogue waited for an accumulator",
                                            "ERR_WAIT_ACCUM_FREE: MMA waited for a free accumulator",
                                            "ERR_WAIT_FINAL: final drain of in-flight MMAs",
                                            "ERR_LAYOUT: shared-memory layout check failed"};
        const std::string what = (err >= 1 && err <= 6) ? names[err] : "code " + std::to_string(err);
        throw Error("INT8 tensor-core kernel gave up waiting (" + what + ")", 2);
    }
}

int KoszulCtx::i8_dim(int buf) const { return buf == I8_Z ? co : ci; }
uint64_t KoszulCtx::i8_rows(int buf) const { return buf == I8_Z ? n_tgt : n_src; }

void KoszulCtx::i8_to_limbs(const uint32_t* in, int buf, cudaStream_t st) {
    const uint64_t count = i8_rows(buf) * nbi;
    unsigned grid = static_cast<unsigned>(std::min<uint64_t>((count + 255) / 256, static_cast<uint64_t>(sms) * 8));
    int8_t** pl = i8->planes[buf];
    dispatch_i8_nb(nbi, [&](auto NBc) {
        to_limbs_kernel<decltype(NBc)::value><<<std::max(grid, 1u), 256, 0, st>>>(
            in, pl[0], pl[1], pl[2], pl[3], static_cast<long long>(count), i8_dim(buf), nb, mod);
    });
    BW_CHECK_LAUNCH();
    ++launches;
}

void KoszulCtx::i8_from_limbs(int buf, uint32_t* out, cudaStream_t st) {
    const uint64_t count = i8_rows(buf) * nb;
    unsigned grid = static_cast<unsigned>(std::min<uint64_t>((count + 255) / 256, static_cast<uint64_t>(sms) * 8));
    int8_t** pl = i8->planes[buf];
    dispatch_i8_nb(nbi, [&](auto NBc) {
        from_limbs_kernel<decltype(NBc)::value><<<std::max(grid, 1u), 256, 0, st>>>(
            pl[0], pl[1], out, static_cast<long long>(count), i8_dim(buf), nb, mod);
    });
    BW_CHECK_LAUNCH();
    ++launches;
}

void KoszulCtx::i8_load_x(const uint32_t* x, cudaStream_t st) {
    const I8Proj& P = i8->proj;
    const long long units = static_cast<long long>(P.n_stages) * 2 * P.mg * P.kp;
    unsigned grid = static_cast<unsigned>(std::min<long long>((units + 255) / 256, static_cast<long long>(sms) * 8));
    x_tiles_kernel<<<std::max(grid, 1u), 256, 0, st>>>(x, i8->xt, static_cast<long long>(n_src), m, P.mg, ci, P.sb,
                                                        P.kp, units, mod);
    BW_CHECK_LAUNCH();
    ++launches;
}

void KoszulCtx::i8_project(int buf, cudaStream_t st) {
    I8Proj P = i8->proj;
    P.w[0] = i8->planes[buf][0];
    P.w[1] = i8->planes[buf][1];
    P.partials = d_partials;
    P.counter = d_counter;
    P.seq = d_seq;
    P.seq_index = d_seq_index;
    dispatch_i8_nb(nbi, [&](auto NBc) {
        i8_project_tc_kernel<decltype(NBc)::value><<<i8->proj_grid, kProjThreads, i8->proj_smem, st>>>(P);
    });
    BW_CHECK_LAUNCH();
    ++launches;
}

// One INT8 step on the limb state: cur -> other, append a_i.
void KoszulCtx::i8_step_once(cudaStream_t st) {
    const int src = cur_is_a ? I8_YA : I8_YB, dst = cur_is_a ? I8_YB : I8_YA;
    i8_run(true, src, I8_Z, false, st);
    i8_run(false, I8_Z, dst, true, st);
    i8_project(dst, st);
    cur_is_a = !cur_is_a;
}

}  // namespace bw
