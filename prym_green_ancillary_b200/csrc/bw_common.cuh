// Shared helpers of the B200 block-Wiedemann engine: error plumbing, modular
// arithmetic on balanced residues, the counter-based seeded stream and the
// lexicographic subset ranking used by every Koszul table.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <stdexcept>
#include <string>

namespace bw {

// ------------------------------------------------------------------ errors

struct Error : std::runtime_error {
    int code;
    explicit Error(const std::string& msg, int c = 1) : std::runtime_error(msg), code(c) {}
};

void set_last_error(const std::string& msg);

// Largest dynamic shared memory a block may opt into on `device`.
int max_dynamic_smem(int device);

#define BW_CUDA(call)                                                              \
    do {                                                                           \
        cudaError_t bw_err_ = (call);                                              \
        if (bw_err_ != cudaSuccess)                                                \
            throw ::bw::Error(std::string(#call) + " failed: " +                   \
                              cudaGetErrorString(bw_err_) + " (" __FILE__ ":" +    \
                              std::to_string(__LINE__) + ")", 2);                  \
    } while (0)

#define BW_CHECK_LAUNCH() BW_CUDA(cudaGetLastError())

#define BW_REQUIRE(cond, msg)                                                      \
    do {                                                                           \
        if (!(cond)) throw ::bw::Error(msg, 3);                                    \
    } while (0)

// An argument the caller passed outside what the entry point accepts (a null
// pointer, a size or value beyond its documented range): status 1.
#define BW_ARG(cond, msg)                                                          \
    do {                                                                           \
        if (!(cond)) throw ::bw::Error(msg, 1);                                    \
    } while (0)

// Kernels that use dynamic shared memory get the largest limit the device
// allows them (the opt-in maximum less their static shared memory): the
// per-function limit is process-wide, so setting one context's own size could
// lower it under another context's launches of the same kernel.  Returns it.
template <class Kernel>
int allow_dynamic_smem(Kernel kernel, int device) {
    cudaFuncAttributes a{};
    BW_CUDA(cudaFuncGetAttributes(&a, kernel));
    const int cap = max_dynamic_smem(device) - static_cast<int>(a.sharedSizeBytes);
    BW_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, cap));
    return cap;
}

// Every C-ABI entry point runs its body through this wrapper: exceptions never
// cross the ABI; the message goes to the thread-local last-error slot.
template <class F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return 1;
    }
}

// --------------------------------------------------------------- residues
//
// Inside the engine a residue x of GF(p) (p odd, p < 2^15) is stored in
// balanced form: the representative in [-(p-1)/2, (p-1)/2] as int32.  A
// product of two balanced residues is below 2^28 in magnitude, so eight of
// them sum inside int32 next to a partially reduced value below 2^16.
// reduce_partial() brings any int32 back below 2p in magnitude with one
// multiply-high and one multiply-add (a Barrett step with m = floor(2^32/p)).

struct Mod {
    int32_t p;
    int32_t half;       // (p-1)/2
    int32_t barrett;    // floor(2^32 / p)
    uint32_t shift;     // half + K p with K p the largest multiple of p below 2^31 (reduce_balanced_fast)
};

inline Mod make_mod(uint32_t p) {
    Mod m;
    m.p = static_cast<int32_t>(p);
    m.half = static_cast<int32_t>((p - 1) / 2);
    m.barrett = static_cast<int32_t>((uint64_t{1} << 32) / p);
    m.shift = static_cast<uint32_t>(m.half) + static_cast<uint32_t>(((uint32_t{1} << 31) - 1) / p * p);
    return m;
}

__host__ __device__ __forceinline__ int32_t mulhi_s32(int32_t a, int32_t b) {
#if defined(__CUDA_ARCH__)
    return __mulhi(a, b);
#else
    return static_cast<int32_t>((static_cast<int64_t>(a) * b) >> 32);
#endif
}

// result in [-p, 2p), result == x (mod p).  q = floor(x*barrett / 2^32) is
// floor(x/p) or one off (below for x >= 0, above for x < 0).
__host__ __device__ __forceinline__ int32_t reduce_partial(int32_t x, const Mod& m) {
    return x - mulhi_s32(x, m.barrett) * m.p;
}

// Exact balanced representative of any int32.
__host__ __device__ __forceinline__ int32_t reduce_balanced(int32_t x, const Mod& m) {
    int32_t r = reduce_partial(x, m);   // [-p, 2p)
    if (r < 0) r += m.p;                // [0, 2p)
    if (r >= m.p) r -= m.p;             // [0, p)
    if (r > m.half) r -= m.p;           // balanced
    return r;
}

__host__ __device__ __forceinline__ uint32_t mulhi_u32(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
    return __umulhi(a, b);
#else
    return static_cast<uint32_t>((static_cast<uint64_t>(a) * b) >> 32);
#endif
}

// Exact balanced representative of x for |x| <= 2^31 - 2p, with one Barrett
// step and one correction.  y = x + half + K p lies in [0, 2^32); q =
// floor(y * barrett / 2^32) is floor(y / p) or one below, so s = y - q p is in
// [0, 2p) and s - half is congruent to x; one subtraction of p brings it into
// [-half, half].
__host__ __device__ __forceinline__ int32_t reduce_balanced_fast(int32_t x, const Mod& m) {
    const uint32_t y = static_cast<uint32_t>(x) + m.shift;
    const uint32_t q = mulhi_u32(y, static_cast<uint32_t>(m.barrett));
    const int32_t s = static_cast<int32_t>(y - q * static_cast<uint32_t>(m.p));
    return s - (s >= m.p ? m.p + m.half : m.half);
}

// Bytewise negation of four signed bytes in [-127, 127] (SWAR: 0x80 - the low
// seven bits never borrows across a byte; the sign bit is then fixed up).
__host__ __device__ __forceinline__ uint32_t neg_bytes4(uint32_t w) {
    return (0x80808080u - (w & 0x7F7F7F7Fu)) ^ (~w & 0x80808080u);
}

__host__ __device__ __forceinline__ int32_t to_balanced(uint32_t canonical, const Mod& m) {
    int32_t v = static_cast<int32_t>(canonical);
    return v > m.half ? v - m.p : v;
}

__host__ __device__ __forceinline__ uint32_t to_canonical(int32_t balanced, const Mod& m) {
    return static_cast<uint32_t>(balanced < 0 ? balanced + m.p : balanced);
}

// ------------------------------------------------------------ seeded data
//
// Counter-based stream: value number idx of stream (seed, tag) is the
// splitmix64 finaliser of  mix(seed ^ golden2*(tag+1)) + (idx+1)*golden,
// mapped onto [lo, p) by a 64x64->128 multiply-shift.  Host and device give
// identical values, so large seeded blocks are filled on the GPU.

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

__host__ __device__ __forceinline__ uint64_t seeded_stream_base(uint64_t seed, uint32_t tag) {
    return mix64(seed ^ (0xD1B54A32D192ED03ULL * static_cast<uint64_t>(tag + 1)));
}

__host__ __device__ __forceinline__ uint32_t seeded_residue_from_base(uint64_t base, uint64_t idx,
                                                                      uint32_t p, uint32_t lo) {
    uint64_t z = mix64(base + (idx + 1) * 0x9E3779B97F4A7C15ULL);
#if defined(__CUDA_ARCH__)
    uint64_t hi = __umul64hi(z, static_cast<uint64_t>(p - lo));
#else
    uint64_t hi = static_cast<uint64_t>((static_cast<unsigned __int128>(z) * (p - lo)) >> 64);
#endif
    return lo + static_cast<uint32_t>(hi);
}

enum SeedTag : uint32_t { TAG_MAPS = 1, TAG_DIAG = 2, TAG_X = 3, TAG_Y = 4 };

// ---------------------------------------------------------------- subsets

// Binomial coefficients C(n, k) for n, k <= 64 (host table).
uint64_t binom(int n, int k);

// Lexicographic rank of a sorted k-subset of {0..r-1}:
// rank = C(r,k) - 1 - sum_pos C(r-1-s_pos, k-pos).
uint64_t lex_rank(const int* s, int r, int k);

// Unrank (lexicographic, itertools.combinations order).
void lex_unrank(uint64_t rank, int r, int k, int* out);

// ------------------------------------------------------------- device info

int sm_count(int device);

}  // namespace bw
