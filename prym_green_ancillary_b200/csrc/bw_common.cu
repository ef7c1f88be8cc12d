// Host helpers and the seeded-fill kernel shared by all engine parts.
#include "bw_common.cuh"
#include "../../include/bw_engine.h"

#include <mutex>
#include <vector>

namespace bw {

namespace {
thread_local std::string g_last_error;

struct BinomTable {
    uint64_t c[65][65];
    BinomTable() {
        for (int n = 0; n <= 64; ++n) {
            c[n][0] = 1;
            for (int k = 1; k <= 64; ++k) c[n][k] = (k > n) ? 0 : (n == 0 ? 0 : c[n - 1][k - 1] + c[n - 1][k]);
        }
    }
};
const BinomTable& binom_table() {
    static BinomTable t;
    return t;
}
}  // namespace

void set_last_error(const std::string& msg) { g_last_error = msg; }

uint64_t binom(int n, int k) {
    if (n < 0 || k < 0 || k > n || n > 64) return 0;
    return binom_table().c[n][k];
}

uint64_t lex_rank(const int* s, int r, int k) {
    uint64_t acc = 0;
    for (int pos = 0; pos < k; ++pos) acc += binom(r - 1 - s[pos], k - pos);
    return binom(r, k) - 1 - acc;
}

void lex_unrank(uint64_t rank, int r, int k, int* out) {
    int start = 0;
    for (int pos = 0; pos < k; ++pos) {
        int remaining = k - pos - 1;
        for (int v = start; v < r; ++v) {
            uint64_t cnt = binom(r - v - 1, remaining);
            if (rank < cnt) {
                out[pos] = v;
                start = v + 1;
                break;
            }
            rank -= cnt;
        }
    }
}

int sm_count(int device) {
    int n = 0;
    BW_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device));
    return n;
}

__global__ void seeded_fill_kernel(uint32_t* __restrict__ out, uint64_t count, uint64_t base,
                                   uint32_t p, uint32_t lo) {
    uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride)
        out[i] = seeded_residue_from_base(base, i, p, lo);
}

int max_dynamic_smem(int device) {
    int v = 0;
    BW_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    return v;
}

}  // namespace bw

using namespace bw;

extern "C" const char* bw_last_error(void) { return g_last_error.c_str(); }

extern "C" int bw_abi_version(void) { return BW_ABI_VERSION; }

extern "C" int bw_seeded_fill(uint32_t* d_out, uint64_t count, uint64_t seed, uint32_t tag,
                              uint32_t p, uint32_t lo, int device, void* stream) {
    return guarded([&] {
        BW_REQUIRE(p >= 2 && lo < p, "bw_seeded_fill: need 0 <= lo < p");
        if (count == 0) return;
        BW_REQUIRE(d_out != nullptr, "bw_seeded_fill: null output");
        BW_CUDA(cudaSetDevice(device));
        int sms = sm_count(device);
        uint64_t blocks = (count + 255) / 256;
        unsigned grid = static_cast<unsigned>(blocks < static_cast<uint64_t>(sms) * 8 ? blocks : sms * 8);
        seeded_fill_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(
            d_out, count, seeded_stream_base(seed, tag), p, lo);
        BW_CHECK_LAUNCH();
    });
}

extern "C" int bw_seeded_fill_host(uint32_t* out, uint64_t count, uint64_t seed, uint32_t tag,
                                   uint32_t p, uint32_t lo) {
    return guarded([&] {
        BW_REQUIRE(p >= 2 && lo < p, "bw_seeded_fill_host: need 0 <= lo < p");
        uint64_t base = seeded_stream_base(seed, tag);
        for (uint64_t i = 0; i < count; ++i) out[i] = seeded_residue_from_base(base, i, p, lo);
    });
}
