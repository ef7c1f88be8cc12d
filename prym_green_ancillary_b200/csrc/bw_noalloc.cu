// Block projection a = X^T W that allocates nothing.
//
// Some callers cannot allocate device memory: a host framework whose caching
// allocator or arena owns every byte of HBM (an allocation behind its back
// can fail or fragment its pool), or a caller in a section where cudaMalloc /
// cudaFree would implicitly synchronise the device and stall its other
// streams.  For them this entry point keeps its cross-CTA scratch in a fixed
// array compiled into the library instead of memory the engine or the caller
// allocates.
//
// The scratch array (kScratchWords 32-bit words, 1 MiB + 256 B) lives on every
// GPU that loads the library until the process exits.  All calls share it:
// calls that overlap on the GPU (two streams, or two threads on one device)
// race on it and give wrong results.  The arrival counter it holds is cleared
// at the start of every call; the partial sums are overwritten before they
// are read.
#include "bw_common.cuh"
#include "../../include/bw_engine.h"

#include <cuda.h>   // CUcontext, CUresult: the driver's cuCtxGetCurrent, reached through the runtime

#include <algorithm>
#include <cstdint>
#include <mutex>

namespace bw {

namespace {

constexpr int kNoAllocThreads = 256;
constexpr unsigned kNoAllocMaxCtas = 256;
constexpr unsigned kNoAllocMaxEntries = 32 * 32;   // m x n
constexpr size_t kCounterWords = 64;               // 256 B: the arrival counter, padded
constexpr size_t kScratchWords = kCounterWords + static_cast<size_t>(kNoAllocMaxCtas) * kNoAllocMaxEntries;

// In host code this name is only a host-side stand-in: the kernel receives the
// device address obtained with cudaGetSymbolAddress.
static __device__ __align__(256) int32_t bw_noalloc_scratch[kScratchWords];

// The calling thread's current CUDA context.  The scratch address is only
// valid in the context it was looked up in: after cudaDeviceReset the device's
// primary context is a new one, with the library's module loaded anew.
using CtxGetCurrentFn = CUresult (*)(CUcontext*);

void* current_context() {
    static const CtxGetCurrentFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<CtxGetCurrentFn>(f);
    }();
    BW_REQUIRE(fn != nullptr, "bw_project_noalloc: cuCtxGetCurrent is not available from the driver");
    CUcontext ctx = nullptr;
    BW_REQUIRE(fn(&ctx) == CUDA_SUCCESS && ctx != nullptr, "bw_project_noalloc: no current CUDA context");
    return ctx;
}

struct ScratchEntry {
    void* context = nullptr;   // the context the address belongs to
    void* address = nullptr;
};
std::mutex g_symbol_mutex;
ScratchEntry g_symbol_address[64];   // per device ordinal

// Device address of the scratch array on `device` (which must be current):
// looked up once per device with cudaGetSymbolAddress, and again when the
// device's current context has changed since (cudaDeviceReset).
void* scratch_address(int device) {
    BW_ARG(device >= 0 && device < 64, "bw_project_noalloc: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_symbol_mutex);
    ScratchEntry& e = g_symbol_address[device];
    void* ctx = current_context();
    if (e.address == nullptr || e.context != ctx) {
        void* ptr = nullptr;
        BW_CUDA(cudaGetSymbolAddress(&ptr, bw_noalloc_scratch));
        BW_REQUIRE(ptr != nullptr, "bw_project_noalloc: scratch symbol has no device address");
        e.context = ctx;
        e.address = ptr;
    }
    return e.address;
}

// Same decomposition as the engine's projection: every CTA folds a strided
// share of the rows into m x n partial sums, the last CTA to arrive reduces
// the partials in a fixed order and writes canonical residues.
template <int NB>
__global__ void __launch_bounds__(kNoAllocThreads) project_noalloc_kernel(
    const uint32_t* __restrict__ X, const uint32_t* __restrict__ W, long long rows, int m, uint32_t* __restrict__ out,
    int32_t* __restrict__ scratch, Mod mod) {
    constexpr int JG = NB / 4;
    unsigned int* counter = reinterpret_cast<unsigned int*>(scratch);
    int32_t* partials = scratch + kCounterWords;
    const int tps = m * JG;
    const int slices = blockDim.x / tps;
    const int slice = threadIdx.x / tps;
    const int sub = threadIdx.x - slice * tps;
    const int x = sub / JG;
    const int jg = sub - x * JG;
    __shared__ int32_t red[kNoAllocThreads * 4];
    __shared__ bool am_last;

    int32_t acc[4] = {0, 0, 0, 0};
    int cnt = 0;
    for (long long row = static_cast<long long>(blockIdx.x) * slices + slice; row < rows;
         row += static_cast<long long>(gridDim.x) * slices) {
        const uint32_t p = static_cast<uint32_t>(mod.p);
        const int32_t xv = to_balanced(__ldg(X + row * m + x) % p, mod);
        const uint4 w = __ldg(reinterpret_cast<const uint4*>(W + row * NB) + jg);
        acc[0] += xv * to_balanced(w.x % p, mod);
        acc[1] += xv * to_balanced(w.y % p, mod);
        acc[2] += xv * to_balanced(w.z % p, mod);
        acc[3] += xv * to_balanced(w.w % p, mod);
        if (++cnt == 8) {
            cnt = 0;
#pragma unroll
            for (int a = 0; a < 4; ++a) acc[a] = reduce_partial(acc[a], mod);
        }
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) red[threadIdx.x * 4 + a] = reduce_balanced(acc[a], mod);
    __syncthreads();
    if (threadIdx.x < tps) {
        int32_t s[4] = {0, 0, 0, 0};
        for (int sl = 0; sl < slices; ++sl)
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                s[a] += red[(sl * tps + threadIdx.x) * 4 + a];
                if ((sl & 7) == 7) s[a] = reduce_partial(s[a], mod);
            }
        const int xx = threadIdx.x / JG, jj = threadIdx.x - xx * JG;
        int32_t* dst = partials + (static_cast<size_t>(blockIdx.x) * m + xx) * NB + jj * 4;
#pragma unroll
        for (int a = 0; a < 4; ++a) dst[a] = reduce_balanced(s[a], mod);
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) am_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    const int entries = m * NB;
    for (int e = threadIdx.x; e < entries; e += blockDim.x) {
        int32_t s = 0;
        for (unsigned b = 0; b < gridDim.x; ++b) {
            s += reinterpret_cast<volatile int32_t*>(partials)[static_cast<size_t>(b) * entries + e];
            if ((b & 7) == 7) s = reduce_partial(s, mod);
        }
        out[e] = to_canonical(reduce_balanced(s, mod), mod);
    }
    __syncthreads();
    if (threadIdx.x == 0) *counter = 0;
}

}  // namespace

}  // namespace bw

using namespace bw;

extern "C" int bw_project_noalloc(const uint32_t* d_x, const uint32_t* d_w, uint64_t rows, uint32_t m, uint32_t n,
                                  uint32_t prime, uint32_t* d_out, int device, void* stream) {
    return guarded([&] {
        BW_ARG(d_x && d_w && d_out, "bw_project_noalloc: null buffer");
        auto ok_w = [](uint32_t w) { return w == 4 || w == 8 || w == 16 || w == 32; };
        BW_ARG(ok_w(m) && ok_w(n),
                   "bw_project_noalloc: m and n must be 4, 8, 16 or 32 (the scratch holds at most 32 x 32 sums per CTA)");
        BW_ARG(prime >= 3 && prime < 32768 && (prime & 1u), "bw_project_noalloc: prime must be odd and below 2^15");
        BW_ARG(rows >= 1 && rows < (1ull << 40), "bw_project_noalloc: rows must be in 1..2^40-1");
        BW_ARG(reinterpret_cast<uintptr_t>(d_w) % 16 == 0, "bw_project_noalloc: W must be 16-byte aligned");
        BW_CUDA(cudaSetDevice(device));
        int32_t* scratch = static_cast<int32_t*>(scratch_address(device));
        const int sms = sm_count(device);
        const uint64_t wanted = (rows + kNoAllocThreads - 1) / kNoAllocThreads;
        const unsigned grid = static_cast<unsigned>(
            std::max<uint64_t>(1, std::min<uint64_t>({wanted, static_cast<uint64_t>(sms) * 2, kNoAllocMaxCtas})));
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        // The arrival counter must start at zero; an earlier call that failed
        // mid-way could have left it elsewhere.
        BW_CUDA(cudaMemsetAsync(scratch, 0, sizeof(unsigned int), st));
        const Mod mod = make_mod(prime);
        switch (n) {
            case 4: project_noalloc_kernel<4><<<grid, kNoAllocThreads, 0, st>>>(d_x, d_w, (long long)rows, (int)m, d_out, scratch, mod); break;
            case 8: project_noalloc_kernel<8><<<grid, kNoAllocThreads, 0, st>>>(d_x, d_w, (long long)rows, (int)m, d_out, scratch, mod); break;
            case 16: project_noalloc_kernel<16><<<grid, kNoAllocThreads, 0, st>>>(d_x, d_w, (long long)rows, (int)m, d_out, scratch, mod); break;
            default: project_noalloc_kernel<32><<<grid, kNoAllocThreads, 0, st>>>(d_x, d_w, (long long)rows, (int)m, d_out, scratch, mod); break;
        }
        BW_CHECK_LAUNCH();
    });
}
