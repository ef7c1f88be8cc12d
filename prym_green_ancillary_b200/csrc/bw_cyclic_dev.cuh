// Device helpers shared by the paper-mode kernels (bw_cyclic.cu,
// bw_cyclic_subset.cu): four-column balanced-residue rows held as one int4.
#pragma once

#include "bw_common.cuh"

namespace bw {
namespace cyc {

// Programmatic dependent launch.  A kernel launched with the programmatic
// stream-serialization attribute may begin (stage its constant tables) while
// the kernel before it on the stream is still finishing; pdl_wait() blocks
// until that kernel has completed and its writes are visible, so it must come
// before the first access to any buffer an earlier kernel reads or writes.
// pdl_trigger() lets the next kernel begin early.  Launched without the
// attribute, both are no-ops.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ int32_t red64(long long x, const Mod& m) {
    long long r = x % m.p;
    if (r > m.half) r -= m.p;
    if (r < -m.half) r += m.p;
    return static_cast<int32_t>(r);
}

// Four-column accumulator.  SMALL: int32 sums, exact because the host checked
// that (terms per output) * ((p-1)/2)^2 + 2p < 2^31 for every kernel of this
// sector (always true at the paper primes); otherwise int64 sums.
template <bool SMALL>
struct Acc4;

template <>
struct Acc4<true> {
    int32_t x = 0, y = 0, z = 0, w = 0;
    __device__ __forceinline__ void mac(int32_t c, const int4& v) {
        x += c * v.x;
        y += c * v.y;
        z += c * v.z;
        w += c * v.w;
    }
    __device__ __forceinline__ int4 reduce(const Mod& m) const {
        return make_int4(reduce_balanced(x, m), reduce_balanced(y, m), reduce_balanced(z, m), reduce_balanced(w, m));
    }
};

template <>
struct Acc4<false> {
    long long x = 0, y = 0, z = 0, w = 0;
    __device__ __forceinline__ void mac(int32_t c, const int4& v) {
        x += static_cast<long long>(c) * v.x;
        y += static_cast<long long>(c) * v.y;
        z += static_cast<long long>(c) * v.z;
        w += static_cast<long long>(c) * v.w;
    }
    __device__ __forceinline__ int4 reduce(const Mod& m) const {
        return make_int4(red64(x, m), red64(y, m), red64(z, m), red64(w, m));
    }
};

__device__ __forceinline__ int4 ld4(const int32_t* base, long long row) {
    return __ldg(reinterpret_cast<const int4*>(base) + row);
}
__device__ __forceinline__ void st4(int32_t* base, long long row, const int4& v) {
    reinterpret_cast<int4*>(base)[row] = v;
}
__device__ __forceinline__ int4 scale4(const int4& v, int32_t s, const Mod& m) {
    return make_int4(reduce_balanced(v.x * s, m), reduce_balanced(v.y * s, m), reduce_balanced(v.z * s, m),
                     reduce_balanced(v.w * s, m));
}
__device__ __forceinline__ int4 neg4(const int4& v) { return make_int4(-v.x, -v.y, -v.z, -v.w); }

// Operator column of base column q: q itself, or (replacement) q less the
// dropped columns before it, -1 for a dropped column (drop0 < drop1; -1: none).
__device__ __forceinline__ long long op_col(long long drop0, long long drop1, long long q) {
    if (drop0 < 0) return q;
    if (q == drop0 || q == drop1) return -1;
    return q - (q > drop0 ? 1 : 0) - (q > drop1 ? 1 : 0);
}

// Grid-wide sum of W balanced residues per CTA, without a partials array:
// threads 0..W-1 of every CTA add their CTA's value into acc[0..W) (int32 at
// L2; |total| <= gridDim.x * p/2 stays far below 2^31 for p < 2^15), and the
// CTA that finishes last gets the totals back, each thread t < W taking
// acc[t] and leaving 0 for the next launch.  Integer sums do not depend on
// the order of the additions, so the result is deterministic.  Every thread
// of the CTA calls it; returns true only in the last CTA.
__device__ __forceinline__ bool grid_sum(int32_t* acc, unsigned int* counter, int W, int32_t mine, int32_t& total,
                                         bool* am_last /* shared */) {
    if (static_cast<int>(threadIdx.x) < W) atomicAdd(acc + threadIdx.x, mine);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) *am_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!*am_last) return false;
    __threadfence();
    if (static_cast<int>(threadIdx.x) < W) total = atomicExch(acc + threadIdx.x, 0);
    return true;
}

}  // namespace cyc
}  // namespace bw
