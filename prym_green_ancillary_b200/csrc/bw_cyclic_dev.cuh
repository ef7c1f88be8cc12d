// Device helpers shared by the paper-mode kernels (bw_cyclic.cu,
// bw_cyclic_subset.cu): four-column balanced-residue rows held as one int4.
#pragma once

#include "bw_common.cuh"

namespace bw {
namespace cyc {

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

}  // namespace cyc
}  // namespace bw
