// INT8-limb tensor-core form of the synthetic Koszul operator (tcgen05 kind::i8).
// Not yet built: requesting the form fails loudly at context creation.
#include "bw_koszul.cuh"

namespace bw {

struct KoszulCtx::I8State {};

void KoszulCtx::i8_destroy() {
    delete i8;
    i8 = nullptr;
}
void KoszulCtx::i8_setup() { throw Error("the INT8-limb tensor-core form is not available in this build", 3); }
void KoszulCtx::i8_forward(const int32_t*, int32_t*, cudaStream_t) { i8_setup(); }
void KoszulCtx::i8_transpose(const int32_t*, int32_t*, bool, cudaStream_t) { i8_setup(); }
uint64_t KoszulCtx::i8_kernels_per_step() const { return 3; }

}  // namespace bw
