// Context of the synthetic Koszul engine (shared by the plain and INT8 forms).
#pragma once

#include "bw_common.cuh"
#include "../../include/bw_engine.h"

#include <memory>
#include <string>
#include <vector>

namespace bw {

struct KoszulCtx {
    // shape
    int device = 0, sms = 0;
    int r = 0, k = 0, ci = 0, co = 0, ci8 = 0, co8 = 0, nb = 0, m = 0;
    // plain form: output rows per thread of the d and d^T gathers (4 or 8)
    int tile_fwd = 4, tile_bwd = 4;
    int nbi = 0;   // block width inside the INT8 form (nb, or 16 for nb = 4 / 8: zero columns appended)
    uint32_t p = 0, form = BW_FORM_PLAIN;
    Mod mod{};
    uint64_t n_s = 0, n_t = 0, n_src = 0, n_tgt = 0;

    // device state
    cudaStream_t own_stream = nullptr;
    cudaEvent_t ev_join = nullptr;     // orders NULL-stream calls with the legacy stream
    std::vector<void*> allocations;
    uint64_t device_bytes = 0, scratch_bytes = 0;
    int32_t *d_coef_fwd = nullptr, *d_coef_bwd = nullptr;
    uint32_t *d_fwd = nullptr, *d_bwd = nullptr;
    int32_t* d_diag = nullptr;
    int32_t *d_ya = nullptr, *d_yb = nullptr, *d_z = nullptr, *d_xb = nullptr;
    std::vector<uint32_t> maps_canonical;

    // projection scratch
    unsigned proj_grid = 1;
    int32_t* d_partials = nullptr;
    unsigned int* d_counter = nullptr;
    unsigned long long* d_seq_index = nullptr;

    // sequence session
    bool in_session = false, cur_is_a = true;
    uint32_t* d_seq = nullptr;
    uint64_t seq_capacity = 0, seq_len = 0;
    static constexpr int kGraphPairs = 8;
    cudaGraphExec_t graphs[2] = {nullptr, nullptr};
    const uint32_t* graph_seq = nullptr;   // the sequence buffer the step graphs write
    uint64_t graph_launch_kernels = 0;
    uint64_t launches = 0;

    // host-buffer staging
    uint32_t *d_stage_x = nullptr, *d_stage_y = nullptr, *d_stage_seq = nullptr;
    uint64_t stage_seq_cap = 0;

    // INT8-limb form state (bw_koszul_i8.cu)
    struct I8State;
    I8State* i8 = nullptr;

    static KoszulCtx* create(const bw_koszul_desc& d, int dev);
    ~KoszulCtx();

    template <class T>
    T* alloc(uint64_t count);
    void release(void* p);

    void launch_to_balanced(const uint32_t* in, int32_t* out, uint64_t count, cudaStream_t st);
    void launch_to_canonical(const int32_t* in, uint32_t* out, uint64_t count, cudaStream_t st);

    void plain_forward(const int32_t* y, int32_t* z, cudaStream_t st);
    void plain_transpose(const int32_t* z, int32_t* w, bool scale, cudaStream_t st);
    void project(const int32_t* w, cudaStream_t st);
    void step_once(cudaStream_t st);

    void seq_start(const uint32_t* x, const uint32_t* y0, uint32_t* seq, uint64_t capacity, cudaStream_t st);
    void seq_step(uint64_t steps, cudaStream_t st);
    void seq_finish(uint32_t* y_out, uint64_t* nlen_out, cudaStream_t st);
    uint64_t kernels_per_step() const;
    uint64_t launches_in_pair_graph() const;
    void ensure_host_staging(uint64_t nlen);

    // INT8-limb form
    void plain_setup();            // chooses the plain gathers' tile heights (tile_fwd, tile_bwd)
    std::string plain_plan;        // the choice and its timings
    void i8_setup();
    void i8_destroy();
    uint64_t i8_kernels_per_step() const;
    enum { I8_YA = 0, I8_YB = 1, I8_Z = 2 };   // limb-plane block arrays
    void i8_run(bool forward_dir, int in_buf, int out_buf, bool scale, cudaStream_t st);
    void i8_check_error();
    double i8_time_direction(bool forward_dir, int in_buf, int out_buf);
    const std::string& i8_plan_text() const;
    void i8_to_limbs(const uint32_t* in, int buf, cudaStream_t st);
    void i8_from_limbs(int buf, uint32_t* out, cudaStream_t st);
    void i8_load_x(const uint32_t* x, cudaStream_t st);
    void i8_project(int buf, cudaStream_t st);
    void i8_step_once(cudaStream_t st);
    int i8_dim(int buf) const;
    uint64_t i8_rows(int buf) const;
};

}  // namespace bw

// Opaque handle of the C ABI (include/bw_engine.h).
struct bw_koszul {
    bw::KoszulCtx* impl;
};
