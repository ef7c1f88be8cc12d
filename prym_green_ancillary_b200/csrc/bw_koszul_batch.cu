// Batches of synthetic Koszul operators ("sectors" of uneven shapes, block
// widths and forms) whose block-Wiedemann sequences advance together.
//
// Each sector is an ordinary context (its own tables, limb planes and
// projection state).  A batch step advances every sector by one step; 16
// steps of all sectors are captured as ONE CUDA graph in which every sector
// runs on its own forked stream, so the sectors' kernels overlap wherever one
// sector's kernel leaves SMs idle (its tail), and the whole batch costs one
// graph launch per 16 steps.  Every sector kernel is already a persistent
// grid over all SMs with thousands of tiles, so merging sectors into a single
// kernel would save only those tails; the graph gives that overlap without
// giving up per-sector shared-memory plans.
#include "bw_koszul.cuh"

#include <memory>
#include <vector>

namespace bw {

struct KoszulBatch {
    int device = 0;
    std::vector<std::unique_ptr<KoszulCtx>> sectors;
    std::vector<bw_koszul> handles;        // borrowed per-sector handles
    std::vector<cudaStream_t> lanes;       // one stream per sector (graph branches)
    std::vector<cudaEvent_t> joins;
    cudaStream_t own_stream = nullptr;
    cudaEvent_t fork = nullptr, ev_legacy = nullptr;
    cudaGraphExec_t graphs[2] = {nullptr, nullptr};   // by the sectors' common starting buffer
    uint64_t graph_kernels = 0, launches = 0;
    bool in_session = false;
    uint64_t seq_len = 0, capacity = 0;
    static constexpr int kGraphSteps = 16;

    ~KoszulBatch() {
        cudaSetDevice(device);
        for (auto& g : graphs)
            if (g) cudaGraphExecDestroy(g);
        for (auto e : joins) cudaEventDestroy(e);
        for (auto s : lanes) cudaStreamDestroy(s);
        if (fork) cudaEventDestroy(fork);
        if (ev_legacy) cudaEventDestroy(ev_legacy);
        if (own_stream) cudaStreamDestroy(own_stream);
    }

    void drop_graphs() {
        for (auto& g : graphs)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
    }

    bool parity() const { return sectors.front()->cur_is_a; }

    void step_direct(cudaStream_t st) {
        for (auto& s : sectors) s->step_once(st);
    }

    // 16 steps of every sector, each sector on its own branch of one graph.
    void step_graph(cudaStream_t st) {
        const int gi = parity() ? 0 : 1;
        if (!graphs[gi]) {
            std::vector<bool> par;
            std::vector<uint64_t> l0;
            for (auto& s : sectors) {
                par.push_back(s->cur_is_a);
                l0.push_back(s->launches);
            }
            cudaGraph_t graph;
            BW_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            try {
                BW_CUDA(cudaEventRecord(fork, st));
                for (size_t i = 0; i < sectors.size(); ++i) {
                    BW_CUDA(cudaStreamWaitEvent(lanes[i], fork, 0));
                    for (int k = 0; k < kGraphSteps; ++k) sectors[i]->step_once(lanes[i]);
                    BW_CUDA(cudaEventRecord(joins[i], lanes[i]));
                    BW_CUDA(cudaStreamWaitEvent(st, joins[i], 0));
                }
            } catch (...) {
                cudaStreamEndCapture(st, &graph);
                throw;
            }
            BW_CUDA(cudaStreamEndCapture(st, &graph));
            graph_kernels = 0;
            for (size_t i = 0; i < sectors.size(); ++i) {   // capture does not execute
                sectors[i]->cur_is_a = par[i];
                graph_kernels += sectors[i]->launches - l0[i];
                sectors[i]->launches = l0[i];
            }
            BW_CUDA(cudaGraphInstantiate(&graphs[gi], graph, 0));
            cudaGraphDestroy(graph);
        }
        BW_CUDA(cudaGraphLaunch(graphs[gi], st));
        launches += graph_kernels;
        for (auto& s : sectors) {
            s->seq_len += kGraphSteps;
            for (int k = 0; k < kGraphSteps; ++k) s->cur_is_a = !s->cur_is_a;
        }
    }
};

}  // namespace bw

using namespace bw;

struct bw_koszul_batch {
    KoszulBatch* impl;
};

namespace {

// NULL stream: ordered like the legacy default stream (as for single contexts).
struct BatchStream {
    KoszulBatch& b;
    cudaStream_t st;
    bool joined;
    BatchStream(KoszulBatch& batch, void* stream)
        : b(batch), st(stream ? static_cast<cudaStream_t>(stream) : batch.own_stream), joined(stream == nullptr) {
        if (joined) {
            BW_CUDA(cudaEventRecord(b.ev_legacy, cudaStreamLegacy));
            BW_CUDA(cudaStreamWaitEvent(st, b.ev_legacy, 0));
        }
    }
    ~BatchStream() {
        if (joined && cudaEventRecord(b.ev_legacy, st) == cudaSuccess)
            cudaStreamWaitEvent(cudaStreamLegacy, b.ev_legacy, 0);
    }
};

}  // namespace

extern "C" int bw_koszul_batch_create(const bw_koszul_desc* descs, uint32_t count, int device,
                                      bw_koszul_batch** out) {
    return guarded([&] {
        BW_ARG(descs && out && count > 0, "bw_koszul_batch_create: null argument or empty batch");
        *out = nullptr;
        std::unique_ptr<KoszulBatch> b(new KoszulBatch());
        b->device = device;
        BW_CUDA(cudaSetDevice(device));
        BW_CUDA(cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking));
        BW_CUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
        BW_CUDA(cudaEventCreateWithFlags(&b->ev_legacy, cudaEventDisableTiming));
        for (uint32_t i = 0; i < count; ++i) {
            try {
                b->sectors.emplace_back(KoszulCtx::create(descs[i], device));
            } catch (const Error& e) {
                throw Error("sector " + std::to_string(i) + ": " + e.what(), e.code);
            }
            cudaStream_t lane;
            cudaEvent_t ev;
            BW_CUDA(cudaStreamCreateWithFlags(&lane, cudaStreamNonBlocking));
            b->lanes.push_back(lane);
            BW_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
            b->joins.push_back(ev);
        }
        for (auto& s : b->sectors) b->handles.push_back(bw_koszul{s.get()});
        *out = new bw_koszul_batch{b.release()};
    });
}

extern "C" void bw_koszul_batch_destroy(bw_koszul_batch* batch) {
    if (!batch) return;
    delete batch->impl;
    delete batch;
}

extern "C" int bw_koszul_batch_sector(bw_koszul_batch* batch, uint32_t index, bw_koszul** out) {
    return guarded([&] {
        BW_ARG(batch && out, "bw_koszul_batch_sector: null argument");
        BW_REQUIRE(index < batch->impl->sectors.size(), "bw_koszul_batch_sector: index out of range");
        *out = &batch->impl->handles[index];
    });
}

extern "C" int bw_koszul_batch_seq_start(bw_koszul_batch* batch, const uint32_t* const* d_x,
                                         const uint32_t* const* d_y0, uint32_t* const* d_seq,
                                         uint64_t seq_capacity, void* stream) {
    return guarded([&] {
        BW_ARG(batch && d_x && d_y0 && d_seq, "bw_koszul_batch_seq_start: null argument");
        KoszulBatch& b = *batch->impl;
        BW_CUDA(cudaSetDevice(b.device));
        BatchStream bs(b, stream);
        for (size_t i = 0; i < b.sectors.size(); ++i)
            b.sectors[i]->seq_start(d_x[i], d_y0[i], d_seq[i], seq_capacity, bs.st);
        b.capacity = seq_capacity;
        b.seq_len = 1;
        b.in_session = true;
        b.drop_graphs();   // new sequence buffers
    });
}

extern "C" int bw_koszul_batch_seq_step(bw_koszul_batch* batch, uint64_t steps, void* stream) {
    return guarded([&] {
        BW_REQUIRE(batch != nullptr, "bw_koszul_batch_seq_step: null batch");
        KoszulBatch& b = *batch->impl;
        BW_REQUIRE(b.in_session, "bw_koszul_batch_seq_step: no sequence session");
        BW_REQUIRE(b.seq_len + steps <= b.capacity, "bw_koszul_batch_seq_step: sequence capacity exceeded");
        BW_CUDA(cudaSetDevice(b.device));
        BatchStream bs(b, stream);
        for (; steps >= KoszulBatch::kGraphSteps; steps -= KoszulBatch::kGraphSteps) {
            b.step_graph(bs.st);
            b.seq_len += KoszulBatch::kGraphSteps;
        }
        for (; steps > 0; --steps) {
            b.step_direct(bs.st);
            for (auto& s : b.sectors) ++s->seq_len;
            ++b.seq_len;
        }
    });
}

extern "C" int bw_koszul_batch_seq_finish(bw_koszul_batch* batch, uint32_t* const* d_y_out, uint64_t* nlen_out,
                                          void* stream) {
    return guarded([&] {
        BW_REQUIRE(batch != nullptr, "bw_koszul_batch_seq_finish: null batch");
        KoszulBatch& b = *batch->impl;
        BW_REQUIRE(b.in_session, "bw_koszul_batch_seq_finish: no sequence session");
        BW_CUDA(cudaSetDevice(b.device));
        BatchStream bs(b, stream);
        for (size_t i = 0; i < b.sectors.size(); ++i)
            b.sectors[i]->seq_finish(d_y_out ? d_y_out[i] : nullptr, nullptr, bs.st);
        b.in_session = false;
        if (nlen_out) *nlen_out = b.seq_len;
    });
}

extern "C" uint64_t bw_koszul_batch_launch_count(const bw_koszul_batch* batch) {
    if (!batch) return 0;
    uint64_t n = batch->impl->launches;
    for (const auto& s : batch->impl->sectors) n += s->launches;
    return n;
}
