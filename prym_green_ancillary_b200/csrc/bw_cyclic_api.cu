// C ABI of the paper-mode engine (bw_cyclic_*), see include/bw_engine.h.
#include "bw_cyclic.cuh"
#include "wdm.hpp"

#include <cstring>
#include <filesystem>
#include <iostream>

using namespace bw;

struct bw_cyclic {
    CyclicCtx* impl;
};

extern "C" int bw_cyclic_open(const char* instance_path, const char* op, uint32_t sector, uint32_t num_v,
                              uint64_t seed, uint32_t rowmix_rounds, uint64_t rowmix_seed, const char* dense_path,
                              const char* drop_path, int device, bw_cyclic** out) {
    return guarded([&] {
        BW_ARG(instance_path && op && out, "bw_cyclic_open: null argument");
        *out = nullptr;
        DeformInputs deform{dense_path ? dense_path : "", drop_path ? drop_path : ""};
        CyclicCtx* c = CyclicCtx::open(instance_path, op, sector, num_v, seed, rowmix_rounds, rowmix_seed, device,
                                       nullptr, &deform);
        *out = new bw_cyclic{c};
    });
}

extern "C" int bw_cyclic_info_get(const bw_cyclic* ctx, bw_cyclic_info* out) {
    return guarded([&] {
        BW_ARG(ctx && out, "bw_cyclic_info_get: null argument");
        const CyclicCtx& c = *ctx->impl;
        std::memset(out, 0, sizeof(*out));
        out->rows = c.es.target_rows;
        out->cols = c.op_cols;
        out->x_cols = c.es.x_cols;
        out->z_cols = c.es.z_cols;
        out->t_rows = c.es.t_rows;
        out->y_rows = c.es.y_rows;
        out->dm_nnz = c.es.dm_nnz;
        out->d2_nnz = c.es.d2_nnz;
        out->default_nlen = (2 * c.op_cols) / c.num_v + 50;
        out->seq_len = c.seq_len;
        out->rowmix_realized_seed = c.plan.realized_seed;
        out->rowmix_hash = cyclic::rowmix_plan_hash(c.plan);
        out->device_bytes = c.device_bytes;
        out->genus = static_cast<uint32_t>(c.inst.genus);
        out->prime = c.p;
        out->order = static_cast<uint32_t>(c.inst.r);
        out->sector = static_cast<uint32_t>(c.es.sector);
        out->y_sector = static_cast<uint32_t>(c.es.y_sector);
        out->num_v = static_cast<uint32_t>(c.num_v);
    });
}

extern "C" void bw_cyclic_close(bw_cyclic* ctx) {
    if (!ctx) return;
    delete ctx->impl;
    delete ctx;
}

extern "C" int bw_cyclic_apply_host(bw_cyclic* ctx, int what, const uint32_t* in, uint32_t* out) {
    return guarded([&] {
        BW_ARG(ctx && in && out, "bw_cyclic_apply_host: null argument");
        ctx->impl->require_device();
        BW_CUDA(cudaSetDevice(ctx->impl->device));
        ctx->impl->apply_host(what, in, out);
    });
}

extern "C" int bw_cyclic_generate(bw_cyclic* ctx, uint64_t nlen) {
    return guarded([&] {
        BW_REQUIRE(ctx, "bw_cyclic_generate: null context");
        ctx->impl->require_device();
        BW_CUDA(cudaSetDevice(ctx->impl->device));
        ctx->impl->generate(nlen);
    });
}

extern "C" int bw_cyclic_generate_timed(bw_cyclic* ctx, uint64_t nlen, float* device_ms) {
    return guarded([&] {
        BW_ARG(ctx && device_ms, "bw_cyclic_generate_timed: null argument");
        ctx->impl->require_device();
        BW_CUDA(cudaSetDevice(ctx->impl->device));
        ctx->impl->generate(nlen, device_ms);
    });
}

extern "C" int bw_cyclic_download(bw_cyclic* ctx, uint32_t* packed_seq, uint64_t seq_capacity, uint32_t* current) {
    return guarded([&] {
        BW_REQUIRE(ctx, "bw_cyclic_download: null context");
        CyclicCtx& c = *ctx->impl;
        c.require_device();
        BW_REQUIRE(c.seq_len > 0, "bw_cyclic_download: no sequence generated");
        BW_CUDA(cudaSetDevice(c.device));
        std::vector<uint32_t> cur, packed;
        c.download_state(cur, packed);
        if (packed_seq) {
            BW_REQUIRE(seq_capacity >= c.seq_len, "bw_cyclic_download: sequence buffer too small");
            std::memcpy(packed_seq, packed.data(), packed.size() * sizeof(uint32_t));
        }
        if (current) std::memcpy(current, cur.data(), cur.size() * sizeof(uint32_t));
    });
}

extern "C" int bw_cyclic_output_path(const bw_cyclic* ctx, const char* out_dir, char* buf, size_t cap) {
    return guarded([&] {
        BW_ARG(ctx && buf, "bw_cyclic_output_path: null argument");
        const CyclicCtx& c = *ctx->impl;
        const std::string path = cyclic::sector_filename(out_dir ? out_dir : ".", c.op, c.es.sector, c.num_v,
                                                         c.plan.rounds, c.plan.seed);
        BW_REQUIRE(path.size() + 1 <= cap, "bw_cyclic_output_path: buffer too small");
        std::memcpy(buf, path.c_str(), path.size() + 1);
    });
}

extern "C" int bw_cyclic_check_outputs_absent(const char* wdm_path) {
    return guarded([&] {
        BW_REQUIRE(wdm_path, "bw_cyclic_check_outputs_absent: null path");
        cyclic::ensure_output_absent(wdm_path);
    });
}

extern "C" int bw_cyclic_write_sidecar(const bw_cyclic* ctx, const char* wdm_path) {
    return guarded([&] {
        BW_ARG(ctx && wdm_path, "bw_cyclic_write_sidecar: null argument");
        const CyclicCtx& c = *ctx->impl;
        cyclic::write_rowmix_sidecar(wdm_path, c.op, c.es.sector, c.es.target_rows, c.op_cols, c.num_v, c.p,
                                     c.seed, c.plan, c.row_precond, c.col_precond, c.initial_block);
    });
}

// save_all_data (cuda/cuprym_cyclic.cu:965-1007).
extern "C" int bw_cyclic_write_wdm(bw_cyclic* ctx, const char* wdm_path) {
    return guarded([&] {
        BW_ARG(ctx && wdm_path, "bw_cyclic_write_wdm: null argument");
        CyclicCtx& c = *ctx->impl;
        c.require_device();
        BW_REQUIRE(c.seq_len > 0, "bw_cyclic_write_wdm: no sequence generated");
        BW_CUDA(cudaSetDevice(c.device));
        std::vector<uint32_t> cur, packed;
        c.download_state(cur, packed);
        const std::string text = wdm::format_sym(c.es.target_rows, c.op_cols, c.p, c.num_v, c.row_precond,
                                                 c.col_precond, c.initial_block, cur, packed, c.seq_len);
        const std::string tmp = std::string(wdm_path) + ".tmp";
        wdm::write_file(tmp, text);
        std::filesystem::rename(tmp, wdm_path);
    });
}

extern "C" int bw_cyclic_validate(bw_cyclic* ctx, uint32_t columns) {
    return guarded([&] {
        BW_REQUIRE(ctx, "bw_cyclic_validate: null context");
        validate_ctx(*ctx->impl, columns);
    });
}

void bw::validate_ctx(CyclicCtx& c, uint32_t columns) {
    {
        c.require_device();
        BW_CUDA(cudaSetDevice(c.device));
        const size_t cols = std::max<size_t>(1, std::min<size_t>(columns, 16));
        std::cout << "Running eliminated CUDA self-validation with " << c.num_v << " deterministic RHS columns..."
                  << std::endl;
        cyclic::validate_rowmix_transpose_identity(c.plan, cols, c.p);
        std::cout << "Validation matched: eliminated target rowmix transpose identity" << std::endl;
        const size_t nc = c.op_cols;
        const uint64_t salts[3] = {0x404ULL, 0x505ULL, 0x606ULL};
        std::vector<std::vector<uint32_t>> blocks, images;
        for (int idx = 0; idx < 3; ++idx) {
            std::vector<uint32_t> in = cyclic::deterministic_block(nc, c.num_v, c.p, salts[idx]);
            std::vector<uint32_t> folded(nc * c.num_v), unfolded(nc * c.num_v);
            c.apply_host(BW_CYCLIC_APPLY_SQUARE, in.data(), folded.data());
            c.apply_host(BW_CYCLIC_APPLY_SQUARE_UNFOLDED, in.data(), unfolded.data());
            for (size_t e = 0; e < folded.size(); ++e)
                if (folded[e] != unfolded[e])
                    throw Error("eliminated square block " + std::to_string(idx) + " mismatch at (" +
                                    std::to_string(e / c.num_v) + "," + std::to_string(e % c.num_v) +
                                    "): folded=" + std::to_string(folded[e]) + ", round-by-round=" +
                                    std::to_string(unfolded[e]), 3);
            std::cout << "Validation matched: eliminated square block " << idx << " (" << nc << " x " << c.num_v
                      << ")" << std::endl;
            blocks.push_back(std::move(in));
            images.push_back(std::move(folded));
        }
        // S is symmetric: <S x, y> = <x, S y>.
        for (int a = 0; a < 3; ++a) {
            const int b = (a + 1) % 3;
            const uint32_t left = cyclic::dot_mod(images[a], blocks[b], c.p);
            const uint32_t right = cyclic::dot_mod(blocks[a], images[b], c.p);
            if (left != right)
                throw Error("eliminated square symmetry failed: <Sx,y>=" + std::to_string(left) +
                                ", <x,Sy>=" + std::to_string(right), 3);
        }
        std::cout << "Validation matched: eliminated square operator symmetry" << std::endl;
    }
}

extern "C" uint64_t bw_cyclic_launch_count(const bw_cyclic* ctx) { return ctx ? ctx->impl->launches : 0; }

extern "C" int bw_cyclic_gather_path(const bw_cyclic* ctx, char* buf, size_t cap) {
    return guarded([&] {
        BW_ARG(ctx && buf && cap > 0, "bw_cyclic_gather_path: null argument");
        const CyclicCtx& c = *ctx->impl;
        const std::string path = c.host_only ? std::string("none: host-only context")
                                 : c.subset_path ? std::string(c.stream_tables ? "subset: tables evict-first"
                                                                               : "subset: tables cached")
                                                 : "generic: " + c.subset_reason;
        BW_REQUIRE(path.size() < cap, "bw_cyclic_gather_path: buffer too small");
        std::memcpy(buf, path.c_str(), path.size() + 1);
    });
}

extern "C" int bw_file_read_text(const char* path, char* buf, size_t cap, size_t* len) {
    return guarded([&] {
        BW_ARG(path && len, "bw_file_read_text: null argument");
        const std::string text = wdm::read_file(path);
        *len = text.size();
        if (buf) {
            BW_REQUIRE(cap >= text.size(), "bw_file_read_text: buffer too small");
            std::memcpy(buf, text.data(), text.size());
        }
    });
}
