// Kernel-vector recovery for the eliminated operator (paper mode).
//
// Replaces cuda/cuprym_cyclic_kernel_vectors.cu: from the WDM initial state
// V, its sidecar and the bcw generator G(x) = sum_k G_k x^k it forms
//   D = sum_k S^k V G_k^t      (recover_kernel_vectors_core, :2550-2703),
// certifies F Dc D = 0 on the device, ranks the candidate columns on the
// host and writes the two null-vector files and the JSON report in the
// reference's formats (:1412-1468, :1645-1733).
#include "bw_cyclic.cuh"
#include "json_lite.hpp"
#include "wdm.hpp"

#include <chrono>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <sstream>

namespace bw {

namespace {

// D[row][c] += sum_i B[row][i] * G_k[c][i]   (G_k row-major 4 x 4, balanced)
__global__ void cyc_accumulate_generator_kernel(const int32_t* __restrict__ B, const int32_t* __restrict__ G,
                                                const unsigned long long* __restrict__ k_index,
                                                int32_t* __restrict__ D, long long rows, Mod mod) {
    const int32_t* g = G + (*k_index) * 16;
    int32_t gm[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) gm[e] = __ldg(g + e);
    for (long long row = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; row < rows;
         row += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int4 b = __ldg(reinterpret_cast<const int4*>(B) + row);
        int4 d = reinterpret_cast<int4*>(D)[row];
        int32_t acc[4] = {d.x, d.y, d.z, d.w};
#pragma unroll
        for (int c = 0; c < 4; ++c)
            acc[c] = reduce_balanced(acc[c] + gm[c * 4 + 0] * b.x + gm[c * 4 + 1] * b.y + gm[c * 4 + 2] * b.z +
                                         gm[c * 4 + 3] * b.w,
                                     mod);
        reinterpret_cast<int4*>(D)[row] = make_int4(acc[0], acc[1], acc[2], acc[3]);
    }
}

__global__ void cyc_advance_index_kernel(unsigned long long* k_index) { *k_index += 1; }

}  // namespace

void CyclicCtx::recover(const std::vector<uint32_t>& generators, size_t generator_count,
                        std::vector<uint32_t>& candidates, std::vector<uint32_t>& product, long long& runtime_ms) {
    require_device();
    const size_t nc = op_cols, nr = es.target_rows, v = num_v;
    BW_REQUIRE(generators.size() == generator_count * v * v, "generator storage has the wrong size");
    // 4 x 4 balanced generator matrices; products of a 4-term row stay far inside int32
    std::vector<int32_t> g(generators.size());
    for (size_t e = 0; e < g.size(); ++e) g[e] = ::bw::to_balanced(generators[e] % p, mod);
    int32_t* d_g = upload(g);
    int32_t* d_cand = alloc<int32_t>(nc * v);
    unsigned long long* d_k = alloc<unsigned long long>(1);
    BW_CUDA(cudaMemsetAsync(d_cand, 0, nc * v * sizeof(int32_t), stream));
    BW_CUDA(cudaMemsetAsync(d_k, 0, sizeof(unsigned long long), stream));
    uint32_t* tmp = scratch_canonical();
    BW_CUDA(cudaMemcpyAsync(tmp, initial_block.data(), nc * v * 4, cudaMemcpyHostToDevice, stream));
    to_balanced(tmp, d_b, nc * v);
    BW_CUDA(cudaStreamSynchronize(stream));

    const auto t0 = std::chrono::high_resolution_clock::now();
    // One iteration = accumulate G_k, advance k, B <- S B (captured once, replayed).
    auto iteration = [&](int32_t* cur, int32_t* nxt) {
        cyc_accumulate_generator_kernel<<<grid_for(nc), 256, 0, stream>>>(cur, d_g, d_k, d_cand,
                                                                        static_cast<long long>(nc), mod);
        BW_CHECK_LAUNCH();
        cyc_advance_index_kernel<<<1, 1, 0, stream>>>(d_k);
        BW_CHECK_LAUNCH();
        launches += 2;
        apply_square(cur, nxt);
    };
    cudaGraphExec_t pair = nullptr;
    size_t k = 0;
    if (generator_count >= 3) {
        const uint64_t l0 = launches;
        cudaGraph_t graph;
        BW_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        try {
            iteration(d_b, d_d);
            iteration(d_d, d_b);
        } catch (...) {
            cudaStreamEndCapture(stream, &graph);
            throw;
        }
        BW_CUDA(cudaStreamEndCapture(stream, &graph));
        const uint64_t per_pair = launches - l0;
        launches = l0;
        BW_CUDA(cudaGraphInstantiate(&pair, graph, 0));
        cudaGraphDestroy(graph);
        // the last generator needs no further application of S
        while (k + 2 < generator_count) {
            BW_CUDA(cudaGraphLaunch(pair, stream));
            launches += per_pair;
            k += 2;
        }
    }
    int32_t* cur = d_b;
    int32_t* nxt = d_d;
    if (k % 2 == 1) std::swap(cur, nxt);
    for (; k < generator_count; ++k) {
        if (k + 1 < generator_count) {
            iteration(cur, nxt);
            std::swap(cur, nxt);
        } else {
            cyc_accumulate_generator_kernel<<<grid_for(nc), 256, 0, stream>>>(cur, d_g, d_k, d_cand,
                                                                            static_cast<long long>(nc), mod);
            BW_CHECK_LAUNCH();
            ++launches;
        }
    }
    // certificate: F (Dc D)
    forward(d_cand, d_u, true);
    BW_CUDA(cudaStreamSynchronize(stream));
    runtime_ms = std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::high_resolution_clock::now() - t0)
                     .count();
    if (pair) cudaGraphExecDestroy(pair);
    candidates.resize(nc * v);
    product.resize(nr * v);
    to_canonical(d_cand, tmp, nc * v);
    BW_CUDA(cudaMemcpyAsync(candidates.data(), tmp, nc * v * 4, cudaMemcpyDeviceToHost, stream));
    BW_CUDA(cudaStreamSynchronize(stream));
    to_canonical(d_u, tmp, nr * v);
    BW_CUDA(cudaMemcpyAsync(product.data(), tmp, nr * v * 4, cudaMemcpyDeviceToHost, stream));
    BW_CUDA(cudaStreamSynchronize(stream));
}

namespace recovery {

std::string default_generators_filename(const std::string& wdm) {
    for (const char* suf : {".wdm.zst", ".wdm"}) {
        const std::string s(suf);
        if (wdm.size() >= s.size() && wdm.compare(wdm.size() - s.size(), s.size(), s) == 0)
            return wdm.substr(0, wdm.size() - s.size()) + "_generators.txt";
    }
    return wdm + "_generators.txt";
}

// load_generators (cuda/cuprym_cyclic_kernel_vectors.cu:1287-1336): one v x v
// matrix per non-blank line, entries may be negative.
size_t load_generators(const std::string& path, size_t num_v, uint32_t prime, std::vector<uint32_t>& out) {
    std::ifstream in(path);
    if (!in.is_open()) throw std::runtime_error("failed to open generators file " + path);
    out.clear();
    std::string line;
    size_t line_number = 0;
    while (std::getline(in, line)) {
        ++line_number;
        if (line.find_first_not_of(" \t\r\n") == std::string::npos) continue;
        std::istringstream is(line);
        for (size_t i = 0; i < num_v * num_v; ++i) {
            long long v = 0;
            if (!(is >> v))
                throw std::runtime_error("generator line " + std::to_string(line_number) + " has too few entries");
            long long r = v % static_cast<long long>(prime);
            if (r < 0) r += prime;
            out.push_back(static_cast<uint32_t>(r));
        }
        std::string extra;
        if (is >> extra)
            throw std::runtime_error("generator line " + std::to_string(line_number) +
                                     " has more than num_v*num_v entries");
    }
    const size_t gs = num_v * num_v;
    if (out.size() % gs != 0) throw std::runtime_error("generator file does not contain complete generator matrices");
    const size_t count = out.size() / gs;
    if (count == 0) throw std::runtime_error("generator file does not contain any generator matrices");
    return count;
}

std::vector<size_t> column_nonzeros(const std::vector<uint32_t>& m, size_t rows, size_t cols, uint32_t p) {
    std::vector<size_t> counts(cols, 0);
    for (size_t r = 0; r < rows; ++r)
        for (size_t c = 0; c < cols; ++c)
            if (m[r * cols + c] % p) ++counts[c];
    return counts;
}

// rank_dense_candidate_columns (cuda/cuprym_cyclic_kernel_vectors.cu:1490-1546).
size_t rank_columns(const std::vector<uint32_t>& m, size_t rows, size_t cols, uint32_t p,
                    std::vector<size_t>& pivots) {
    std::vector<uint32_t> a = m;
    auto inv = [&](uint64_t x) {
        uint64_t r = 1, b = x % p, e = p - 2;
        while (e) {
            if (e & 1) r = r * b % p;
            b = b * b % p;
            e >>= 1;
        }
        return r;
    };
    pivots.clear();
    size_t rank = 0;
    for (size_t col = 0; col < cols && rank < rows; ++col) {
        size_t piv = rows;
        for (size_t r = rank; r < rows; ++r)
            if (a[r * cols + col] % p) {
                piv = r;
                break;
            }
        if (piv == rows) continue;
        if (piv != rank)
            for (size_t c = 0; c < cols; ++c) std::swap(a[rank * cols + c], a[piv * cols + c]);
        const uint64_t iv = inv(a[rank * cols + col]);
        for (size_t c = col; c < cols; ++c) a[rank * cols + c] = static_cast<uint32_t>(a[rank * cols + c] * iv % p);
        for (size_t r = 0; r < rows; ++r) {
            if (r == rank) continue;
            const uint64_t f = a[r * cols + col] % p;
            if (!f) continue;
            for (size_t c = col; c < cols; ++c) {
                const uint64_t sub = f * (a[rank * cols + c] % p) % p;
                const uint64_t cur = a[r * cols + c] % p;
                a[r * cols + c] = static_cast<uint32_t>(cur >= sub ? cur - sub : cur + p - sub);
            }
        }
        pivots.push_back(col);
        ++rank;
    }
    return rank;
}

// save_candidate_vectors (cuda/cuprym_cyclic_kernel_vectors.cu:1412-1468): one
// vector per line, optionally scaled by the source preconditioner.
void save_candidates(const std::string& path, const std::vector<uint32_t>& d, size_t rows, size_t cols,
                     const std::vector<uint32_t>* scale, uint32_t p) {
    std::filesystem::path out(path);
    if (out.has_parent_path()) std::filesystem::create_directories(out.parent_path());
    const std::string tmp = path + ".tmp";
    {
        std::ofstream o(tmp);
        if (!o.is_open()) throw std::runtime_error("failed to open output file " + tmp);
        std::string line;
        for (size_t c = 0; c < cols; ++c) {
            line.clear();
            for (size_t r = 0; r < rows; ++r) {
                uint64_t v = d[r * cols + c] % p;
                if (scale) v = v * (*scale)[r] % p;
                if (r) line += ' ';
                line += std::to_string(v);
            }
            line += '\n';
            o << line;
        }
        o.close();
        if (!o) throw std::runtime_error("failed while writing output file " + tmp);
    }
    std::filesystem::rename(tmp, path);
}

std::string join(const std::vector<size_t>& v) {
    std::string s;
    for (size_t i = 0; i < v.size(); ++i) s += (i ? ", " : "") + std::to_string(v[i]);
    return s;
}

}  // namespace recovery

}  // namespace bw

using namespace bw;

// Resolves the mixing recipe of a WDM from its sidecar (cuda/cuprym_cyclic_kernel_vectors.cu:1554-1643)
// and opens the operator with the WDM's preconditioners and initial block.
extern "C" int bw_cyclic_recover(const char* instance_path, const char* op, uint32_t sector, const char* wdm_path,
                                 const char* generators_path, const char* preconditioned_out,
                                 const char* original_out, const char* report_out, const char* dense_path,
                                 const char* drop_path, int64_t cli_rounds, uint64_t cli_seed, int rounds_supplied,
                                 int seed_supplied, int validate, int device) {
    return guarded([&] {
        BW_ARG(instance_path && op && wdm_path, "bw_cyclic_recover: null argument");
        const std::string wdm(wdm_path);
        const std::string gens = generators_path && *generators_path ? generators_path
                                                                     : recovery::default_generators_filename(wdm);
        const std::string out1 = preconditioned_out && *preconditioned_out ? preconditioned_out
                                                                           : wdm + "_nullvectors_1.txt";
        const std::string out2 = original_out && *original_out ? original_out : wdm + "_nullvectors_2.txt";
        const std::string rep = report_out && *report_out ? report_out : wdm + "_nullvectors_report.json";
        for (auto [f, label] : {std::pair<std::string, const char*>{instance_path, "Instance"}, {wdm, "WDM"},
                                {gens, "Generators"}})
            if (!std::filesystem::exists(f)) throw Error(std::string(label) + " file does not exist: " + f, 1);

        // Host-only open: assembly, deformation inputs and sector shapes (no device work yet).
        const DeformInputs deform{dense_path ? dense_path : "", drop_path ? drop_path : "", true};
        const bool deformation = std::string(op) != "eliminated";
        std::unique_ptr<CyclicCtx> probe(CyclicCtx::open(instance_path, op, sector, 4, 1, 0, 0, -1, nullptr, &deform));
        wdm::InitialState st = wdm::read_initial_state(wdm);
        const uint32_t p = probe->p;
        BW_REQUIRE(st.prime == p, "WDM prime does not match instance modulus");
        BW_REQUIRE(st.rows == probe->es.target_rows, deformation ? "WDM row count does not match deformation sector"
                                                                 : "WDM row count does not match eliminated sector");
        BW_REQUIRE(st.cols == probe->op_cols, deformation ? "WDM column count does not match deformation operator"
                                                          : "WDM column count does not match eliminated sector");
        BW_REQUIRE(st.num_v == 4, "WDM vector count must be 4 for this engine");
        for (size_t i = 0; i < st.row_precond.size(); ++i)
            BW_REQUIRE(st.row_precond[i] % p, "row preconditioner has a zero entry modulo the prime at index " +
                                                  std::to_string(i));
        for (size_t i = 0; i < st.col_precond.size(); ++i)
            BW_REQUIRE(st.col_precond[i] % p, "column preconditioner has a zero entry modulo the prime at index " +
                                                  std::to_string(i));
        CyclicSource src;
        src.row_precond = st.row_precond;
        src.col_precond = st.col_precond;
        src.initial_block = st.initial_rowmajor;
        const std::string side = cyclic::rowmix_sidecar_filename(wdm);
        if (!std::filesystem::exists(side)) {
            BW_REQUIRE(!(rounds_supplied && cli_rounds < 0), "--rowmix-rounds must be nonnegative");
            src.rowmix_rounds = rounds_supplied ? static_cast<size_t>(cli_rounds) : 0;
            src.rowmix_seed = cli_seed;
            if (src.rowmix_rounds > 0) std::cout << "No rowmix sidecar found; using CLI rowmix settings." << std::endl;
        } else {
            std::ifstream in(side, std::ios::binary);
            std::stringstream ss;
            ss << in.rdbuf();
            const json::Value doc = json::parse(ss.str());
            const json::Value& rm = doc.at("rowmix");
            const json::Value& hs = doc.at("hashes");
            BW_REQUIRE(doc.at("operator").s == op, "rowmix sidecar operator does not match CLI operator");
            BW_REQUIRE(doc.at("sector").as_u64("sector") == sector, "rowmix sidecar sector does not match CLI sector");
            BW_REQUIRE(doc.at("rows").as_u64("rows") == st.rows, "rowmix sidecar row count does not match WDM/operator");
            BW_REQUIRE(doc.at("columns").as_u64("columns") == st.cols,
                       "rowmix sidecar column count does not match WDM/operator");
            BW_REQUIRE(doc.at("vector_count").as_u64("vector_count") == st.num_v,
                       "rowmix sidecar vector count does not match WDM");
            BW_REQUIRE(doc.at("prime").as_u64("prime") == p, "rowmix sidecar prime does not match WDM");
            BW_REQUIRE(rm.at("target_rows").as_u64("target_rows") == st.rows,
                       "rowmix sidecar target row count does not match operator");
            BW_REQUIRE(hs.at("row_preconditioner_fnv1a64").s ==
                           cyclic::hex_u64(cyclic::fnv1a64_vector_hash(st.row_precond)),
                       "rowmix sidecar row-preconditioner hash does not match WDM");
            BW_REQUIRE(hs.at("column_preconditioner_fnv1a64").s ==
                           cyclic::hex_u64(cyclic::fnv1a64_vector_hash(st.col_precond)),
                       "rowmix sidecar column-preconditioner hash does not match WDM");
            BW_REQUIRE(hs.at("initial_block_fnv1a64").s ==
                           cyclic::hex_u64(cyclic::fnv1a64_vector_hash(st.initial_rowmajor)),
                       "rowmix sidecar initial-block hash does not match WDM");
            const uint64_t s_rounds = rm.at("rounds").as_u64("rounds"), s_seed = rm.at("seed").as_u64("seed");
            if (rounds_supplied)
                BW_REQUIRE(cli_rounds >= 0 && static_cast<uint64_t>(cli_rounds) == s_rounds,
                           "CLI --rowmix-rounds conflicts with rowmix sidecar");
            if (seed_supplied) BW_REQUIRE(cli_seed == s_seed, "CLI --rowmix-seed conflicts with rowmix sidecar");
            const cyclic::RowMixPlan plan = cyclic::generate_rowmix_plan(st.rows, op, sector, p, s_rounds, s_seed);
            BW_REQUIRE(plan.realized_seed == rm.at("realized_seed").as_u64("realized_seed"),
                       "regenerated rowmix realized seed does not match sidecar");
            BW_REQUIRE(cyclic::hex_u64(cyclic::rowmix_plan_hash(plan)) == rm.at("hash_fnv1a64").s,
                       "regenerated rowmix hash does not match sidecar");
            src.rowmix_rounds = s_rounds;
            src.rowmix_seed = s_seed;
            std::cout << "Loaded rowmix settings from " << side << std::endl;
        }
        std::vector<uint32_t> flat;
        const size_t count = recovery::load_generators(gens, st.num_v, p, flat);
        std::unique_ptr<CyclicCtx> c(CyclicCtx::open(instance_path, op, sector, 4, 1, 0, 0, device, &src, &deform));
        std::cout << "Recovery dimensions: rows=" << st.rows << ", columns=" << st.cols << ", v=" << st.num_v
                  << ", WDM sequence length=" << st.nlen << ", generator matrices=" << count << std::endl;
        if (count > st.nlen)
            std::cout << "Warning: generator count exceeds WDM sequence length; continuing because rust_rank "
                         "exported it."
                      << std::endl;
        if (validate) validate_ctx(*c, 4);
        std::vector<uint32_t> cand, prod;
        long long ms = 0;
        c->recover(flat, count, cand, prod, ms);
        const size_t nc = st.cols, nr = st.rows, v = st.num_v;
        const std::vector<size_t> prod_nnz = recovery::column_nonzeros(prod, nr, v, p);
        size_t prod_total = 0;
        for (size_t x : prod_nnz) prod_total += x;
        std::cout << "A*(source-preconditioned candidate) nonzeros by vector: ";
        for (size_t i = 0; i < v; ++i) std::cout << (i ? ", " : "") << i << ":" << prod_nnz[i];
        std::cout << std::endl;
        if (prod_total != 0) {
            // the first ten nonzero entries of F Dc D in row-major order, as
            // the reference prints them (cuda/cuprym_cyclic_kernel_vectors.cu:1390-1407, 2638-2641)
            std::cout << "First nonzero entries of certificate product:" << std::endl;
            size_t printed = 0;
            for (size_t row = 0; row < nr && printed < 10; ++row)
                for (size_t col = 0; col < v && printed < 10; ++col) {
                    const uint32_t value = prod[row * v + col] % p;
                    if (value != 0) {
                        std::cout << "  (" << row << ", " << col << ") = " << value << std::endl;
                        ++printed;
                    }
                }
            throw Error("kernel-vector certificate failed", 3);
        }
        std::cout << "Kernel-vector certificate passed." << std::endl;
        const std::vector<size_t> cand_nnz = recovery::column_nonzeros(cand, nc, v, p);
        size_t cand_total = 0;
        for (size_t x : cand_nnz) cand_total += x;
        BW_REQUIRE(cand_total != 0, "all candidate vectors are zero; no kernel vector was produced");
        std::vector<size_t> pivots;
        const size_t rank = recovery::rank_columns(cand, nc, v, p, pivots);
        std::cout << "Candidate block rank: " << rank << "/" << v << std::endl;
        std::cout << "GPU recovery runtime: " << ms << " ms" << std::endl;
        recovery::save_candidates(out1, cand, nc, v, nullptr, p);
        recovery::save_candidates(out2, cand, nc, v, &c->col_precond, p);
        // report (cuda/cuprym_cyclic_kernel_vectors.cu:1645-1733): same keys and order
        std::filesystem::path rp(rep);
        if (rp.has_parent_path()) std::filesystem::create_directories(rp.parent_path());
        const std::string tmp = rep + ".tmp";
        {
            std::ofstream o(tmp);
            if (!o) throw Error("failed to open metadata output " + tmp, 1);
            o << "{\n";
            o << "  \"type\": \"prym_cyclic_kernel_vectors_report\",\n";
            o << "  \"version\": 1,\n";
            o << "  \"instance\": \"" << instance_path << "\",\n";
            o << "  \"wdm_file\": \"" << wdm << "\",\n";
            o << "  \"generators_file\": \"" << gens << "\",\n";
            o << "  \"operator\": \"" << op << "\",\n";
            o << "  \"sector\": " << sector << ",\n";
            o << "  \"rows\": " << nr << ",\n";
            o << "  \"columns\": " << nc << ",\n";
            o << "  \"prime\": " << p << ",\n";
            o << "  \"vector_count\": " << v << ",\n";
            o << "  \"wdm_sequence_length\": " << st.nlen << ",\n";
            o << "  \"generator_count\": " << count << ",\n";
            o << "  \"runtime_ms\": " << ms << ",\n";
            o << "  \"rowmix\": {\n";
            o << "    \"rounds\": " << c->plan.rounds << ",\n";
            o << "    \"seed\": " << c->plan.seed << ",\n";
            o << "    \"realized_seed\": " << c->plan.realized_seed << ",\n";
            o << "    \"hash_fnv1a64\": \"" << cyclic::hex_u64(cyclic::rowmix_plan_hash(c->plan)) << "\"\n";
            o << "  },\n";
            o << "  \"candidate_nonzeros\": [" << recovery::join(cand_nnz) << "],\n";
            o << "  \"product_nonzeros\": [" << recovery::join(prod_nnz) << "],\n";
            o << "  \"candidate_rank\": " << rank << ",\n";
            o << "  \"pivot_columns\": [" << recovery::join(pivots) << "]\n";
            o << "}\n";
            o.close();
            if (!o) throw Error("failed while writing metadata output " + tmp, 1);
        }
        std::filesystem::rename(tmp, rep);
        std::cout << "Saved preconditioned candidates to " << out1 << std::endl;
        std::cout << "Saved original-coordinate candidates to " << out2 << std::endl;
        std::cout << "Saved metadata to " << rep << std::endl;
    });
}
