// Times the reference's own CPU implementation of one application of the
// eliminated square operator S = Dc F^t T^t Dr T F Dc, the paper-mode hot
// path: cpu_apply_eliminated_square (cuda/cuprym_cyclic.cu:1921-1966), the
// function the reference's --validate-rowmix compares its CUDA kernels with.
// It is single-threaded, as the reference wrote it.
//
// Test and bench infrastructure (the CPU baseline of the paper workloads),
// never part of the engine.  oracle/build_ref.sh compiles this file with the
// reference's cuda/cuprym_cyclic.cu included from where it lies in the
// reference checkout (its main renamed), into oracle/_ref/bin/ref_cpu_square.
// The set-up below follows the reference's own order of calls: main
// (cuda/cuprym_cyclic.cu:2555-2676) and the set-up half of
// run_eliminated_sector (:2159-2257), with the paper recipe's seeds (--seed 1,
// --rowmix-rounds 2, --rowmix-seed 10001, v = 4).  No CUDA call is made.
//
//   ref_cpu_square INSTANCE SECTOR SECONDS
// applies S repeatedly (at least once, then until SECONDS have passed) and
// prints one JSON line: rows, cols, applications, seconds, and a checksum of
// the last block.
#define main reference_cuprym_cyclic_main
#include REF_CYCLIC_SOURCE
#undef main

#include <chrono>
#include <cstdio>
#include <cstdlib>

int main(int argc, char** argv) {
    if (argc != 4) {
        std::fprintf(stderr, "usage: %s INSTANCE SECTOR SECONDS\n", argv[0]);
        return 2;
    }
    try {
        const std::string path = argv[1];
        const size_t sector = std::strtoull(argv[2], nullptr, 10);
        const double budget = std::atof(argv[3]);
        const size_t num_v = 4;
        const uint64_t random_seed = 1;
        CyclicInstance instance = load_cyclic_instance(path);
        if (sector >= instance.r) throw std::runtime_error("sector out of range");
        CharacterMap a0_map = build_character_map(instance.weight_a0, instance.r, "A0");
        CharacterMap a1_map = build_character_map(instance.weight_a1, instance.r, "A1");
        vector<size_t> u_indices;
        vector<uint16_t> u_weights;
        for (size_t i = 0; i < instance.n; ++i) {
            if (i == instance.elimination_w_index) continue;
            u_indices.push_back(i);
            u_weights.push_back(instance.weight_v[i]);
        }
        CharacterMap kernel_map = build_character_map(instance.elimination_kernel_weights, instance.r, "ker(mu_w)");
        CyclicCommonIncidence common_dm = build_common_incidences_generic(
            u_indices.size(), instance.m, instance.r, u_indices, u_weights, "eliminated D_m");
        CyclicCommonIncidence common_d2 = build_common_incidences_generic(
            u_indices.size(), instance.m - 1, instance.r, u_indices, u_weights, "eliminated D_(m-1)");

        const size_t y_sector = sub_mod(sector, instance.elimination_w_weight, instance.r);
        CyclicSectorLayout dm_layout =
            build_sector_layout_generic(instance, common_dm, a0_map, a1_map, sector, "eliminated D_m");
        CyclicSectorLayout d2_layout =
            build_sector_layout_generic(instance, common_d2, a0_map, a1_map, y_sector, "eliminated D_(m-1)");
        CyclicTensorLayout z_layout =
            build_tensor_layout(common_dm.row_subset_weights, kernel_map, instance.r, y_sector, "eliminated z");
        const size_t x_cols = dm_layout.column_descriptors.size();
        const size_t t_rows = dm_layout.row_descriptors.size();
        const size_t y_rows = d2_layout.column_descriptors.size();
        const size_t z_cols = z_layout.descriptors.size();
        const size_t target_rows = d2_layout.row_descriptors.size();
        const size_t total_cols = x_cols + z_cols;

        const my_int storage_prime = static_cast<my_int>(instance.modulus);
        std::mt19937_64 gen(seeded_sector_value(random_seed, sector));
        vector<my_int> row_precond = generate_random_vector(target_rows, storage_prime, gen, true);
        vector<my_int> col_precond = generate_random_vector(total_cols, storage_prime, gen, true);
        vector<my_int> block = generate_random_vector(total_cols * num_v, storage_prime, gen);
        RowMixPlan rowmix_plan =
            generate_rowmix_plan(target_rows, "eliminated", sector, instance.modulus, RowMixOptions{2, 10001});
        CyclicPhiHostData<my_int> dm_host = make_operator_host_data(
            instance, common_dm, std::move(dm_layout), a0_map, a1_map, ones_vector(t_rows), ones_vector(x_cols));
        CyclicPhiHostData<my_int> d2_host =
            make_operator_host_data(instance, common_d2, std::move(d2_layout), a0_map, a1_map,
                                    rowmix_plan.enabled() ? ones_vector(target_rows) : row_precond,
                                    ones_vector(y_rows));

        vector<my_int> out;
        size_t applications = 0;
        const auto t0 = std::chrono::steady_clock::now();
        double elapsed = 0.0;
        do {
            cpu_apply_eliminated_square(dm_host, d2_host, z_layout, instance, col_precond, row_precond, rowmix_plan,
                                        x_cols, z_cols, block, num_v, instance.modulus, out);
            block.swap(out);
            ++applications;
            elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        } while (elapsed < budget);
        uint64_t checksum = 0;
        for (my_int v : block) checksum = checksum * 1000003ull + v;
        std::printf("{\"rows\": %zu, \"cols\": %zu, \"applications\": %zu, \"seconds\": %.6f, \"checksum\": %llu}\n",
                    target_rows, total_cols, applications, elapsed, static_cast<unsigned long long>(checksum));
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_cpu_square error: %s\n", e.what());
        return 1;
    }
    return 0;
}
