// Drop-in for the reference's cuprym_cyclic executable (cuda/cuprym_cyclic.cu:2498-2689):
// the same command line, refusals and output files, over the engine's C ABI.
#include "cli_common.hpp"

#include <chrono>
#include <iostream>

int main(int argc, char** argv) {
    try {
        bwcli::Parser app("CUDA cyclic-sector Wiedemann sequence computation for Prym Green Phi_g (B200 engine)");
        app.positional("instance", "Cyclic Prym fixture/instance JSON");
        app.option({"--operator"}, "Production operator: eliminated.", "eliminated");
        app.option({"--sector"}, "Run one sector/character.", "", true);
        app.option({"--out"}, "Output directory for per-sector WDM files.", ".");
        app.option({"-d", "--device"}, "Selects a CUDA device to use.", "0");
        app.option({"-v"}, "Paper block size: 4.", "4");
        app.option({"-s", "--saveafter"}, "Automatic saves every s seconds; 0 disables intermediate saves.", "0");
        app.option({"--seed"}, "Base deterministic RNG seed for preconditioners and starting vectors.", "1");
        app.option({"--rowmix-rounds"}, "Paper target row-mixing rounds: 2.", "2");
        app.option({"--rowmix-seed"}, "Independent deterministic RNG seed for row mixing.", "10001");
        app.flag({"--validate-rowmix"}, "Run the CUDA square-operator self-validation before sequence generation.");
        if (!app.parse(argc, argv)) return 0;

        const unsigned long long rounds = app.unsigned_integer("--rowmix-rounds");
        const unsigned long long rseed = app.unsigned_integer("--rowmix-seed");
        const unsigned long long seed = app.unsigned_integer("--seed");
        const unsigned long long save_after = app.unsigned_integer("--saveafter");
        if (rounds != 2 || rseed != 10001)
            throw std::runtime_error("The paper pipeline requires --rowmix-rounds 2 --rowmix-seed 10001.");
        if (seed != 1 || save_after != 0) throw std::runtime_error("The paper pipeline requires --seed 1 --saveafter 0.");
        if (app.str("--operator") != "eliminated") {
            std::cerr << "--operator must be eliminated." << std::endl;
            return 1;
        }
        if (app.unsigned_integer("-v") != 4) {
            std::cerr << "The paper pipeline requires exactly 4 block vectors." << std::endl;
            return 1;
        }
        const long long sector = app.integer("--sector");
        if (sector < 0) {
            std::cerr << "--sector must be nonnegative." << std::endl;
            return 1;
        }
        const int device = static_cast<int>(app.integer("--device"));

        std::cout << "Loading cyclic Prym instance JSON: " << app.str("instance") << std::endl;
        bw_cyclic* ctx = nullptr;
        bwcli::check(bw_cyclic_open(app.str("instance").c_str(), "eliminated", static_cast<uint32_t>(sector), 4, seed,
                                    static_cast<uint32_t>(rounds), rseed, nullptr, nullptr, device, &ctx));
        bw_cyclic_info info;
        bwcli::check(bw_cyclic_info_get(ctx, &info));
        std::cout << "\n=== Eliminated Sector " << sector << " ===" << std::endl;
        std::cout << "Reduced dimensions: " << info.rows << " x " << info.cols << " (x=" << info.x_cols
                  << ", z=" << info.z_cols << ", y=" << info.y_rows << ", t=" << info.t_rows
                  << "), y_sector=" << info.y_sector << std::endl;
        std::cout << "Implicit D nnz counts: D_m=" << info.dm_nnz << ", D_(m-1)=" << info.d2_nnz << std::endl;
        char path[4096];
        bwcli::check(bw_cyclic_output_path(ctx, app.str("--out").c_str(), path, sizeof(path)));
        bwcli::check(bw_cyclic_check_outputs_absent(path));
        bwcli::check(bw_cyclic_write_sidecar(ctx, path));
        std::cout << "Wrote rowmix sidecar for " << path << std::endl;
        if (app.on("--validate-rowmix")) bwcli::check(bw_cyclic_validate(ctx, 4));
        std::cout << "Computing " << (info.default_nlen - 1 + 3) / 4 << " eliminated BCW rounds for sector " << sector
                  << "." << std::endl;
        const auto t0 = std::chrono::high_resolution_clock::now();
        bwcli::check(bw_cyclic_generate(ctx, 0));
        const auto t1 = std::chrono::high_resolution_clock::now();
        const long long ms = std::chrono::duration_cast<std::chrono::milliseconds>(t1 - t0).count();
        bwcli::check(bw_cyclic_info_get(ctx, &info));
        std::cout << "Eliminated sector " << sector << " BCW sequence runtime: " << ms << " ms" << std::endl;
        if (ms > 0)
            std::cout << "Eliminated sector " << sector << " total throughput: " << info.seq_len * 4 * 1e3 / ms
                      << "/s." << std::endl;
        std::cout << "Saving WDM state to " << path << "..." << std::endl;
        bwcli::check(bw_cyclic_write_wdm(ctx, path));
        std::cout << "Saved " << info.seq_len << " sequence elements to " << path << std::endl;
        bw_cyclic_close(ctx);
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "cuprym_cyclic error: " << e.what() << std::endl;
        return 1;
    }
}
