// Drop-in for the reference's cuprym_deformation_kernel_vectors executable
// (cuda/cuprym_deformation_kernel_vectors.cu:3489-3736): kernel-vector recovery
// for the eliminated operator and its augmented / replacement variants, with
// the same options, defaults, refusals and output files, over the C ABI.
#include "cli_common.hpp"

#include <iostream>

int main(int argc, char** argv) {
    try {
        bwcli::Parser app("CUDA matrix-free deformation Prym-Green kernel-vector recovery (B200 engine)");
        app.positional("instance", "Cyclic Prym fixture/instance JSON");
        app.option({"-f", "--wdm-file"}, "WDM file used for the rank computation", "", true);
        app.option({"-g", "--generators-file"},
                   "Generator file produced by prym-rank --generator; defaults to WDM stem + _generators.txt", "");
        app.option({"--preconditioned-output"},
                   "Output file for kernel candidates in WDM/preconditioned source coordinates", "");
        app.option({"--original-output"}, "Output file for kernel candidates in original source coordinates", "");
        app.option({"--metadata-output"}, "JSON report for certificate, candidate rank, hashes, and provenance", "");
        app.option({"--operator"}, "Production operator: eliminated, augmented, or replacement.", "eliminated");
        app.option({"--dense-file"}, "Dense deformation block JSON for augmented/replacement operators.", "");
        app.option({"--drop-columns"}, "JSON file with two base-sector columns to delete for replacement.", "");
        app.option({"--sector"}, "Cyclic sector/character.", "-1", true);
        app.option({"-d", "--device"}, "Selects a CUDA device to use.", "0");
        app.option({"--rowmix-rounds"}, "Fallback row-mixing rounds when no WDM sidecar exists.", "2");
        app.option({"--rowmix-seed"}, "Fallback row-mixing seed when no WDM sidecar exists.", "10001");
        app.flag({"--validate-rowmix"}, "Run the CUDA square-operator self-validation before recovery.");
        if (!app.parse(argc, argv)) return 0;

        const long long rounds = app.integer("--rowmix-rounds");
        const unsigned long long rseed = app.unsigned_integer("--rowmix-seed");
        if (rounds != 2 || rseed != 10001)
            throw std::runtime_error("The paper pipeline requires --rowmix-rounds 2 --rowmix-seed 10001.");
        const std::string op = app.str("--operator");
        if (op != "eliminated" && op != "augmented" && op != "replacement") {
            std::cerr << "--operator must be one of: eliminated, augmented, replacement." << std::endl;
            return 1;
        }
        const long long sector = app.integer("--sector");
        if (sector < 0) {
            std::cerr << "--sector is required and must be nonnegative." << std::endl;
            return 1;
        }
        const bool deformation = op != "eliminated";
        std::cout << "Loading cyclic Prym instance JSON: " << app.str("instance") << std::endl;
        // the reference validates the eliminated operator only
        bwcli::check(bw_cyclic_recover(app.str("instance").c_str(), op.c_str(), static_cast<uint32_t>(sector),
                                       app.str("--wdm-file").c_str(), app.str("--generators-file").c_str(),
                                       app.str("--preconditioned-output").c_str(), app.str("--original-output").c_str(),
                                       app.str("--metadata-output").c_str(),
                                       deformation ? app.str("--dense-file").c_str() : nullptr,
                                       deformation ? app.str("--drop-columns").c_str() : nullptr, rounds, rseed,
                                       app.has("--rowmix-rounds") ? 1 : 0, app.has("--rowmix-seed") ? 1 : 0,
                                       !deformation && app.on("--validate-rowmix") ? 1 : 0,
                                       static_cast<int>(app.integer("--device"))));
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "cuprym_cyclic_kernel_vectors error: " << e.what() << std::endl;
        return 1;
    }
}
