// recon_lamino: laminographic MBIR reconstruction driven by a TOML config,
// the drop-in for the reference's recon_lamino executable (src/recon.cpp).
//
//   recon_lamino config.toml            reconstruct and write [output]
//   recon_lamino --dry-run config.toml  parse and load only, print a JSON summary
//   recon_lamino                        write config_template.toml, exit 1
//
// The datasets are stacked, normalised, padded, backprojected and solved by
// lc_mbir3d (gpu::MBIR, src/gpu/mbir.cu:41-167) on GPU 0.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "../../include/laminocam.h"
#include "lc_config.hpp"

using namespace lc;

namespace {

void mkdir_p(const std::string &dir) {
    if (dir.empty()) return;
    std::string cur;
    for (size_t k = 0; k <= dir.size(); ++k) {
        if (k == dir.size() || dir[k] == '/') {
            if (!cur.empty()) ::mkdir(cur.c_str(), 0755);
        }
        if (k < dir.size()) cur += dir[k];
    }
}

int run(int argc, char **argv) {
    bool dry = false;
    std::string cfg_path;
    for (int k = 1; k < argc; ++k) {
        if (std::strcmp(argv[k], "--dry-run") == 0) dry = true;
        else cfg_path = argv[k];
    }
    if (cfg_path.empty()) {
        std::cerr << "Usage: " << argv[0] << " [--dry-run] <input.toml>\n"
                  << "Writing an example input file to config_template.toml.\n";
        config::dump_template(config::kLaminoTemplate, "config_template.toml");
        return 1;
    }
    const toml::Table cfg = toml::parse_file(cfg_path);
    auto datasets = config::parse_input_datasets(cfg, config::parent_dir(cfg_path));
    const config::ReconParams params = config::parse_recon_params(cfg);
    config::warn_laminography_dims(params);
    const config::OutputParams output = config::parse_output_params(cfg);
    if (datasets.empty()) throw std::runtime_error("recon_lamino: no [[input]] datasets found");

    // stack the datasets along the projection axis (src/gpu/mbir.cu:62-111)
    const size_t nrows = datasets[0].projs.n2, ncols = datasets[0].projs.n3;
    std::vector<float> projs, shifts;
    std::vector<double> theta, gamma, beta;
    bool any_shift = false;
    for (auto &d : datasets) {
        if (d.projs.n2 != nrows || d.projs.n3 != ncols)
            throw std::runtime_error("recon_lamino: all datasets must have the same detector size");
        projs.insert(projs.end(), d.projs.data.begin(), d.projs.data.end());
        theta.insert(theta.end(), d.angles.begin(), d.angles.end());
        gamma.insert(gamma.end(), d.angles.size(), d.gamma);
        beta.insert(beta.end(), d.angles.size(), d.beta);
        shifts.insert(shifts.end(), d.shifts.begin(), d.shifts.end());
        for (float s : d.shifts) any_shift = any_shift || s != 0.0f;
    }
    const int nproj = (int)theta.size();

    if (dry) {
        double sum = 0.0;
        for (float v : projs) sum += v;
        std::printf("{\"driver\": \"recon_lamino\", \"datasets\": %zu, \"projections\": [%d, %zu, %zu], "
                    "\"sum\": %.9g, \"theta0\": %.17g, \"theta_last\": %.17g, \"gamma\": %.17g, "
                    "\"beta\": %.17g, \"shift0\": [%.9g, %.9g], \"any_shift\": %s, "
                    "\"recon_dims\": [%d, %d, %d], \"method\": %d, \"max_iters\": %d, "
                    "\"tol\": %.9g, \"xtol\": %.9g, \"lambda\": %.9g, \"mu\": %.9g, \"inner_iters\": %d, "
                    "\"output\": \"%s\", \"tiff\": %s}\n",
                    datasets.size(), nproj, nrows, ncols, sum, theta.front(), theta.back(), gamma[0],
                    beta[0], shifts[0], shifts[1], any_shift ? "true" : "false", params.recon_dims[0],
                    params.recon_dims[1], params.recon_dims[2], params.method, params.max_iters,
                    params.tol, params.xtol, params.lambda, params.mu, params.inner_iters,
                    output.filepath.c_str(), output.has("tiff") ? "true" : "false");
        return 0;
    }

    config::print_params(params);
    std::cout << std::endl << "Running reconstruction on GPU...\n";
    lc_context ctx = nullptr;
    if (lc_context_create(0, nullptr, &ctx) != LC_OK)
        throw std::runtime_error("recon_lamino: no usable CUDA device (there is no CPU fallback)");
    lc_recon_params rp;
    lc_recon_params_default(&rp);
    rp.method = params.method;
    rp.solver.max_iters = params.max_iters;
    rp.solver.inner_iters = params.inner_iters;
    rp.solver.tol = params.tol;
    rp.solver.xtol = params.xtol;
    rp.solver.lambda = params.lambda;
    rp.solver.mu = params.mu;
    rp.solver.use_graph = 1;  // replay the iterations as CUDA graphs
    io::Volume recon;
    recon.n1 = params.recon_dims[0];
    recon.n2 = params.recon_dims[1];
    recon.n3 = params.recon_dims[2];
    recon.data.resize(recon.size());
    lc_solver_stats st{};
    const auto t0 = std::chrono::steady_clock::now();
    const int rc = lc_mbir3d(ctx, projs.data(), nproj, (int)nrows, (int)ncols, theta.data(), gamma.data(),
                             beta.data(), any_shift ? shifts.data() : nullptr, params.recon_dims, &rp,
                             recon.data.data(), &st);
    if (rc != LC_OK) {
        std::string msg = lc_last_error(ctx);
        lc_context_destroy(ctx);
        throw std::runtime_error("GPU reconstruction failed: " + msg);
    }
    lc_context_destroy(ctx);
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("Reconstruction completed in %.2f seconds (%d iterations).\n", sec, st.iters);

    mkdir_p(config::parent_dir(output.filepath));
    if (output.has("tiff")) {
        const std::string &f = output.filepath;
        if (f.size() > 4 && f.compare(f.size() - 4, 4, ".npy") == 0) io::write_npy(f, recon);
        else io::write_tiff(f, recon);
        std::cout << "Saved reconstruction to " << f << "\n";
    }
    if (output.has("vti"))
        std::cout << "Note: the 'vti' format is accepted but not written (nor is it by the reference).\n";
    return 0;
}

}  // namespace

int main(int argc, char **argv) {
    try {
        return run(argc, argv);
    } catch (const std::exception &e) {
        std::cerr << "recon_lamino: " << e.what() << "\n";
        return 2;
    }
}
