// recon_tomo: slice-by-slice tomography (vertical rotation axis) driven by a
// TOML config, the drop-in for the reference's recon_tomo executable
// (src/mbir2d.cpp:92-208).
//
//   recon_tomo config.toml            reconstruct and write [output]
//   recon_tomo --dry-run config.toml  parse, load and prepare only, print a JSON summary
//   recon_tomo                        write config_template.toml, exit 1
//
// The projections of all datasets are stacked, normalised by their maximum
// and reordered to a sinogram {nrows, nproj, ncols} (prepare_sinogram,
// include/mbir2d_prep.h:44-65); every detector row is one slice, solved by
// lc_mbir2d (gpu::MBIR2D, src/gpu/mbir2d.cu:36-85) on GPU 0.
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
        config::dump_template(config::kTomoTemplate, "config_template.toml");
        return 1;
    }
    const toml::Table cfg = toml::parse_file(cfg_path);
    auto datasets = config::parse_input_datasets(cfg, config::parent_dir(cfg_path));
    const config::ReconParams params = config::parse_recon_params(cfg);
    const config::OutputParams output = config::parse_output_params(cfg);
    if (datasets.empty()) throw std::runtime_error("recon_tomo: no [[input]] datasets found");
    const int *rd = params.recon_dims;
    if (rd[1] != rd[2])
        throw std::runtime_error("recon_tomo: recon_dims must be square in-plane (n2 == n3), got [" +
                                 std::to_string(rd[0]) + ", " + std::to_string(rd[1]) + ", " +
                                 std::to_string(rd[2]) + "]");
    const double eps = 1e-6;
    for (size_t j = 0; j < datasets.size(); ++j) {
        if (std::abs(datasets[j].gamma) > eps || std::abs(datasets[j].beta) > eps)
            throw std::runtime_error("recon_tomo: dataset " + std::to_string(j) +
                                     " has a non-zero gamma or beta; this executable only supports "
                                     "vertical-axis tomography. Use recon_lamino for laminography.");
        for (float s : datasets[j].shifts)
            if (std::abs(s) > eps) {
                std::cerr << "Warning: dataset " << j << " has non-zero per-projection shifts; "
                          << "recon_tomo does not support centre-of-rotation shifts and ignores them.\n";
                break;
            }
    }

    // prepare_sinogram: stack, normalise by the global maximum, {p, r, c} -> {r, p, c}
    const size_t nrows = datasets[0].projs.n2, ncols = datasets[0].projs.n3;
    std::vector<float> stacked;
    std::vector<double> theta;
    for (auto &d : datasets) {
        if (d.projs.n2 != nrows || d.projs.n3 != ncols)
            throw std::runtime_error("recon_tomo: all datasets must have the same detector size");
        stacked.insert(stacked.end(), d.projs.data.begin(), d.projs.data.end());
        theta.insert(theta.end(), d.angles.begin(), d.angles.end());
    }
    const size_t nproj = theta.size();
    float mx = -INFINITY;
    for (float v : stacked) mx = std::max(mx, v);
    if (mx > 0)
        for (float &v : stacked) v /= mx;
    std::vector<float> sino(stacked.size());
    for (size_t p = 0; p < nproj; ++p)
        for (size_t r = 0; r < nrows; ++r)
            std::memcpy(&sino[(r * nproj + p) * ncols], &stacked[(p * nrows + r) * ncols],
                        ncols * sizeof(float));
    if ((size_t)rd[0] != nrows)
        throw std::runtime_error("recon_tomo: recon_dims[0] = " + std::to_string(rd[0]) +
                                 " must equal the detector row count " + std::to_string(nrows) +
                                 " (after odd trimming): every row is one slice");

    if (dry) {
        double sum = 0.0;
        for (float v : sino) sum += v;
        std::printf("{\"driver\": \"recon_tomo\", \"datasets\": %zu, \"sinogram\": [%zu, %zu, %zu], "
                    "\"sum\": %.9g, \"max_before\": %.9g, \"theta0\": %.17g, \"theta_last\": %.17g, "
                    "\"recon_dims\": [%d, %d, %d], \"method\": %d, \"max_iters\": %d, "
                    "\"output\": \"%s\"}\n",
                    datasets.size(), nrows, nproj, ncols, sum, (double)mx, theta.front(), theta.back(),
                    rd[0], rd[1], rd[2], params.method, params.max_iters, output.filepath.c_str());
        return 0;
    }

    config::print_params(params);
    std::cout << std::endl << "Running reconstruction on GPU...\n";
    lc_context ctx = nullptr;
    if (lc_context_create(0, nullptr, &ctx) != LC_OK)
        throw std::runtime_error("recon_tomo: no usable CUDA device (there is no CPU fallback)");
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
    recon.n1 = rd[0];
    recon.n2 = rd[1];
    recon.n3 = rd[2];
    recon.data.resize(recon.size());
    lc_solver_stats st{};
    const auto t0 = std::chrono::steady_clock::now();
    const int rc = lc_mbir2d(ctx, sino.data(), (int)nrows, (int)nproj, (int)ncols, theta.data(), rd, &rp,
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
        std::cerr << "recon_tomo: " << e.what() << "\n";
        return 2;
    }
}
