// Config files of the recon_lamino / recon_tomo drivers: the reference's
// parse_input_datasets, parse_recon_params and parse_output_params
// (include/config.h:160-460) over the TOML subset parser and the array
// readers of this directory.  Same keys, defaults, unit conventions and
// error cases; HDF5 input is replaced by .npy (see lc_io.hpp).
#pragma once

#include <string>
#include <vector>

#include "lc_io.hpp"
#include "lc_toml.hpp"

namespace lc::config {

struct Dataset {
    io::Volume projs;             // {ntheta, nrows, ncols}, NaN/Inf set to 0
    std::vector<double> angles;   // radians
    double gamma = 0.0;           // radians, negated from the TOML degrees (include/config.h:206)
    double beta = 0.0;            // radians
    std::vector<float> shifts;    // (dx, dy) per projection, pixels
};

struct ReconParams {
    int max_iters = 50;
    float tol = 1e-5f, xtol = 1e-5f;
    int recon_dims[3] = {0, 0, 0};  // forced odd
    int method = 0;                 // 0 unconstrained CG, 1 Split-Bregman
    float lambda = 0.1f, mu = 10.0f;
    int inner_iters = 1;
    // accepted for compatibility; the single-GPU build has no streamed path
    int num_gpus = 0, chunk_slices = 0;
    bool streamed = false;
};

struct OutputParams {
    std::string filepath = "./recon.tiff";
    std::vector<std::string> formats{"tiff"};
    bool has(const std::string &f) const;
};

std::vector<Dataset> parse_input_datasets(const toml::Table &cfg, const std::string &base_dir);
ReconParams parse_recon_params(const toml::Table &cfg);
OutputParams parse_output_params(const toml::Table &cfg);

// resolves a relative path against the config file's directory when the
// file exists there (include/config.h:62-70)
std::string resolve_path(const std::string &p, const std::string &base_dir);
std::string parent_dir(const std::string &path);

// the reference's thickness warning for laminography (include/config.h:405-418)
void warn_laminography_dims(const ReconParams &p);
void print_params(const ReconParams &p);

extern const char *kLaminoTemplate;
extern const char *kTomoTemplate;
void dump_template(const char *tmpl, const std::string &path);

}  // namespace lc::config
