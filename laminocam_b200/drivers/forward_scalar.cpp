// forward_scalar: synthetic laminography projections of a volume, driven by
// a TOML config, the drop-in for the reference's forward_scalar executable
// (src/radon.cpp).
//
//   forward_scalar config.toml            project and write the files
//   forward_scalar --dry-run config.toml  parse and load only, print a JSON summary
//
// Config keys (src/radon.cpp:49-131):
//   [input]  filename = "volume.tiff"      (float32 multi-page TIFF, or .npy)
//   [output] basedir = "out", pad_factor = 1.0,
//            proj_angles = { min = -90, max = 90, n = 180 }   (degrees, [min, max))
//   [[projections]] gamma = 0, filename = "gamma0.tiff"        (one file per entry)
// and, here only, [output] nufft_tol (default 1e-6; the reference's float CPU
// path runs FINUFFT at 5e-4, include/finufft_plan.h:71).
//
// As the reference: the angles are min + i (max - min) / n in float and go to
// basedir/angles.txt in degrees; with pad_factor > 1 every axis of the volume
// is zero-padded, centred, to int(n pad_factor) forced odd (include/padding.h
// pad3d, PadType::SYMMETRIC); each [[projections]] entry (tilt gamma in
// degrees, beta = 0) is projected onto the padded detector by the forward
// operator (lc_forward3d, tomocam::forward) and each projection is cropped,
// centred, back to the volume's rows and columns (crop2d, SYMMETRIC).  The
// projections run on GPU 0.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <string>
#include <sys/stat.h>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/laminocam.h"
#include "lc_io.hpp"
#include "lc_toml.hpp"

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

std::string parent_dir(const std::string &path) {
    const size_t k = path.find_last_of('/');
    return k == std::string::npos ? std::string() : path.substr(0, k + 1);
}

std::string join(const std::string &dir, const std::string &name) {
    if (name.empty() || name[0] == '/' || dir.empty()) return name;
    return dir.back() == '/' ? dir + name : dir + "/" + name;
}

bool ends_with(const std::string &s, const std::string &t) {
    return s.size() >= t.size() && s.compare(s.size() - t.size(), t.size(), t) == 0;
}

double number_or(const toml::Table *t, const std::string &key, double dflt) {
    if (!t) return dflt;
    const toml::Value *v = toml::find(*t, key);
    if (!v) return dflt;
    if (!v->is_number()) throw std::runtime_error("forward_scalar: '" + key + "' must be a number");
    return v->number();
}

std::string string_or(const toml::Table *t, const std::string &key, const std::string &dflt) {
    if (!t) return dflt;
    const toml::Value *v = toml::find(*t, key);
    if (!v) return dflt;
    if (!v->is_string()) throw std::runtime_error("forward_scalar: '" + key + "' must be a string");
    return v->s;
}

// int(n * pad), forced odd (src/radon.cpp:135-142)
size_t padded(size_t n, float pad) {
    size_t m = (size_t)((float)n * pad);
    if (m % 2 == 0) m -= 1;
    return m;
}

void check(lc_context ctx, int rc, const char *what) {
    if (rc) throw std::runtime_error(std::string("forward_scalar: ") + what + ": " + lc_last_error(ctx));
}

void cuda_check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("forward_scalar: ") + what + ": " + cudaGetErrorString(e));
}

struct Projection {
    float gamma;
    std::string filename;
};

int run(int argc, char **argv) {
    bool dry = false;
    std::string cfg_path;
    for (int k = 1; k < argc; ++k) {
        if (std::strcmp(argv[k], "--dry-run") == 0) dry = true;
        else cfg_path = argv[k];
    }
    if (cfg_path.empty()) {
        std::cerr << "Usage: " << argv[0] << " [--dry-run] <input.toml>\n";
        return 1;
    }
    const toml::Table cfg = toml::parse_file(cfg_path);
    const toml::Table *input = toml::find_table(cfg, "input");
    const toml::Table *output = toml::find_table(cfg, "output");
    if (!input || !output)
        throw std::runtime_error("forward_scalar: input and output sections are required in the TOML file");
    const std::string base = parent_dir(cfg_path);
    const std::string in_file = join(base, string_or(input, "filename", ""));
    {
        std::ifstream probe(in_file);
        if (!probe) throw std::runtime_error("forward_scalar: input file " + in_file + " does not exist");
    }
    io::Volume vol = ends_with(in_file, ".npy") ? io::read_npy(in_file) : io::read_tiff(in_file);
    const std::string outdir = join(base, string_or(output, "basedir", "."));
    const float pad = (float)number_or(output, "pad_factor", 1.0);
    const double tol = number_or(output, "nufft_tol", 1e-6);
    const toml::Table *ang = toml::find_table(*output, "proj_angles");
    const float amin = (float)number_or(ang, "min", -90.0), amax = (float)number_or(ang, "max", 90.0);
    const int an = (int)number_or(ang, "n", 180);
    if (an <= 0) throw std::runtime_error("forward_scalar: proj_angles.n must be positive");
    const float astep = (amax - amin) / (float)an;
    std::vector<float> angles(an);
    for (int i = 0; i < an; ++i) angles[i] = amin + (float)i * astep;
    std::vector<Projection> projs;
    if (const toml::Value *arr = toml::find(cfg, "projections"); arr && arr->is_array()) {
        for (const toml::Value &e : *arr->arr) {
            if (!e.is_table()) continue;
            const toml::Value *g = toml::find(*e.tbl, "gamma"), *f = toml::find(*e.tbl, "filename");
            if (g && f && g->is_number() && f->is_string()) projs.push_back({(float)g->number(), f->s});
        }
    }
    if (projs.empty()) projs.push_back({0.0f, "proj.tiff"});

    // the padded volume (centred zero padding of every axis)
    const size_t n1 = vol.n1, n2 = vol.n2, n3 = vol.n3;
    size_t p1 = n1, p2 = n2, p3 = n3;
    if (pad > 1.0f) {
        p1 = padded(n1, pad);
        p2 = padded(n2, pad);
        p3 = padded(n3, pad);
        if (p1 < n1 || p2 < n2 || p3 < n3)
            throw std::runtime_error("forward_scalar: pad_factor too small for the volume's sizes");
    }

    if (dry) {
        double sum = 0.0;
        for (float v : vol.data) sum += v;
        std::printf("{\"driver\": \"forward_scalar\", \"volume\": [%zu, %zu, %zu], \"sum\": %.9g, "
                    "\"padded\": [%zu, %zu, %zu], \"angles\": %d, \"angle0\": %.9g, \"angle_last\": %.9g, "
                    "\"nufft_tol\": %.3g, \"projections\": [",
                    n1, n2, n3, sum, p1, p2, p3, an, angles[0], angles[an - 1], tol);
        for (size_t k = 0; k < projs.size(); ++k)
            std::printf("%s{\"gamma\": %.9g, \"file\": \"%s\"}", k ? ", " : "", projs[k].gamma,
                        join(outdir, projs[k].filename).c_str());
        std::printf("]}\n");
        return 0;
    }

    mkdir_p(outdir);
    {
        std::ofstream out(join(outdir, "angles.txt"));
        for (float a : angles) out << a << "\n";
    }
    std::vector<float> vp(p1 * p2 * p3, 0.0f);
    const size_t o1 = (p1 - n1) / 2, o2 = (p2 - n2) / 2, o3 = (p3 - n3) / 2;
    for (size_t i = 0; i < n1; ++i)
        for (size_t j = 0; j < n2; ++j)
            std::memcpy(&vp[((i + o1) * p2 + j + o2) * p3 + o3], &vol.data[(i * n2 + j) * n3], n3 * sizeof(float));

    lc_context ctx = nullptr;
    if (lc_context_create(0, nullptr, &ctx)) throw std::runtime_error("forward_scalar: no CUDA device");
    float *dvol = nullptr, *dproj = nullptr;
    const size_t nproj = (size_t)an * p2 * p3;
    try {
        cuda_check(cudaMalloc((void **)&dvol, vp.size() * sizeof(float)), "device volume");
        cuda_check(cudaMalloc((void **)&dproj, nproj * sizeof(float)), "device projections");
        cuda_check(cudaMemcpy(dvol, vp.data(), vp.size() * sizeof(float), cudaMemcpyHostToDevice), "upload");
        std::vector<double> theta(an), beta(an, 0.0), gamma(an);
        for (int i = 0; i < an; ++i) theta[i] = (double)(angles[i] * (float)M_PI / 180.0f);
        std::vector<float> hp(nproj);
        int idx = 0;
        for (const Projection &pr : projs) {
            ++idx;
            const std::string file = join(outdir, pr.filename);
            std::printf("[%d/%zu] gamma=%.2f deg -> %s\n", idx, projs.size(), pr.gamma, file.c_str());
            const double g = (double)(pr.gamma * (float)M_PI / 180.0f);
            for (int i = 0; i < an; ++i) gamma[i] = g;
            lc_geometry geo = nullptr;
            check(ctx, lc_geometry3d_create(ctx, theta.data(), gamma.data(), beta.data(), nullptr, an, (int)p2,
                                            (int)p3, &geo),
                  "geometry");
            const int rc = lc_forward3d(ctx, geo, dvol, (int)p1, (int)p2, (int)p3, dproj, tol);
            lc_geometry_destroy(geo);
            check(ctx, rc, "forward projection");
            cuda_check(cudaMemcpy(hp.data(), dproj, nproj * sizeof(float), cudaMemcpyDeviceToHost), "download");
            // crop each projection back to the volume's rows and columns
            io::Volume out;
            out.n1 = an;
            out.n2 = n2;
            out.n3 = n3;
            out.data.resize(out.size());
            const size_t c2 = (p2 - n2) / 2, c3 = (p3 - n3) / 2;
            for (int i = 0; i < an; ++i)
                for (size_t j = 0; j < n2; ++j)
                    std::memcpy(&out.data[((size_t)i * n2 + j) * n3], &hp[((size_t)i * p2 + j + c2) * p3 + c3],
                                n3 * sizeof(float));
            mkdir_p(parent_dir(file));
            io::write_tiff(file, out);
        }
    } catch (...) {
        cudaFree(dvol);
        cudaFree(dproj);
        lc_context_destroy(ctx);
        throw;
    }
    cudaFree(dvol);
    cudaFree(dproj);
    lc_context_destroy(ctx);
    std::printf("Done.\n");
    return 0;
}

}  // namespace

int main(int argc, char **argv) {
    try {
        return run(argc, argv);
    } catch (const std::exception &e) {
        std::cerr << e.what() << "\n";
        return 1;
    }
}
