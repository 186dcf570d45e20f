// Config parsing for the drivers (see lc_config.hpp).
#include "lc_config.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <sys/stat.h>

namespace lc::config {
namespace {

const double kPi = 3.14159265358979323846;

bool exists(const std::string &p) {
    struct stat st;
    return ::stat(p.c_str(), &st) == 0;
}

std::string lower_ext(const std::string &p) {
    const size_t slash = p.find_last_of('/');
    const size_t dot = p.find_last_of('.');
    if (dot == std::string::npos || (slash != std::string::npos && dot < slash)) return "";
    std::string e = p.substr(dot);
    std::transform(e.begin(), e.end(), e.begin(), ::tolower);
    return e;
}

void warn_unknown_keys(const toml::Table &t, std::initializer_list<const char *> allowed,
                       const std::string &section) {
    for (auto &kv : t) {
        bool known = false;
        for (const char *a : allowed) known = known || kv.first == a;
        if (!known)
            std::cerr << "Warning: unknown key '" << kv.first << "' in " << section << " (ignored)\n";
    }
}

double num(const toml::Table &t, const char *key, double dflt, const std::string &where) {
    const toml::Value *v = toml::find(t, key);
    if (!v) return dflt;
    if (!v->is_number()) throw std::runtime_error(where + " '" + key + "' must be a number");
    return v->number();
}

std::string str(const toml::Table &t, const char *key, const std::string &dflt,
                const std::string &where) {
    const toml::Value *v = toml::find(t, key);
    if (!v) return dflt;
    if (!v->is_string()) throw std::runtime_error(where + " '" + key + "' must be a string");
    return v->s;
}

void to_radians(std::vector<double> &a, const std::string &units) {
    if (units == "deg") {
        for (double &x : a) x = x * kPi / 180.0;
    } else if (units != "rad") {
        throw std::runtime_error("[[input]] 'angle_units' must be \"deg\" or \"rad\", got '" + units + "'");
    }
}

std::vector<double> read_angles(const std::string &path, const std::string &units) {
    std::vector<double> a;
    if (lower_ext(path) == ".npy") {
        io::Volume v = io::read_npy(path);
        a.assign(v.data.begin(), v.data.end());
    } else {
        a = io::read_numbers(path);
    }
    if (a.empty()) throw std::runtime_error("No angles found in file: " + path);
    to_radians(a, units);
    return a;
}

std::vector<float> read_shifts(const std::string &path) {
    std::vector<double> n = io::read_numbers(path);
    if (n.empty()) throw std::runtime_error("No shifts found in file: " + path);
    n.resize(n.size() - n.size() % 2);
    return std::vector<float>(n.begin(), n.end());
}

}  // namespace

bool OutputParams::has(const std::string &f) const {
    return std::find(formats.begin(), formats.end(), f) != formats.end();
}

std::string parent_dir(const std::string &path) {
    const size_t s = path.find_last_of('/');
    return s == std::string::npos ? std::string() : path.substr(0, s);
}

std::string resolve_path(const std::string &p, const std::string &base_dir) {
    if (!p.empty() && p[0] != '/' && !base_dir.empty()) {
        const std::string cand = base_dir + "/" + p;
        if (exists(cand)) return cand;
    }
    return p;
}

std::vector<Dataset> parse_input_datasets(const toml::Table &cfg, const std::string &base_dir) {
    const toml::Value *inputs = toml::find(cfg, "input");
    if (!inputs || !inputs->is_array()) throw std::runtime_error("Missing [[input]] array in TOML file");
    std::vector<Dataset> out;
    for (const toml::Value &e : *inputs->arr) {
        if (!e.is_table()) throw std::runtime_error("Invalid [[input]] entry");
        const toml::Table &in = *e.tbl;
        if (!toml::find(in, "filename")) throw std::runtime_error("[[input]] entry must have a 'filename' field");
        warn_unknown_keys(in, {"filename", "angles", "angle_units", "gamma", "beta", "shifts",
                               "cor-offset", "alignment", "projs_dataset"},
                          "[[input]]");
        const std::string filename = resolve_path(str(in, "filename", "", "[[input]]"), base_dir);
        const std::string units = str(in, "angle_units", "deg", "[[input]]");
        if (!exists(filename)) throw std::runtime_error("Projection file does not exist: " + filename);
        Dataset d;
        d.gamma = -num(in, "gamma", 0.0, "[[input]]") * kPi / 180.0;
        d.beta = num(in, "beta", 0.0, "[[input]]") * kPi / 180.0;

        // 'shifts' (a two-column file) takes priority over the scalar 'cor-offset'
        bool broadcast = false;
        if (toml::find(in, "shifts")) {
            const std::string sp = resolve_path(str(in, "shifts", "", "[[input]]"), base_dir);
            if (!exists(sp)) throw std::runtime_error("Shifts file does not exist: " + sp);
            d.shifts = read_shifts(sp);
        } else if (const toml::Value *co = toml::find(in, "cor-offset")) {
            if (!co->is_array() || co->arr->size() != 2)
                throw std::runtime_error("[[input]] 'cor-offset' must be in form [dx, dy]");
            for (const toml::Value &x : *co->arr) {
                if (!x.is_number()) throw std::runtime_error("[[input]] 'cor-offset' must be an array of numbers");
                d.shifts.push_back((float)x.number());
            }
            broadcast = true;
        }

        const std::string ext = lower_ext(filename);
        if (ext == ".tiff" || ext == ".tif" || ext == ".npy") {
            if (!toml::find(in, "angles"))
                throw std::runtime_error("[[input]] 'angles' is required for TIFF and .npy files");
            const std::string ap = resolve_path(str(in, "angles", "", "[[input]]"), base_dir);
            if (!exists(ap)) throw std::runtime_error("Angles file does not exist: " + ap);
            d.projs = ext == ".npy" ? io::read_npy(filename) : io::read_tiff(filename);
            d.angles = read_angles(ap, units);
            if (d.projs.n1 != d.angles.size())
                throw std::runtime_error("'" + filename + "' has " + std::to_string(d.projs.n1) +
                                         " pages but '" + ap + "' has " +
                                         std::to_string(d.angles.size()) + " entries");
        } else if (ext == ".h5" || ext == ".hdf5") {
            throw std::runtime_error("HDF5 input needs the HDF5 library, which this build does not "
                                     "have: store the projections as .npy (or TIFF) with an angles "
                                     "file instead (" + filename + ")");
        } else {
            throw std::runtime_error("Unsupported file extension '" + ext + "': " + filename);
        }
        for (float &x : d.projs.data)
            if (!std::isfinite(x)) x = 0.0f;  // include/mask.h:43-54

        const size_t n = d.angles.size();
        if (broadcast) {
            const float dx = d.shifts[0], dy = d.shifts[1];
            d.shifts.clear();
            for (size_t k = 0; k < n; ++k) {
                d.shifts.push_back(dx);
                d.shifts.push_back(dy);
            }
        } else if (d.shifts.empty()) {
            d.shifts.assign(2 * n, 0.0f);
        } else if (d.shifts.size() != 2 * n) {
            throw std::runtime_error("shifts file has " + std::to_string(d.shifts.size() / 2) +
                                     " entries but " + std::to_string(n) + " projections were loaded");
        }

        // an alignment TOML overrides angles, shifts, gamma and beta
        if (toml::find(in, "alignment")) {
            const std::string alp = resolve_path(str(in, "alignment", "", "[[input]]"), base_dir);
            if (!exists(alp)) throw std::runtime_error("Alignment file does not exist: " + alp);
            const toml::Table al = toml::parse_file(alp);
            if (const toml::Value *g = toml::find(al, "gamma_deg"))
                if (g->is_number()) d.gamma = -g->number() * kPi / 180.0;
            if (const toml::Value *b = toml::find(al, "beta_deg"))
                if (b->is_number()) d.beta = b->number() * kPi / 180.0;
            const toml::Value *ca = toml::find(al, "corrected_angles_deg");
            if (!ca || !ca->is_array()) throw std::runtime_error("Alignment TOML missing 'corrected_angles_deg'");
            d.angles.clear();
            for (const toml::Value &x : *ca->arr) {
                if (!x.is_number()) throw std::runtime_error("Alignment TOML 'corrected_angles_deg' must hold numbers");
                d.angles.push_back(x.number() * kPi / 180.0);
            }
            if (const toml::Value *sp = toml::find(al, "shifts_px")) {
                if (!sp->is_array()) throw std::runtime_error("Alignment TOML 'shifts_px' must be an array");
                d.shifts.clear();
                for (const toml::Value &pr : *sp->arr) {
                    if (!pr.is_array() || pr.arr->size() < 2 || !(*pr.arr)[0].is_number() ||
                        !(*pr.arr)[1].is_number())
                        throw std::runtime_error("Alignment TOML 'shifts_px' entries must be [dx, dy] pairs");
                    d.shifts.push_back((float)(*pr.arr)[0].number());
                    d.shifts.push_back((float)(*pr.arr)[1].number());
                }
            }
            if (d.shifts.size() != 2 * d.angles.size())
                throw std::runtime_error("Alignment TOML: shifts_px has " + std::to_string(d.shifts.size() / 2) +
                                         " entries but corrected_angles_deg has " +
                                         std::to_string(d.angles.size()));
            if (d.angles.size() != d.projs.n1)
                throw std::runtime_error("Alignment TOML: corrected_angles_deg has " +
                                         std::to_string(d.angles.size()) + " entries but " +
                                         std::to_string(d.projs.n1) + " projections were loaded");
        }
        out.push_back(std::move(d));
    }
    return out;
}

ReconParams parse_recon_params(const toml::Table &cfg) {
    const toml::Table *r = toml::find_table(cfg, "recon_params");
    if (!r) throw std::runtime_error("Missing [recon_params] section in config file");
    const std::string w = "[recon_params]";
    warn_unknown_keys(*r, {"max_iters", "tol", "xtol", "recon_dims", "regularizer", "num_gpus",
                           "chunk_slices", "streamed"},
                      w);
    ReconParams p;
    p.max_iters = (int)num(*r, "max_iters", 50, w);
    const toml::Value *dims = toml::find(*r, "recon_dims");
    if (!dims || !dims->is_array() || dims->arr->size() != 3)
        throw std::runtime_error("[recon_params] 'recon_dims' must be an array of three integers");
    for (int i = 0; i < 3; ++i) {
        const toml::Value &x = (*dims->arr)[i];
        long v = x.kind == toml::Value::INT ? (long)x.i : 0;
        if (v <= 0)
            throw std::runtime_error("[recon_params] 'recon_dims[" + std::to_string(i) +
                                     "]' must be a positive integer");
        if (v % 2 == 0) v -= 1;  // include/config.h:377
        p.recon_dims[i] = (int)v;
    }
    p.tol = (float)num(*r, "tol", 1e-5, w);
    p.xtol = (float)num(*r, "xtol", 1e-5, w);
    p.num_gpus = (int)num(*r, "num_gpus", 0, w);
    p.chunk_slices = (int)num(*r, "chunk_slices", 0, w);
    if (const toml::Value *s = toml::find(*r, "streamed")) p.streamed = s->kind == toml::Value::BOOL && s->b;
    if (const toml::Table *reg = toml::find_table(*r, "regularizer")) {
        warn_unknown_keys(*reg, {"method", "split_bregman"}, "[recon_params.regularizer]");
        const std::string m = str(*reg, "method", "split_bregman", "[recon_params.regularizer]");
        if (m != "split_bregman") throw std::runtime_error("[recon_params] 'regularizer' must be 'split_bregman'");
        p.method = 1;
        const toml::Table *sb = toml::find_table(*reg, "split_bregman");
        if (!sb)
            throw std::runtime_error("Missing [recon_params.regularizer.split_bregman] section in config file");
        const std::string ws = "[recon_params.regularizer.split_bregman]";
        warn_unknown_keys(*sb, {"lambda", "mu", "inner_iters"}, ws);
        p.lambda = (float)num(*sb, "lambda", 0.1, ws);
        p.mu = (float)num(*sb, "mu", 10.0, ws);
        p.inner_iters = (int)num(*sb, "inner_iters", 1, ws);
    }
    return p;
}

OutputParams parse_output_params(const toml::Table &cfg) {
    const toml::Table *o = toml::find_table(cfg, "output");
    if (!o) throw std::runtime_error("Missing [output] section in config file");
    warn_unknown_keys(*o, {"filename", "formats"}, "[output]");
    OutputParams out;
    out.filepath = str(*o, "filename", "./recon.tiff", "[output]");
    if (const toml::Value *f = toml::find(*o, "formats")) {
        if (!f->is_array()) throw std::runtime_error("[output] 'formats' array must contain strings");
        out.formats.clear();
        for (const toml::Value &x : *f->arr) {
            if (!x.is_string()) throw std::runtime_error("[output] 'formats' array must contain strings");
            if (x.s != "tiff" && x.s != "vti")
                throw std::runtime_error("[output] invalid format '" + x.s + "'. Must be 'tiff' or 'vti'");
            if (!out.has(x.s)) out.formats.push_back(x.s);
        }
    }
    return out;
}

void warn_laminography_dims(const ReconParams &p) {
    const float ratio = (float)p.recon_dims[0] / (float)p.recon_dims[2];
    if (ratio > 0.15f) {
        char buf[256];
        std::snprintf(buf, sizeof(buf),
                      "Warning: recon_dims[0] / recon_dims[2] = %.2f > 0.15.\nlaminography thickness "
                      "(recon_dims[0]) is expected to be much smaller than the in-plane dimensions "
                      "(recon_dims[1], recon_dims[2]).\n",
                      ratio);
        std::cerr << buf;
    }
}

void print_params(const ReconParams &p) {
    std::cout << "Reconstruction parameters:\n"
              << "  recon_dims: [" << p.recon_dims[0] << ", " << p.recon_dims[1] << ", "
              << p.recon_dims[2] << "]\n"
              << "  max_iters: " << p.max_iters << "\n  tol: " << p.tol << "\n  xtol: " << p.xtol
              << "\n  regularizer: " << (p.method ? "split_bregman" : "unconstrained") << "\n";
    if (p.method) std::cout << "  lambda: " << p.lambda << "\n  mu: " << p.mu << "\n  inner_iters: " << p.inner_iters << "\n";
}

void dump_template(const char *tmpl, const std::string &path) {
    std::ofstream f(path);
    if (!f) throw std::runtime_error("Could not open file for writing: " + path);
    f << tmpl;
}

const char *kLaminoTemplate = R"(# recon_lamino configuration: laminographic MBIR reconstruction on one GPU.
# Relative paths are looked up next to this file first.

[[input]]
filename = "projections.tiff"    # float32 multi-page TIFF, or .npy {nproj, nrows, ncols}
angles = "angles.txt"            # one rotation angle per projection (text or .npy)
angle_units = "deg"              # "deg" or "rad"
gamma = 0                        # laminographic tilt in degrees
# beta = 0                       # second tilt in degrees
# shifts = "shifts.txt"          # per-projection "dx dy" in pixels
# cor-offset = [0.0, 0.0]        # one (dx, dy) for every projection
# alignment = "alignment.toml"   # corrected_angles_deg, shifts_px, gamma_deg, beta_deg

[output]
filename = "recon.tiff"
formats = ["tiff"]

[recon_params]
max_iters = 50
tol = 1e-5
xtol = 1e-5
recon_dims = [51, 511, 511]      # (thickness, y, x); even sizes become odd

[recon_params.regularizer]       # remove for unconstrained least squares (CG)
method = "split_bregman"

[recon_params.regularizer.split_bregman]
lambda = 0.1
mu = 10.0
inner_iters = 1
)";

const char *kTomoTemplate = R"(# recon_tomo configuration: slice-by-slice tomography (vertical rotation axis).
# Relative paths are looked up next to this file first.

[[input]]
filename = "projections.npy"     # .npy {nproj, nrows, ncols} or a float32 multi-page TIFF
angles = "angles.txt"            # one rotation angle per projection (text or .npy)
angle_units = "deg"              # "deg" or "rad"; gamma and beta must stay 0

[output]
filename = "recon2d.tiff"
formats = ["tiff"]

[recon_params]
max_iters = 50
tol = 1e-5
xtol = 1e-5
recon_dims = [255, 255, 255]     # (slices = detector rows, y, x); y == x; even sizes become odd

[recon_params.regularizer]       # remove for unconstrained least squares (CG)
method = "split_bregman"

[recon_params.regularizer.split_bregman]
lambda = 0.1
mu = 10.0
inner_iters = 1
)";

}  // namespace lc::config
