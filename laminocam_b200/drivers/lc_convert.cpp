// lc_convert: converts float32 arrays between multi-page TIFF and .npy.
//
//   lc_convert in.npy out.tiff
//   lc_convert [--no-trim] in.tiff out.npy
//
// HDF5 input is not available in this build, so projections stored in HDF5
// are converted (elsewhere) to .npy or TIFF, and this tool moves them between
// the two.  Reading a TIFF drops the last row and column of even-sized pages
// like the drivers do, unless --no-trim is given.
#include <cstring>
#include <iostream>
#include <string>

#include "lc_io.hpp"

using namespace lc;

static bool ends_with(const std::string &s, const std::string &e) {
    return s.size() >= e.size() && s.compare(s.size() - e.size(), e.size(), e) == 0;
}

static bool is_tiff(const std::string &p) { return ends_with(p, ".tif") || ends_with(p, ".tiff"); }

int main(int argc, char **argv) {
    bool trim = true;
    std::string in, out;
    for (int k = 1; k < argc; ++k) {
        if (std::strcmp(argv[k], "--no-trim") == 0) trim = false;
        else if (in.empty()) in = argv[k];
        else out = argv[k];
    }
    if (in.empty() || out.empty()) {
        std::cerr << "usage: " << argv[0] << " [--no-trim] <in.npy|in.tiff> <out.npy|out.tiff>\n";
        return 1;
    }
    try {
        io::Volume v = is_tiff(in) ? io::read_tiff(in, trim) : io::read_npy(in);
        if (is_tiff(out)) io::write_tiff(out, v);
        else io::write_npy(out, v);
        std::cout << v.n1 << " " << v.n2 << " " << v.n3 << "\n";
    } catch (const std::exception &e) {
        std::cerr << "lc_convert: " << e.what() << "\n";
        return 2;
    }
    return 0;
}
