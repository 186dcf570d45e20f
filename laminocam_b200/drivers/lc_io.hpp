// Array files for the reconstruction drivers: float32 multi-page TIFF and
// NumPy .npy.
//
// TIFF follows the reference's tomocam::tiff::read / write
// (include/tiff.h:29-113, built on libtiff, which is not available here):
// pages are the slowest dimension; reading drops the last row and column of
// even-sized pages so that both sizes are odd (include/tiff.h:51-53); writing
// produces uncompressed little-endian IEEE float32 pages of one strip each.
// The reader accepts either byte order, any strip layout and 8/16/32-bit
// unsigned integer or 32/64-bit float samples (converted to float32), without
// compression.  The reference reads projections from HDF5 as its second
// format (include/hdfread.h); HDF5 is not available here, so .npy (float32 or
// float64, C order, 1D to 3D) stands in for it, read without the odd trim
// like the HDF5 path (include/hdfread.h:57).
#pragma once

#include <cstddef>
#include <string>
#include <vector>

namespace lc::io {

struct Volume {
    size_t n1 = 0, n2 = 0, n3 = 0;  // pages (or slices), rows, columns
    std::vector<float> data;         // row-major {n1, n2, n3}
    size_t size() const { return n1 * n2 * n3; }
};

Volume read_tiff(const std::string &path, bool trim_to_odd = true);
void write_tiff(const std::string &path, const Volume &v);

Volume read_npy(const std::string &path);
void write_npy(const std::string &path, const Volume &v);

// one number per line (whitespace separated)
std::vector<double> read_numbers(const std::string &path);

}  // namespace lc::io
