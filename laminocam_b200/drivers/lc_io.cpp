// float32 TIFF and .npy readers and writers (see lc_io.hpp).
#include "lc_io.hpp"

#include <cstdint>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace lc::io {
namespace {

std::vector<unsigned char> slurp(const std::string &path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot open " + path);
    return std::vector<unsigned char>((std::istreambuf_iterator<char>(f)),
                                      std::istreambuf_iterator<char>());
}

struct Reader {
    const std::vector<unsigned char> &b;
    bool big;
    std::string path;
    void need(size_t off, size_t n) const {
        if (off + n > b.size()) throw std::runtime_error(path + ": truncated TIFF");
    }
    uint16_t u16(size_t off) const {
        need(off, 2);
        return big ? (uint16_t)(b[off] << 8 | b[off + 1]) : (uint16_t)(b[off] | b[off + 1] << 8);
    }
    uint32_t u32(size_t off) const {
        need(off, 4);
        uint32_t v = 0;
        for (int k = 0; k < 4; ++k) v |= (uint32_t)b[off + (big ? 3 - k : k)] << (8 * k);
        return v;
    }
    uint64_t u64(size_t off) const {
        return big ? ((uint64_t)u32(off) << 32 | u32(off + 4)) : ((uint64_t)u32(off + 4) << 32 | u32(off));
    }
};

struct Ifd {
    uint32_t width = 0, height = 0, bits = 0, format = 1, spp = 1, compression = 1, planar = 1;
    uint32_t rows_per_strip = 0xffffffffu;
    std::vector<uint64_t> offsets, counts;
};

// values of one directory entry (SHORT or LONG, any count)
std::vector<uint64_t> entry_values(const Reader &r, size_t e) {
    const uint16_t type = r.u16(e + 2);
    const uint32_t count = r.u32(e + 4);
    const size_t sz = type == 3 ? 2 : (type == 4 ? 4 : (type == 16 ? 8 : 0));
    if (sz == 0) return {};
    const size_t total = sz * count;
    const size_t at = total <= 4 ? e + 8 : r.u32(e + 8);
    std::vector<uint64_t> v(count);
    for (uint32_t k = 0; k < count; ++k)
        v[k] = type == 3 ? r.u16(at + 2 * k) : (type == 4 ? r.u32(at + 4 * k) : r.u64(at + 8 * k));
    return v;
}

float sample(const Reader &r, const Ifd &d, size_t off) {
    if (d.format == 3) {
        if (d.bits == 32) {
            uint32_t u = r.u32(off);
            float f;
            std::memcpy(&f, &u, 4);
            return f;
        }
        uint64_t u = r.u64(off);
        double x;
        std::memcpy(&x, &u, 8);
        return (float)x;
    }
    if (d.bits == 8) return (float)r.b[off];
    if (d.bits == 16) return (float)r.u16(off);
    return (float)r.u32(off);
}

}  // namespace

Volume read_tiff(const std::string &path, bool trim_to_odd) {
    const std::vector<unsigned char> bytes = slurp(path);
    if (bytes.size() < 8) throw std::runtime_error(path + ": not a TIFF file");
    Reader r{bytes, bytes[0] == 'M', path};
    if (!((bytes[0] == 'I' && bytes[1] == 'I') || (bytes[0] == 'M' && bytes[1] == 'M')) ||
        r.u16(2) != 42)
        throw std::runtime_error(path + ": not a classic TIFF file");
    std::vector<Ifd> pages;
    uint64_t next = r.u32(4);
    while (next) {
        if (pages.size() > (1u << 20)) throw std::runtime_error(path + ": directory loop");
        const size_t n = r.u16(next);
        Ifd d;
        for (size_t k = 0; k < n; ++k) {
            const size_t e = next + 2 + 12 * k;
            const uint16_t tag = r.u16(e);
            auto v = entry_values(r, e);
            if (v.empty()) continue;
            switch (tag) {
                case 256: d.width = (uint32_t)v[0]; break;
                case 257: d.height = (uint32_t)v[0]; break;
                case 258: d.bits = (uint32_t)v[0]; break;
                case 259: d.compression = (uint32_t)v[0]; break;
                case 273: d.offsets = v; break;
                case 277: d.spp = (uint32_t)v[0]; break;
                case 278: d.rows_per_strip = (uint32_t)v[0]; break;
                case 279: d.counts = v; break;
                case 284: d.planar = (uint32_t)v[0]; break;
                case 339: d.format = (uint32_t)v[0]; break;
                default: break;
            }
        }
        if (d.compression != 1) throw std::runtime_error(path + ": compressed TIFF is not supported");
        if (d.spp != 1) throw std::runtime_error(path + ": only one sample per pixel is supported");
        if (d.offsets.empty()) throw std::runtime_error(path + ": tiled TIFF is not supported");
        const bool fmt_ok = (d.format == 3 && (d.bits == 32 || d.bits == 64)) ||
                            ((d.format == 1 || d.format == 0) && (d.bits == 8 || d.bits == 16 || d.bits == 32));
        if (!fmt_ok) throw std::runtime_error(path + ": unsupported sample format");
        pages.push_back(d);
        next = r.u32(next + 2 + 12 * n);
    }
    if (pages.empty()) throw std::runtime_error(path + ": no pages");
    const Ifd &p0 = pages[0];
    for (auto &p : pages)
        if (p.width != p0.width || p.height != p0.height)
            throw std::runtime_error(path + ": pages of different sizes");
    Volume v;
    v.n1 = pages.size();
    v.n2 = p0.height;
    v.n3 = p0.width;
    if (trim_to_odd) {
        if (v.n2 % 2 == 0) v.n2 -= 1;
        if (v.n3 % 2 == 0) v.n3 -= 1;
    }
    v.data.resize(v.size());
    const size_t bps = p0.bits / 8;
    for (size_t i = 0; i < pages.size(); ++i) {
        const Ifd &d = pages[i];
        const uint32_t rps = std::min<uint32_t>(d.rows_per_strip, d.height);
        for (size_t j = 0; j < v.n2; ++j) {
            const size_t strip = j / rps;
            if (strip >= d.offsets.size()) throw std::runtime_error(path + ": missing strip");
            const size_t row_off = d.offsets[strip] + (j % rps) * (size_t)d.width * bps;
            r.need(row_off, (size_t)d.width * bps);
            float *dst = v.data.data() + (i * v.n2 + j) * v.n3;
            for (size_t k = 0; k < v.n3; ++k) dst[k] = sample(r, d, row_off + k * bps);
        }
    }
    return v;
}

void write_tiff(const std::string &path, const Volume &v) {
    std::ofstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot write " + path);
    auto put16 = [&](uint16_t x) { f.write((const char *)&x, 2); };
    auto put32 = [&](uint32_t x) { f.write((const char *)&x, 4); };
    f.write("II", 2);
    put16(42);
    put32(8);
    const uint32_t w = (uint32_t)v.n3, h = (uint32_t)v.n2;
    const uint64_t page_bytes = (uint64_t)w * h * 4;
    const int nent = 11;
    const uint64_t ifd_bytes = 2 + 12 * nent + 4;
    for (size_t i = 0; i < v.n1; ++i) {
        const uint64_t ifd_at = (uint64_t)f.tellp();
        const uint64_t data_at = ifd_at + ifd_bytes;
        const uint64_t next = i + 1 < v.n1 ? data_at + page_bytes : 0;
        if (next > 0xffffffffull || data_at + page_bytes > 0xffffffffull)
            throw std::runtime_error(path + ": volume too large for a classic TIFF");
        put16(nent);
        auto entry = [&](uint16_t tag, uint16_t type, uint32_t count, uint32_t value) {
            put16(tag);
            put16(type);
            put32(count);
            if (type == 3 && count == 1) {
                put16((uint16_t)value);
                put16(0);
            } else {
                put32(value);
            }
        };
        entry(256, 4, 1, w);                       // width
        entry(257, 4, 1, h);                       // height
        entry(258, 3, 1, 32);                      // bits per sample
        entry(259, 3, 1, 1);                       // no compression
        entry(262, 3, 1, 1);                       // min-is-black
        entry(273, 4, 1, (uint32_t)data_at);       // strip offset
        entry(274, 3, 1, 1);                       // orientation top-left
        entry(277, 3, 1, 1);                       // samples per pixel
        entry(278, 4, 1, h);                       // rows per strip: one strip
        entry(279, 4, 1, (uint32_t)page_bytes);    // strip byte count
        entry(339, 3, 1, 3);                       // IEEE float samples
        put32((uint32_t)next);
        f.write((const char *)(v.data.data() + i * (size_t)w * h), (std::streamsize)page_bytes);
    }
    if (!f) throw std::runtime_error("failed writing " + path);
}

Volume read_npy(const std::string &path) {
    const std::vector<unsigned char> b = slurp(path);
    if (b.size() < 10 || std::memcmp(b.data(), "\x93NUMPY", 6) != 0)
        throw std::runtime_error(path + ": not a .npy file");
    const int major = b[6];
    size_t hlen, hstart;
    if (major == 1) {
        hlen = b[8] | b[9] << 8;
        hstart = 10;
    } else {
        if (b.size() < 12) throw std::runtime_error(path + ": truncated .npy");
        hlen = b[8] | b[9] << 8 | b[10] << 16 | (size_t)b[11] << 24;
        hstart = 12;
    }
    if (hstart + hlen > b.size()) throw std::runtime_error(path + ": truncated .npy");
    const std::string h(b.begin() + hstart, b.begin() + hstart + hlen);
    auto field = [&](const std::string &key) {
        size_t at = h.find("'" + key + "'");
        if (at == std::string::npos) throw std::runtime_error(path + ": .npy header lacks " + key);
        return at + key.size() + 2;
    };
    size_t d = h.find('\'', h.find(':', field("descr")));
    const std::string descr = h.substr(d + 1, h.find('\'', d + 1) - d - 1);
    const bool fortran = h.find("True", field("fortran_order")) < h.find(',', field("fortran_order"));
    if (fortran) throw std::runtime_error(path + ": Fortran-ordered .npy is not supported");
    size_t s0 = h.find('(', field("shape")), s1 = h.find(')', s0);
    std::vector<size_t> shape;
    std::stringstream ss(h.substr(s0 + 1, s1 - s0 - 1));
    std::string tok;
    while (std::getline(ss, tok, ','))
        if (tok.find_first_not_of(" ") != std::string::npos) shape.push_back(std::stoull(tok));
    if (shape.empty() || shape.size() > 3)
        throw std::runtime_error(path + ": .npy array must be 1D, 2D or 3D");
    while (shape.size() < 3) shape.insert(shape.begin(), 1);
    Volume v;
    v.n1 = shape[0];
    v.n2 = shape[1];
    v.n3 = shape[2];
    v.data.resize(v.size());
    const unsigned char *src = b.data() + hstart + hlen;
    const size_t avail = b.size() - hstart - hlen;
    if (descr == "<f4") {
        if (avail < v.size() * 4) throw std::runtime_error(path + ": truncated .npy data");
        std::memcpy(v.data.data(), src, v.size() * 4);
    } else if (descr == "<f8") {
        if (avail < v.size() * 8) throw std::runtime_error(path + ": truncated .npy data");
        for (size_t k = 0; k < v.size(); ++k) {
            double x;
            std::memcpy(&x, src + 8 * k, 8);
            v.data[k] = (float)x;
        }
    } else {
        throw std::runtime_error(path + ": .npy dtype must be <f4 or <f8, got " + descr);
    }
    return v;
}

void write_npy(const std::string &path, const Volume &v) {
    std::string h = "{'descr': '<f4', 'fortran_order': False, 'shape': (" + std::to_string(v.n1) +
                    ", " + std::to_string(v.n2) + ", " + std::to_string(v.n3) + "), }";
    while ((10 + h.size() + 1) % 64) h += ' ';
    h += '\n';
    std::ofstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot write " + path);
    f.write("\x93NUMPY\x01\x00", 8);
    const uint16_t hl = (uint16_t)h.size();
    f.write((const char *)&hl, 2);
    f.write(h.data(), (std::streamsize)h.size());
    f.write((const char *)v.data.data(), (std::streamsize)(v.size() * 4));
    if (!f) throw std::runtime_error("failed writing " + path);
}

std::vector<double> read_numbers(const std::string &path) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot open " + path);
    std::vector<double> out;
    double x;
    while (f >> x) out.push_back(x);
    return out;
}

}  // namespace lc::io
