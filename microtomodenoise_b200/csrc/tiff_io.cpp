// Baseline TIFF sequence IO (see tiff_io.hpp) and its C ABI:
//   inlm_tiff_shape           <- HdCommunication::GetFilelist_And_ImageSequenceDimensions
//                                (Geometry/hdcommunication.cpp:51-104)
//   inlm_tiff_read            <- GetTif_unknowndim_32bit (:106-124),
//                                Get3DTifSequence_32bitPointer (:975-1060),
//                                Custom3DTifReader for one multi-page file (:164-439)
//   inlm_tiff_write_sequence  <- SaveTifSequence_32bit (:1576-1600),
//                                SaveTifSequence_as16bit (:1602-1626) with the
//                                slice writers Save2DTifImage_32bit (:1356-1416)
//                                and Save2DTifImage_as16bit (:1418-1486)
#include "tiff_io.hpp"

#include <dirent.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <mutex>
#include <set>
#include <thread>

#include "../../include/inlm.h"

namespace inlm {
int fail(int code, const char* fmt, ...);

namespace tiff {
namespace {

struct File {
    FILE* f = nullptr;
    explicit File(const std::string& path, const char* mode) { f = std::fopen(path.c_str(), mode); }
    ~File() {
        if (f) std::fclose(f);
    }
    bool read_at(uint64_t off, void* dst, size_t n) {
        if (fseeko(f, (off_t)off, SEEK_SET) != 0) return false;
        return std::fread(dst, 1, n, f) == n;
    }
    uint64_t size() {
        if (fseeko(f, 0, SEEK_END) != 0) return 0;
        return (uint64_t)ftello(f);
    }
};

bool ends_with(const std::string& s, const char* suffix) {
    const size_t n = std::strlen(suffix);
    return s.size() >= n && s.compare(s.size() - n, n, suffix) == 0;
}

uint16_t get16(const uint8_t* p, bool be) { return be ? (uint16_t)(p[0] << 8 | p[1]) : (uint16_t)(p[1] << 8 | p[0]); }
uint32_t get32(const uint8_t* p, bool be) {
    return be ? ((uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3])
              : ((uint32_t)p[3] << 24 | (uint32_t)p[2] << 16 | (uint32_t)p[1] << 8 | p[0]);
}

int type_size(uint16_t type) {
    switch (type) {
        case 1: case 2: case 6: case 7: return 1;
        case 3: case 8: return 2;
        case 4: case 9: case 11: return 4;
        case 5: case 10: case 12: return 8;
        default: return 0;
    }
}

// Reads the values of one IFD entry as unsigned integers (SHORT / LONG / BYTE).
bool entry_values(File& f, const uint8_t* e, bool be, std::vector<uint64_t>& out) {
    const uint16_t type = get16(e + 2, be);
    const uint32_t count = get32(e + 4, be);
    const int ts = type_size(type);
    if (ts == 0 || count == 0 || count > (1u << 28)) return false;
    const uint64_t bytes = (uint64_t)count * ts;
    std::vector<uint8_t> buf(bytes);
    if (bytes <= 4) {
        std::memcpy(buf.data(), e + 8, bytes);
    } else if (!f.read_at(get32(e + 8, be), buf.data(), bytes)) {
        return false;
    }
    out.resize(count);
    for (uint32_t i = 0; i < count; i++) {
        const uint8_t* p = buf.data() + (uint64_t)i * ts;
        if (type == 3 || type == 8) out[i] = get16(p, be);
        else if (type == 4 || type == 9) out[i] = get32(p, be);
        else if (ts == 1) out[i] = p[0];
        else return false;
    }
    return true;
}

bool entry_ascii(File& f, const uint8_t* e, bool be, std::string& out) {
    const uint32_t count = get32(e + 4, be);
    if (get16(e + 2, be) != 2 || count == 0 || count > (1u << 24)) return false;
    std::vector<char> buf(count);
    if (count <= 4) std::memcpy(buf.data(), e + 8, count);
    else if (!f.read_at(get32(e + 8, be), buf.data(), count)) return false;
    out.assign(buf.data(), strnlen(buf.data(), count));
    return true;
}

uint64_t page_bytes(const PageInfo& p) { return (uint64_t)p.width * p.height * p.samples * (p.bits / 8); }

// ImageJ writes stacks above 4 GB as one IFD followed by the pages back to
// back, with "images=N" in the description (the layout Custom3DTifReader reads).
uint64_t imagej_images(const PageInfo& p) {
    const size_t k = p.description.find("images=");
    if (k == std::string::npos) return 0;
    return std::strtoull(p.description.c_str() + k + 7, nullptr, 10);
}

void put16(std::vector<uint8_t>& b, uint16_t v) {
    b.push_back((uint8_t)(v & 0xff));
    b.push_back((uint8_t)(v >> 8));
}
void put32(std::vector<uint8_t>& b, uint32_t v) {
    for (int i = 0; i < 4; i++) b.push_back((uint8_t)(v >> (8 * i)));
}

}  // namespace

bool list_directory(const std::string& dir, std::vector<std::string>& files) {
    DIR* dp = opendir(dir.c_str());
    if (!dp) return false;
    std::string base = dir;
    if (!base.empty() && base.back() != '/') base += '/';
    while (dirent* e = readdir(dp)) {
        const std::string name = e->d_name;
        if (ends_with(name, ".tif") || ends_with(name, ".tiff")) files.push_back(base + name);
    }
    closedir(dp);
    std::sort(files.begin(), files.end());
    return true;
}

int read_pages(const std::string& file, std::vector<PageInfo>& pages) {
    File f(file, "rb");
    if (!f.f) return fail(INLM_ERR_IO, "cannot open %s", file.c_str());
    uint8_t hdr[8];
    if (!f.read_at(0, hdr, 8)) return fail(INLM_ERR_IO, "%s: short file", file.c_str());
    bool be;
    if (hdr[0] == 'I' && hdr[1] == 'I') be = false;
    else if (hdr[0] == 'M' && hdr[1] == 'M') be = true;
    else return fail(INLM_ERR_IO, "%s: not a TIFF file", file.c_str());
    const uint16_t magic = get16(hdr + 2, be);
    if (magic == 43) return fail(INLM_ERR_UNSUPPORTED, "%s: BigTIFF is not supported", file.c_str());
    if (magic != 42) return fail(INLM_ERR_IO, "%s: not a TIFF file (magic %u)", file.c_str(), magic);
    uint64_t ifd = get32(hdr + 4, be);
    std::set<uint64_t> seen;
    while (ifd != 0) {
        if (!seen.insert(ifd).second || seen.size() > (1u << 20))
            return fail(INLM_ERR_IO, "%s: IFD chain loops", file.c_str());
        uint8_t nb[2];
        if (!f.read_at(ifd, nb, 2)) return fail(INLM_ERR_IO, "%s: bad IFD offset", file.c_str());
        const uint16_t n = get16(nb, be);
        std::vector<uint8_t> ent((size_t)n * 12 + 4);
        if (!f.read_at(ifd + 2, ent.data(), ent.size()))
            return fail(INLM_ERR_IO, "%s: truncated IFD", file.c_str());
        PageInfo p;
        p.big_endian = be;
        std::vector<uint64_t> v;
        for (int i = 0; i < n; i++) {
            const uint8_t* e = ent.data() + i * 12;
            const uint16_t tag = get16(e, be);
            if (tag == 270) {
                entry_ascii(f, e, be, p.description);
                continue;
            }
            if (tag != 256 && tag != 257 && tag != 258 && tag != 259 && tag != 273 && tag != 277 &&
                tag != 278 && tag != 279 && tag != 284 && tag != 339 && tag != 322 && tag != 324)
                continue;
            if (!entry_values(f, e, be, v)) return fail(INLM_ERR_IO, "%s: bad tag %u", file.c_str(), tag);
            switch (tag) {
                case 256: p.width = (uint32_t)v[0]; break;
                case 257: p.height = (uint32_t)v[0]; break;
                case 258: p.bits = (uint16_t)v[0]; break;
                case 259: p.compression = (uint16_t)v[0]; break;
                case 273: p.strip_offsets = v; break;
                case 277: p.samples = (uint16_t)v[0]; break;
                case 278: p.rows_per_strip = (uint32_t)v[0]; break;
                case 279: p.strip_bytes = v; break;
                case 284: p.planar = (uint16_t)v[0]; break;
                case 339: p.sample_format = (uint16_t)v[0]; break;
                default: p.tiled = true; break;  // TileWidth / TileOffsets
            }
        }
        if (p.bits == 0) p.bits = 1;
        if (p.rows_per_strip == 0 || p.rows_per_strip > p.height) p.rows_per_strip = p.height;
        pages.push_back(std::move(p));
        ifd = get32(ent.data() + (size_t)n * 12, be);
    }
    if (pages.empty()) return fail(INLM_ERR_IO, "%s: no image directory", file.c_str());
    return INLM_OK;
}

static int check_page(const std::string& file, const PageInfo& p) {
    if (p.width == 0 || p.height == 0) return fail(INLM_ERR_IO, "%s: missing image size", file.c_str());
    if (p.tiled) return fail(INLM_ERR_UNSUPPORTED, "%s: tiled TIFF is not supported", file.c_str());
    if (p.compression != 1)
        return fail(INLM_ERR_UNSUPPORTED, "%s: compression %u is not supported (uncompressed only)",
                    file.c_str(), p.compression);
    if (p.samples != 1)
        return fail(INLM_ERR_UNSUPPORTED, "%s: %u samples per pixel (greyscale only)", file.c_str(),
                    p.samples);
    const bool ok = p.bits == 8 || p.bits == 16 || (p.bits == 32) || (p.bits == 64 && p.sample_format == 3);
    if (!ok) return fail(INLM_ERR_UNSUPPORTED, "%s: %u bits per sample", file.c_str(), p.bits);
    if (p.strip_offsets.empty()) return fail(INLM_ERR_IO, "%s: no strip offsets", file.c_str());
    return INLM_OK;
}

template <typename T>
static T load_sample(const uint8_t* s, bool swap) {
    uint8_t b[sizeof(T)];
    if (swap) {
        for (size_t i = 0; i < sizeof(T); i++) b[i] = s[sizeof(T) - 1 - i];
    } else {
        std::memcpy(b, s, sizeof(T));
    }
    T v;
    std::memcpy(&v, b, sizeof(T));
    return v;
}

static void convert_row(const uint8_t* src, const PageInfo& p, float* dst) {
    const bool swap = p.big_endian;  // hosts are little-endian
    const uint32_t w = p.width;
    const uint16_t sf = p.sample_format;
    switch (p.bits) {
        case 8:
            for (uint32_t x = 0; x < w; x++) dst[x] = sf == 2 ? (float)(int8_t)src[x] : (float)src[x];
            break;
        case 16:
            for (uint32_t x = 0; x < w; x++)
                dst[x] = sf == 2 ? (float)load_sample<int16_t>(src + 2 * x, swap)
                                 : (float)load_sample<uint16_t>(src + 2 * x, swap);
            break;
        case 32:
            for (uint32_t x = 0; x < w; x++) {
                if (sf == 3) dst[x] = load_sample<float>(src + 4 * x, swap);
                else if (sf == 2) dst[x] = (float)load_sample<int32_t>(src + 4 * x, swap);
                else dst[x] = (float)load_sample<uint32_t>(src + 4 * x, swap);
            }
            break;
        default:  // 64-bit IEEE
            for (uint32_t x = 0; x < w; x++) dst[x] = (float)load_sample<double>(src + 8 * x, swap);
            break;
    }
}

int read_page(const std::string& file, const PageInfo& p, uint64_t data_offset, float* out) {
    int rc = check_page(file, p);
    if (rc) return rc;
    File f(file, "rb");
    if (!f.f) return fail(INLM_ERR_IO, "cannot open %s", file.c_str());
    const uint64_t row_bytes = (uint64_t)p.width * (p.bits / 8);
    std::vector<uint8_t> buf;
    if (data_offset != UINT64_MAX) {  // pages stored back to back
        buf.resize(row_bytes * p.height);
        if (!f.read_at(data_offset, buf.data(), buf.size()))
            return fail(INLM_ERR_IO, "%s: truncated page data", file.c_str());
        for (uint32_t y = 0; y < p.height; y++) convert_row(buf.data() + y * row_bytes, p, out + (uint64_t)y * p.width);
        return INLM_OK;
    }
    const uint32_t rps = p.rows_per_strip;
    const uint64_t n_strips = (p.height + rps - 1) / rps;
    if (p.strip_offsets.size() < n_strips)
        return fail(INLM_ERR_IO, "%s: %zu strips for %llu", file.c_str(), p.strip_offsets.size(),
                    (unsigned long long)n_strips);
    for (uint64_t s = 0; s < n_strips; s++) {
        const uint32_t y0 = (uint32_t)(s * rps);
        const uint32_t rows = std::min<uint32_t>(rps, p.height - y0);
        const uint64_t need = rows * row_bytes;
        if (s < p.strip_bytes.size() && p.strip_bytes[s] < need)
            return fail(INLM_ERR_IO, "%s: strip %llu holds %llu bytes, %llu needed", file.c_str(),
                        (unsigned long long)s, (unsigned long long)p.strip_bytes[s],
                        (unsigned long long)need);
        buf.resize(need);
        if (!f.read_at(p.strip_offsets[s], buf.data(), need))
            return fail(INLM_ERR_IO, "%s: truncated strip %llu", file.c_str(), (unsigned long long)s);
        for (uint32_t r = 0; r < rows; r++)
            convert_row(buf.data() + r * row_bytes, p, out + (uint64_t)(y0 + r) * p.width);
    }
    return INLM_OK;
}

int write_slice(const std::string& file, const float* image, uint32_t width, uint32_t height,
                bool as_16bit) {
    const uint16_t bits = as_16bit ? 16 : 32;
    const uint64_t row_bytes = (uint64_t)width * (bits / 8);
    // 2048 samples per strip, at least one row (Save2DTifImage_32bit)
    uint32_t rps = 2048 / width;
    if (rps == 0) rps = 1;
    if (rps > height) rps = height;
    const uint32_t n_strips = (height + rps - 1) / rps;
    const uint64_t data_bytes = row_bytes * height;
    if (8 + data_bytes + 4096 + 8ull * n_strips > 0xffffffffull)
        return fail(INLM_ERR_UNSUPPORTED, "%s: slice too large for classic TIFF", file.c_str());

    std::vector<uint8_t> data(data_bytes);
    if (as_16bit) {
        for (uint64_t i = 0; i < (uint64_t)width * height; i++) {
            // std::min(std::max(0.f, round(v)), 65535.f): NaN maps to 0
            const float v = std::min(std::max(0.f, std::round(image[i])), 65535.f);
            const uint16_t u = (uint16_t)v;
            data[2 * i] = (uint8_t)(u & 0xff);
            data[2 * i + 1] = (uint8_t)(u >> 8);
        }
    } else {
        std::memcpy(data.data(), image, data_bytes);
    }

    const uint32_t data_off = 8;
    uint32_t ifd_off = (uint32_t)(data_off + data_bytes);
    ifd_off += ifd_off & 1;  // word boundary
    const uint16_t n_tags = 11;
    const uint32_t ifd_bytes = 2 + n_tags * 12 + 4;
    const uint32_t arrays_off = ifd_off + ifd_bytes;  // strip offset / byte count arrays
    std::vector<uint8_t> out;
    out.reserve(ifd_off + ifd_bytes + 8ull * n_strips);
    out.push_back('I');
    out.push_back('I');
    put16(out, 42);
    put32(out, ifd_off);
    out.insert(out.end(), data.begin(), data.end());
    while (out.size() < ifd_off) out.push_back(0);

    auto entry = [&](uint16_t tag, uint16_t type, uint32_t count, uint32_t value) {
        put16(out, tag);
        put16(out, type);
        put32(out, count);
        if (type == 3 && count == 1) {
            put16(out, (uint16_t)value);
            put16(out, 0);
        } else {
            put32(out, value);
        }
    };
    const uint32_t off_array = arrays_off, cnt_array = arrays_off + 4 * n_strips;
    put16(out, n_tags);
    entry(256, 4, 1, width);
    entry(257, 4, 1, height);
    entry(258, 3, 1, bits);
    entry(259, 3, 1, 1);  // no compression
    entry(262, 3, 1, 1);  // min-is-black
    entry(273, 4, n_strips, n_strips == 1 ? data_off : off_array);
    entry(277, 3, 1, 1);
    entry(278, 4, 1, rps);
    entry(279, 4, n_strips, n_strips == 1 ? (uint32_t)data_bytes : cnt_array);
    entry(284, 3, 1, 1);                 // contiguous
    entry(339, 3, 1, as_16bit ? 1 : 3);  // unsigned / IEEE float
    put32(out, 0);                       // last IFD
    if (n_strips > 1) {
        for (uint32_t s = 0; s < n_strips; s++) put32(out, (uint32_t)(data_off + (uint64_t)s * rps * row_bytes));
        for (uint32_t s = 0; s < n_strips; s++) {
            const uint32_t rows = std::min(rps, height - s * rps);
            put32(out, (uint32_t)(rows * row_bytes));
        }
    }
    File f(file, "wb");
    if (!f.f) return fail(INLM_ERR_IO, "cannot write %s", file.c_str());
    if (std::fwrite(out.data(), 1, out.size(), f.f) != out.size())
        return fail(INLM_ERR_IO, "short write to %s", file.c_str());
    return INLM_OK;
}

// An RGB(A) page as three float planes: 8- or 16-bit unsigned samples,
// interleaved (planar configuration 1); alpha is ignored
// (GetRGBTif_32bitChannels, hdcommunication.cpp:674-795).
int read_page_rgb(const std::string& file, const PageInfo& p, float* r, float* g, float* b) {
    if (p.width == 0 || p.height == 0) return fail(INLM_ERR_IO, "%s: missing image size", file.c_str());
    if (p.tiled || p.compression != 1)
        return fail(INLM_ERR_UNSUPPORTED, "%s: tiled or compressed TIFF is not supported", file.c_str());
    if ((p.samples != 3 && p.samples != 4) || p.planar != 1)
        return fail(INLM_ERR_UNSUPPORTED, "%s: %u samples per pixel, planar %u (RGB or RGBA, interleaved)",
                    file.c_str(), p.samples, p.planar);
    if ((p.bits != 8 && p.bits != 16) || p.sample_format == 3 || p.sample_format == 2)
        return fail(INLM_ERR_UNSUPPORTED, "%s: %u-bit RGB samples (8- or 16-bit unsigned only)", file.c_str(),
                    p.bits);
    if (p.strip_offsets.empty()) return fail(INLM_ERR_IO, "%s: no strip offsets", file.c_str());
    File f(file, "rb");
    if (!f.f) return fail(INLM_ERR_IO, "cannot open %s", file.c_str());
    const uint32_t bps = p.bits / 8;
    const uint64_t row_bytes = (uint64_t)p.width * p.samples * bps;
    const uint32_t rps = p.rows_per_strip;
    const uint64_t n_strips = (p.height + rps - 1) / rps;
    if (p.strip_offsets.size() < n_strips) return fail(INLM_ERR_IO, "%s: too few strips", file.c_str());
    std::vector<uint8_t> buf;
    for (uint64_t s = 0; s < n_strips; s++) {
        const uint32_t y0 = (uint32_t)(s * rps);
        const uint32_t rows = std::min<uint32_t>(rps, p.height - y0);
        const uint64_t need = rows * row_bytes;
        if (s < p.strip_bytes.size() && p.strip_bytes[s] < need)
            return fail(INLM_ERR_IO, "%s: short strip %llu", file.c_str(), (unsigned long long)s);
        buf.resize(need);
        if (!f.read_at(p.strip_offsets[s], buf.data(), need))
            return fail(INLM_ERR_IO, "%s: truncated strip %llu", file.c_str(), (unsigned long long)s);
        for (uint32_t yy = 0; yy < rows; yy++) {
            const uint8_t* row = buf.data() + yy * row_bytes;
            const uint64_t o = (uint64_t)(y0 + yy) * p.width;
            for (uint32_t x = 0; x < p.width; x++) {
                const uint8_t* px = row + (uint64_t)x * p.samples * bps;
                float v[3];
                for (int c = 0; c < 3; c++)
                    v[c] = bps == 1 ? (float)px[c] : (float)load_sample<uint16_t>(px + 2 * c, p.big_endian);
                r[o + x] = v[0];
                g[o + x] = v[1];
                b[o + x] = v[2];
            }
        }
    }
    return INLM_OK;
}

// 8-bit RGB slice (Save2DTifImage_RGB, hdcommunication.cpp:1487-1547):
// interleaved, photometric RGB, strips of max(1, 2048 / width) rows.
int write_rgb(const std::string& file, const uint8_t* rgb, uint32_t width, uint32_t height) {
    uint32_t rps = 2048 / width;
    if (rps == 0) rps = 1;
    if (rps > height) rps = height;
    const uint64_t row_bytes = 3ull * width;
    const uint32_t n_strips = (height + rps - 1) / rps;
    const uint64_t data_bytes = row_bytes * height;
    if (8 + data_bytes + 4096 + 8ull * n_strips > 0xffffffffull)
        return fail(INLM_ERR_UNSUPPORTED, "%s: image too large for classic TIFF", file.c_str());
    const uint32_t data_off = 8;
    uint32_t ifd_off = (uint32_t)(data_off + data_bytes);
    ifd_off += ifd_off & 1;
    const uint16_t n_tags = 11;
    const uint32_t bits_off = ifd_off + 2 + n_tags * 12 + 4;  // BitsPerSample: 3 SHORTs
    const uint32_t arrays_off = bits_off + 6 + 2;
    std::vector<uint8_t> out;
    out.reserve(arrays_off + 8ull * n_strips);
    out.push_back('I');
    out.push_back('I');
    put16(out, 42);
    put32(out, ifd_off);
    out.insert(out.end(), rgb, rgb + data_bytes);
    while (out.size() < ifd_off) out.push_back(0);
    auto entry = [&](uint16_t tag, uint16_t type, uint32_t count, uint32_t value) {
        put16(out, tag);
        put16(out, type);
        put32(out, count);
        if (type == 3 && count == 1) {
            put16(out, (uint16_t)value);
            put16(out, 0);
        } else {
            put32(out, value);
        }
    };
    const uint32_t off_array = arrays_off, cnt_array = arrays_off + 4 * n_strips;
    put16(out, n_tags);
    entry(256, 4, 1, width);
    entry(257, 4, 1, height);
    entry(258, 3, 3, bits_off);
    entry(259, 3, 1, 1);
    entry(262, 3, 1, 2);  // RGB
    entry(273, 4, n_strips, n_strips == 1 ? data_off : off_array);
    entry(277, 3, 1, 3);
    entry(278, 4, 1, rps);
    entry(279, 4, n_strips, n_strips == 1 ? (uint32_t)data_bytes : cnt_array);
    entry(284, 3, 1, 1);
    entry(339, 3, 1, 1);
    put32(out, 0);
    for (int c = 0; c < 3; c++) put16(out, 8);
    put16(out, 0);  // pad to a word boundary
    if (n_strips > 1) {
        for (uint32_t s = 0; s < n_strips; s++) put32(out, (uint32_t)(data_off + (uint64_t)s * rps * row_bytes));
        for (uint32_t s = 0; s < n_strips; s++) put32(out, (uint32_t)(std::min(rps, height - s * rps) * row_bytes));
    }
    File f(file, "wb");
    if (!f.f) return fail(INLM_ERR_IO, "cannot write %s", file.c_str());
    if (std::fwrite(out.data(), 1, out.size(), f.f) != out.size())
        return fail(INLM_ERR_IO, "short write to %s", file.c_str());
    return INLM_OK;
}

namespace {

// What one path holds: slice files, or the pages of one file.
struct Source {
    bool single_file = false;
    std::vector<std::string> files;     // one per slice (directory form)
    std::vector<PageInfo> pages;        // single-file form: one per slice ...
    uint64_t contiguous_base = UINT64_MAX;  // ... or one page repeated back to back
    uint32_t width = 0, height = 0;
    uint16_t samples = 1;
    uint64_t depth = 0;
};

int open_source(const std::string& path, Source& src) {
    if (ends_with(path, "tif") || ends_with(path, "tiff")) {
        if (!std::filesystem::is_regular_file(path))
            return fail(INLM_ERR_IO, "Directory or file not found: %s", path.c_str());
        src.single_file = true;
        src.files.push_back(path);
        int rc = read_pages(path, src.pages);
        if (rc) return rc;
        const PageInfo& p0 = src.pages[0];
        src.width = p0.width;
        src.height = p0.height;
        src.samples = p0.samples;
        src.depth = src.pages.size();
        const uint64_t n_ij = imagej_images(p0);
        if (src.pages.size() == 1 && n_ij > 1 && !p0.strip_offsets.empty() && p0.bits % 8 == 0) {
            File f(path, "rb");
            const uint64_t end = p0.strip_offsets[0] + n_ij * page_bytes(p0);
            if (f.f && f.size() >= end) {
                src.contiguous_base = p0.strip_offsets[0];
                src.depth = n_ij;
            }
        }
        return INLM_OK;
    }
    if (!std::filesystem::is_directory(path))
        return fail(INLM_ERR_IO, "Directory or file not found: %s", path.c_str());
    if (!list_directory(path, src.files)) return fail(INLM_ERR_IO, "cannot open directory %s", path.c_str());
    if (src.files.empty()) return fail(INLM_ERR_IO, "No tif-file in directory %s", path.c_str());
    std::vector<PageInfo> first;
    int rc = read_pages(src.files[0], first);
    if (rc) return rc;
    src.width = first[0].width;
    src.height = first[0].height;
    src.samples = first[0].samples;
    src.depth = src.files.size();
    return INLM_OK;
}

// Reads slice z of the source into out.
int read_slice(const Source& src, uint64_t z, float* out) {
    if (src.single_file) {
        const std::string& file = src.files[0];
        if (src.contiguous_base != UINT64_MAX)
            return read_page(file, src.pages[0], src.contiguous_base + z * page_bytes(src.pages[0]), out);
        const PageInfo& p = src.pages[z];
        if (p.width != src.width || p.height != src.height)
            return fail(INLM_ERR_IO, "%s: page %llu is %ux%u, page 0 is %ux%u", file.c_str(),
                        (unsigned long long)z, p.width, p.height, src.width, src.height);
        return read_page(file, p, UINT64_MAX, out);
    }
    const std::string& file = src.files[z];
    std::vector<PageInfo> pages;
    int rc = read_pages(file, pages);
    if (rc) return rc;
    if (pages[0].width != src.width || pages[0].height != src.height)
        return fail(INLM_ERR_IO, "%s is %ux%u, the first slice is %ux%u", file.c_str(), pages[0].width,
                    pages[0].height, src.width, src.height);
    return read_page(file, pages[0], UINT64_MAX, out);
}

// Runs fn(i) for i in [0, n) on up to 16 host threads; returns the first error.
template <typename Fn>
int parallel_slices(uint64_t n, Fn fn) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned nt = (unsigned)std::min<uint64_t>(std::min(hw, 16u), n);
    std::atomic<uint64_t> next{0};
    std::atomic<int> status{INLM_OK};
    std::mutex err_mu;
    std::string err_text;
    auto work = [&]() {
        for (;;) {
            const uint64_t i = next.fetch_add(1);
            if (i >= n || status.load() != INLM_OK) return;
            const int rc = fn(i);
            if (rc != INLM_OK) {
                int expected = INLM_OK;
                if (status.compare_exchange_strong(expected, rc)) {
                    std::lock_guard<std::mutex> g(err_mu);
                    err_text = inlm_last_error();
                }
                return;
            }
        }
    };
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < nt; t++) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    if (status.load() != INLM_OK) return fail(status.load(), "%s", err_text.c_str());
    return INLM_OK;
}

}  // namespace
}  // namespace tiff
}  // namespace inlm

using namespace inlm;

extern "C" int inlm_tiff_shape(const char* path, int shape[3], int* samples_per_pixel) {
    if (!path || !shape) return fail(INLM_ERR_ARG, "null argument");
    tiff::Source src;
    int rc = tiff::open_source(path, src);
    if (rc) return rc;
    if (src.depth > 0x7fffffff) return fail(INLM_ERR_UNSUPPORTED, "%s: too many slices", path);
    shape[0] = (int)src.width;
    shape[1] = (int)src.height;
    shape[2] = (int)src.depth;
    if (samples_per_pixel) *samples_per_pixel = src.samples;
    return INLM_OK;
}

extern "C" int inlm_tiff_read(const char* path, int first_slice, int last_slice, float* out,
                              uint64_t n_out) {
    if (!path || !out) return fail(INLM_ERR_ARG, "null argument");
    tiff::Source src;
    int rc = tiff::open_source(path, src);
    if (rc) return rc;
    if (src.samples != 1)
        return fail(INLM_ERR_UNSUPPORTED, "%s: %u samples per pixel (greyscale only)", path, src.samples);
    const int64_t depth = (int64_t)src.depth;
    // main.cpp:278-281: a range given at either end is clamped to the stack
    int64_t z0 = 0, z1 = depth - 1;
    if (first_slice != -1 || last_slice != -1) {
        z0 = std::max<int64_t>(0, first_slice);
        z1 = last_slice == -1 ? depth - 1 : std::min<int64_t>(depth - 1, last_slice);
    }
    if (z1 < z0) return fail(INLM_ERR_ARG, "empty slice range %d..%d of %lld", first_slice, last_slice,
                             (long long)depth);
    const uint64_t nslice = (uint64_t)src.width * src.height;
    const uint64_t nz = (uint64_t)(z1 - z0 + 1);
    if (n_out < nslice * nz)
        return fail(INLM_ERR_ARG, "output holds %llu floats, %llu needed", (unsigned long long)n_out,
                    (unsigned long long)(nslice * nz));
    return tiff::parallel_slices(nz, [&](uint64_t i) { return tiff::read_slice(src, (uint64_t)z0 + i, out + i * nslice); });
}

extern "C" int inlm_tiff_write_sequence(const float* image, const int shape[3], int z0,
                                        const char* dir, const char* name, int as_16bit) {
    if (!image || !shape || !dir || !name) return fail(INLM_ERR_ARG, "null argument");
    if (shape[0] <= 0 || shape[1] <= 0 || shape[2] <= 0 || z0 < 0)
        return fail(INLM_ERR_ARG, "bad shape %dx%dx%d or first index %d", shape[0], shape[1], shape[2], z0);
    std::error_code ec;
    std::filesystem::create_directories(dir, ec);
    if (ec) return fail(INLM_ERR_IO, "cannot create %s: %s", dir, ec.message().c_str());
    const uint64_t nslice = (uint64_t)shape[0] * shape[1];
    const std::string base = std::string(dir) + "/" + name;
    return tiff::parallel_slices((uint64_t)shape[2], [&](uint64_t i) {
        // name + 4-digit zero-filled slice index (zfill_int2string, hdcommunication.cpp:42)
        char id[32];
        std::snprintf(id, sizeof id, "%04llu", (unsigned long long)(z0 + i));
        return tiff::write_slice(base + id + ".tif", image + i * nslice, (uint32_t)shape[0],
                                 (uint32_t)shape[1], as_16bit != 0);
    });
}

extern "C" int inlm_tiff_read_rgb(const char* file, int shape[2], float* r, float* g, float* b,
                                  uint64_t n_out) {
    if (!file || !shape) return fail(INLM_ERR_ARG, "null argument");
    std::vector<tiff::PageInfo> pages;
    int rc = tiff::read_pages(file, pages);
    if (rc) return rc;
    const tiff::PageInfo& p = pages[0];
    shape[0] = (int)p.width;
    shape[1] = (int)p.height;
    if (!r && !g && !b) return INLM_OK;  // size query
    if (!r || !g || !b) return fail(INLM_ERR_ARG, "null channel plane");
    if (n_out < (uint64_t)p.width * p.height)
        return fail(INLM_ERR_ARG, "planes hold %llu values, %llu needed", (unsigned long long)n_out,
                    (unsigned long long)p.width * p.height);
    return tiff::read_page_rgb(file, p, r, g, b);
}

extern "C" int inlm_tiff_write_rgb(const char* dir, const char* name, const float* r, const float* g,
                                   const float* b, int nx, int ny) {
    if (!dir || !name || !r || !g || !b) return fail(INLM_ERR_ARG, "null argument");
    if (nx <= 0 || ny <= 0) return fail(INLM_ERR_ARG, "bad image size %dx%d", nx, ny);
    std::error_code ec;
    std::filesystem::create_directories(dir, ec);
    if (ec) return fail(INLM_ERR_IO, "cannot create %s: %s", dir, ec.message().c_str());
    const uint64_t n = (uint64_t)nx * ny;
    std::vector<uint8_t> rgb(3 * n);
    const float* ch[3] = {r, g, b};
    for (uint64_t i = 0; i < n; i++)
        for (int c = 0; c < 3; c++) {
            // (uint8_t) std::min(255.f, v) (color_denoising.h:76-78): NaN gives
            // 255, values truncate toward zero; below zero gives 0
            const float v = ch[c][i];
            const float t = (v < 255.f) ? v : 255.f;
            rgb[3 * i + c] = (t > 0.f) ? (uint8_t)t : 0;
        }
    return tiff::write_rgb(std::string(dir) + "/" + name + ".tif", rgb.data(), (uint32_t)nx, (uint32_t)ny);
}
