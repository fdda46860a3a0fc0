// Uncompressed baseline TIFF reading and writing for slice sequences, without
// libtiff. Covers what the iterNLM driver reads and writes through
// hdcom::HdCommunication (Geometry/hdcommunication.cpp): greyscale slices of
// 8, 16 or 32 bits per sample in strips, little- or big-endian, one file per
// z slice or one multi-page file.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace inlm {
namespace tiff {

struct PageInfo {
    uint32_t width = 0, height = 0;
    uint16_t bits = 0;           // bits per sample
    uint16_t samples = 1;        // samples per pixel
    uint16_t sample_format = 1;  // 1 unsigned, 2 signed, 3 IEEE float
    uint16_t compression = 1;
    uint16_t planar = 1;
    bool tiled = false;
    bool big_endian = false;
    std::vector<uint64_t> strip_offsets, strip_bytes;
    uint32_t rows_per_strip = 0;
    std::string description;  // ImageDescription (tag 270), ImageJ's "images=N"
};

// Sorted .tif / .tiff file names of a directory (GetFilelist,
// hdcommunication.cpp:1788); returns false if the directory cannot be opened.
bool list_directory(const std::string& dir, std::vector<std::string>& files);

// Reads the IFD chain of a file. Returns 0 or an INLM_ERR_* code.
int read_pages(const std::string& file, std::vector<PageInfo>& pages);

// Converts one page's samples to float by value into out (width*height).
int read_page(const std::string& file, const PageInfo& page, uint64_t data_offset, float* out);

// Writes one slice, width x height floats at image, as 32-bit IEEE float or
// as 16-bit unsigned (clamp to [0, 65535] after rounding).
int write_slice(const std::string& file, const float* image, uint32_t width, uint32_t height,
                bool as_16bit);

}  // namespace tiff
}  // namespace inlm
