// MVTools vector data on the host: the two frame properties the vnlb plugin
// reads from its mvfw / mvbw clips, with the reference's checks and messages.
//
//   MVTools_MVAnalysisData  21 little-endian 32-bit fields, of which fields
//                           2-7 and 10-20 are read (parse_mvtools_analysis,
//                           src/flow/flow.hpp:193-250)
//   MVTools_vectors         u32 total size, u32 valid flag, then the levels
//                           of the search, each a u32 byte size followed by
//                           16-byte vectors (i32 x, i32 y, u64 SAD); the last
//                           level is the finest and the one used
//                           (parse_mvtools_vectors, flow.hpp:252-318)
#include "mvtools.h"

#include <climits>
#include <stdexcept>

namespace vnlbgpu {
namespace mvtools {
namespace {

uint32_t read_u32(const unsigned char* data, size_t size, size_t offset) {
    if (offset + 4 > size) throw std::invalid_argument("truncated MVTools data");
    return static_cast<uint32_t>(data[offset]) | (static_cast<uint32_t>(data[offset + 1]) << 8) |
           (static_cast<uint32_t>(data[offset + 2]) << 16) | (static_cast<uint32_t>(data[offset + 3]) << 24);
}

int read_i32(const unsigned char* data, size_t size, size_t offset) {
    const uint32_t u = read_u32(data, size, offset);
    return u <= static_cast<uint32_t>(INT_MAX) ? static_cast<int>(u)
                                               : -static_cast<int>(~u) - 1;  // two's complement
}

int positive(uint32_t value, const char* what) {
    if (value == 0 || value > static_cast<uint32_t>(INT_MAX)) throw std::invalid_argument(what);
    return static_cast<int>(value);
}

int nonnegative(uint32_t value, const char* what) {
    if (value > static_cast<uint32_t>(INT_MAX)) throw std::invalid_argument(what);
    return static_cast<int>(value);
}

}  // namespace

vnlbgpu_mvtools_analysis parse_analysis(const void* bytes, size_t size) {
    if (size != 21 * 4) throw std::invalid_argument("MVTools_MVAnalysisData must contain 21 32-bit fields");
    const auto* d = static_cast<const unsigned char*>(bytes);
    vnlbgpu_mvtools_analysis a{};
    a.block_size_x = positive(read_u32(d, size, 2 * 4), "invalid MVTools horizontal block size");
    a.block_size_y = positive(read_u32(d, size, 3 * 4), "invalid MVTools vertical block size");
    a.pel = positive(read_u32(d, size, 4 * 4), "invalid MVTools pel");
    a.level_count = positive(read_u32(d, size, 5 * 4), "invalid MVTools level count");
    a.delta_frame = read_i32(d, size, 6 * 4);
    a.backwards = read_u32(d, size, 7 * 4) != 0 ? 1 : 0;
    a.width = positive(read_u32(d, size, 10 * 4), "invalid MVTools width");
    a.height = positive(read_u32(d, size, 11 * 4), "invalid MVTools height");
    a.overlap_x = nonnegative(read_u32(d, size, 12 * 4), "invalid MVTools horizontal overlap");
    a.overlap_y = nonnegative(read_u32(d, size, 13 * 4), "invalid MVTools vertical overlap");
    a.block_count_x = positive(read_u32(d, size, 14 * 4), "invalid MVTools horizontal block count");
    a.block_count_y = positive(read_u32(d, size, 15 * 4), "invalid MVTools vertical block count");
    a.bits_per_sample = positive(read_u32(d, size, 16 * 4), "invalid MVTools bit depth");
    a.chroma_ratio_y = positive(read_u32(d, size, 17 * 4), "invalid MVTools vertical chroma ratio");
    a.chroma_ratio_x = positive(read_u32(d, size, 18 * 4), "invalid MVTools horizontal chroma ratio");
    a.padding_x = nonnegative(read_u32(d, size, 19 * 4), "invalid MVTools horizontal padding");
    a.padding_y = nonnegative(read_u32(d, size, 20 * 4), "invalid MVTools vertical padding");
    if (a.overlap_x >= a.block_size_x || a.overlap_y >= a.block_size_y)
        throw std::invalid_argument("MVTools overlap must be smaller than block size");
    return a;
}

bool parse_vectors(const void* bytes, size_t size, const vnlbgpu_mvtools_analysis& a, std::vector<int>& xy) {
    if (size < 8) throw std::invalid_argument("MVTools_vectors is too small");
    const auto* d = static_cast<const unsigned char*>(bytes);
    if (read_u32(d, size, 0) != size) throw std::invalid_argument("MVTools_vectors size header is invalid");
    xy.clear();
    if (read_u32(d, size, 4) != 1) return false;
    // walk the levels; the last one is the finest
    size_t position = 8, finest_begin = 0, finest_end = 0;
    while (position < size) {
        const size_t level_begin = position;
        if (level_begin + 4 > size) throw std::invalid_argument("truncated MVTools level header");
        const uint32_t level_size = read_u32(d, size, level_begin);
        if (level_size < 4 || level_begin + level_size > size)
            throw std::invalid_argument("invalid MVTools level size");
        finest_begin = level_begin + 4;
        finest_end = level_begin + level_size;
        position = finest_end;
    }
    const size_t finest = finest_end - finest_begin;
    if (finest % 16 != 0) throw std::invalid_argument("MVTools finest level has invalid vector size");
    const size_t count = finest / 16;
    if (count != static_cast<size_t>(a.block_count_x) * static_cast<size_t>(a.block_count_y))
        throw std::invalid_argument("MVTools finest level vector count does not match analysis data");
    xy.resize(2 * count);
    for (size_t i = 0; i < count; ++i) {
        xy[2 * i] = read_i32(d, size, finest_begin + 16 * i);
        xy[2 * i + 1] = read_i32(d, size, finest_begin + 16 * i + 4);
    }
    return true;
}

}  // namespace mvtools
}  // namespace vnlbgpu

extern "C" {

int vnlbgpu_parse_mvtools_analysis(const void* data, size_t size, vnlbgpu_mvtools_analysis* out) {
    try {
        if (!data || !out) throw std::invalid_argument("null argument");
        *out = vnlbgpu::mvtools::parse_analysis(data, size);
        return 0;
    } catch (const std::exception& e) {
        vnlbgpu::set_last_error(std::string("VNLB: ") + e.what());
        return -1;
    }
}

int vnlbgpu_parse_mvtools_vectors(const void* data, size_t size, const vnlbgpu_mvtools_analysis* analysis,
                                  int* valid, int* xy, size_t capacity, size_t* count) {
    try {
        if (!data || !analysis || !valid || !count) throw std::invalid_argument("null argument");
        std::vector<int> v;
        *valid = vnlbgpu::mvtools::parse_vectors(data, size, *analysis, v) ? 1 : 0;
        *count = v.size() / 2;
        for (size_t i = 0; i < v.size() && i < 2 * capacity; ++i) xy[i] = v[i];
        return 0;
    } catch (const std::exception& e) {
        vnlbgpu::set_last_error(std::string("VNLB: ") + e.what());
        return -1;
    }
}

}  // extern "C"
