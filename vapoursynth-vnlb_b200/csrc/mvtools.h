// MVTools vector data on the host (mvtools.cpp): the parsers the session and
// the C ABI share.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/vnlbgpu.h"

namespace vnlbgpu {

// the calling thread's vnlbgpu_last_error text (session.cpp)
void set_last_error(const std::string& message);

namespace mvtools {

// parse_mvtools_analysis (src/flow/flow.hpp:193-250); throws
// std::invalid_argument with the reference's message.
vnlbgpu_mvtools_analysis parse_analysis(const void* bytes, size_t size);

// parse_mvtools_vectors (flow.hpp:252-318): the valid flag, and (when valid)
// the finest level's vectors as x, y pairs in xy.
bool parse_vectors(const void* bytes, size_t size, const vnlbgpu_mvtools_analysis& analysis, std::vector<int>& xy);

}  // namespace mvtools
}  // namespace vnlbgpu
