// SPDX-License-Identifier: Apache-2.0
//
// Host-side format core for the B200 backend: format normalisation, section
// layout and the per-call Plan.  Restates normalize_format / make_layout /
// write_header / FormatSizeCache (src/internal.hpp:225-454) so the library
// is self-contained.
#pragma once

#include "plan.hpp"

#include <cstdint>
#include <string>

namespace bpb200 {

enum Status : int {
    kOk = 0,
    kInvalidArgument = 1, // std::invalid_argument
    kOverflow = 2,        // std::overflow_error
    kLength = 3,          // std::length_error
    kRuntime = 4,         // std::runtime_error
    kUnavailable = 6,     // backend not usable on this machine
};

struct Format {
    uint8_t middle_group_log2 = 5;
    uint8_t middle_placement = 0;
    uint8_t input_cluster_count = 0;
    uint8_t output_cluster_count = 0;
    uint8_t input_clusters[64] = {};
    uint8_t output_clusters[64] = {};
};

struct Layout {
    Format format;        // normalised
    uint64_t size = 0;
    uint64_t network_size = 0;
    uint64_t switch_bits = 0;
    uint64_t middle_bits = 0;
    uint32_t depth = 0;   // routing depth
    uint64_t header_bytes = 0;
    uint64_t input_offset = 0;
    uint64_t output_offset = 0;
    uint64_t middle_offset = 0;
    uint64_t end_offset = 0;
};

struct Error {
    int code = kOk;
    std::string message;
    bool ok() const { return code == kOk; }
};

// make_layout(count, format) including normalisation.  Same error kinds
// and messages as the reference.
Error make_layout(uint64_t count, const Format& format, Layout* out);

// Header bytes (src/internal.hpp:431-454) into out[0 .. layout.header_bytes).
void write_header(const Layout& layout, uint8_t* out);

// Fill the per-call plan.  `tile_max` is the largest node the shared-memory
// tile kernel accepts; levels whose padded node capacity exceeds it are
// processed by the level kernels in global memory.
Error make_plan(const Layout& layout, uint64_t tile_max, Plan* plan);

} // namespace bpb200
