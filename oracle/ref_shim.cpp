// SPDX-License-Identifier: Apache-2.0
//
// C-ABI shim over the reference library built from its own, unmodified
// sources (see oracle/Makefile).  TEST INFRASTRUCTURE ONLY: it is the
// checker for the oracle restatement and the timed CPU baseline; the B200
// library never links or loads it.
//
// Calls: benes::compress with Backend::portable_cpu
// (include/benes/benes.hpp:47-52, src/benes.cpp:460-496),
// CompressedPermutationView (src/benes.cpp:581-620), and the reference's
// SectionAddress (src/internal.hpp:475-718) for address probes.
#include <benes/benes.hpp>

#include "internal.hpp"

#include <cstdio>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <thread>
#include <vector>

namespace {

struct ref_format {
    std::uint8_t middle_group_log2;
    std::uint8_t middle_placement;
    std::uint8_t input_cluster_count;
    std::uint8_t output_cluster_count;
    std::uint8_t input_clusters[64];
    std::uint8_t output_clusters[64];
};

benes::FormatOptions to_options(const ref_format* f) {
    benes::FormatOptions o;
    o.middle_group_log2 = f->middle_group_log2;
    o.middle_placement = static_cast<benes::MiddlePlacement>(f->middle_placement);
    o.input_clusters.assign(f->input_clusters, f->input_clusters + f->input_cluster_count);
    o.output_clusters.assign(f->output_clusters, f->output_clusters + f->output_cluster_count);
    return o;
}

template <typename Fn>
int guarded(char* err, std::size_t err_len, Fn&& fn) {
    auto note = [&](const std::exception& e) {
        if (err != nullptr && err_len > 0) {
            std::snprintf(err, err_len, "%s", e.what());
        }
    };
    try {
        fn();
        return 0;
    } catch (const std::invalid_argument& e) {
        note(e);
        return 1;
    } catch (const std::length_error& e) {
        note(e);
        return 3;
    } catch (const std::out_of_range& e) {
        note(e);
        return 4;
    } catch (const std::logic_error& e) {
        note(e);
        return 5;
    } catch (const std::overflow_error& e) {
        note(e);
        return 2;
    } catch (const std::exception& e) {
        note(e);
        return 4;
    }
}

void walk(std::uint64_t count, const benes::FormatOptions& options, int depth,
    const std::uint8_t* turns, benes::detail::FormatSizeCache& sizes,
    const benes::detail::Layout& layout, benes::detail::SectionAddress& in,
    benes::detail::SectionAddress& out, std::uint64_t& node, std::uint64_t& middle) {
    (void)options;
    in = benes::detail::SectionAddress(count, layout.input_clusters,
        layout.middle_placement == benes::MiddlePlacement::embedded_input, sizes);
    out = benes::detail::SectionAddress(count, layout.output_clusters,
        layout.middle_placement == benes::MiddlePlacement::embedded_output, sizes);
    middle = 0;
    for (int d = 0; d < depth; ++d) {
        if (count <= sizes.leaf_size()) {
            throw std::invalid_argument("path descends below a leaf");
        }
        const std::uint64_t left = count / 2 + count % 2;
        if (turns[d]) {
            middle += sizes.middle_bits(left);
        }
        in = in.child(turns[d] != 0, count);
        out = out.child(turns[d] != 0, count);
        count = turns[d] ? count / 2 : left;
    }
    node = count;
}

} // namespace

extern "C" {

unsigned ref_hardware_threads(void) {
    return std::max(1U, std::thread::hardware_concurrency());
}

int ref_encoded_size(std::uint64_t count, const ref_format* f, std::uint64_t* size,
    char* err, std::size_t err_len) {
    return guarded(err, err_len, [&] {
        *size = benes::detail::make_layout(count, to_options(f)).end_offset;
    });
}

int ref_compress(const void* permutation, std::uint64_t count, std::uint32_t entry_bytes,
    const ref_format* f, std::size_t threads, std::uint8_t* blob, std::uint64_t capacity,
    std::uint64_t* blob_len, char* err, std::size_t err_len) {
    return guarded(err, err_len, [&] {
        benes::CompressOptions options;
        options.backend = benes::Backend::portable_cpu;
        options.threads = threads;
        options.format = to_options(f);
        std::vector<std::byte> bytes;
        if (entry_bytes == 4) {
            bytes = benes::compress(std::span<const std::uint32_t>(
                static_cast<const std::uint32_t*>(permutation), count), options);
        } else if (entry_bytes == 8) {
            bytes = benes::compress(std::span<const std::uint64_t>(
                static_cast<const std::uint64_t*>(permutation), count), options);
        } else {
            throw std::invalid_argument("entry width must be 4 or 8 bytes");
        }
        if (bytes.size() > capacity) {
            throw std::length_error("blob buffer is too small");
        }
        std::memcpy(blob, bytes.data(), bytes.size());
        *blob_len = bytes.size();
    });
}

int ref_validate(const std::uint8_t* blob, std::uint64_t len, char* err, std::size_t err_len) {
    return guarded(err, err_len, [&] {
        const benes::CompressedPermutationView view(
            std::span<const std::byte>(reinterpret_cast<const std::byte*>(blob), len));
        (void)view;
    });
}

int ref_lookup(const std::uint8_t* blob, std::uint64_t len, std::uint64_t value, int inverse,
    std::uint64_t* result, char* err, std::size_t err_len) {
    return guarded(err, err_len, [&] {
        const benes::CompressedPermutationView view(
            std::span<const std::byte>(reinterpret_cast<const std::byte*>(blob), len));
        *result = inverse ? view.inverse(value) : view.forward(value);
    });
}

int ref_switch_bit(std::uint64_t count, const ref_format* f, int side, int depth,
    const std::uint8_t* turns, std::uint64_t pair, std::uint64_t* bit) {
    return guarded(nullptr, 0, [&] {
        const auto options = to_options(f);
        const auto layout = benes::detail::make_layout(count, options);
        benes::detail::FormatSizeCache sizes(layout.middle_group_log2);
        benes::detail::SectionAddress in, out;
        std::uint64_t node = 0, middle = 0;
        walk(count, options, depth, turns, sizes, layout, in, out, node, middle);
        if (node <= sizes.leaf_size() || pair >= node / 2) {
            throw std::invalid_argument("no such switch");
        }
        *bit = (side ? out : in).switch_bit(pair);
    });
}

int ref_middle_bit(std::uint64_t count, const ref_format* f, int depth,
    const std::uint8_t* turns, std::uint64_t* bit) {
    return guarded(nullptr, 0, [&] {
        const auto options = to_options(f);
        const auto layout = benes::detail::make_layout(count, options);
        benes::detail::FormatSizeCache sizes(layout.middle_group_log2);
        benes::detail::SectionAddress in, out;
        std::uint64_t node = 0, middle = 0;
        walk(count, options, depth, turns, sizes, layout, in, out, node, middle);
        if (node > sizes.leaf_size()) {
            throw std::invalid_argument("not a leaf");
        }
        if (layout.middle_placement == benes::MiddlePlacement::embedded_input) {
            *bit = in.middle_bit();
        } else if (layout.middle_placement == benes::MiddlePlacement::embedded_output) {
            *bit = out.middle_bit();
        } else {
            *bit = middle;
        }
    });
}

} // extern "C"
