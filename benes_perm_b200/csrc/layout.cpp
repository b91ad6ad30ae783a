// SPDX-License-Identifier: Apache-2.0
#include "layout.hpp"

#include <cstring>
#include <map>
#include <utility>

namespace bpb200 {
namespace {

struct Fail {
    int code;
    const char* message;
};

uint64_t add(uint64_t a, uint64_t b) {
    if (b > UINT64_MAX - a) {
        throw Fail{kOverflow, "compressed permutation is too large"};
    }
    return a + b;
}

// ceil(log2(c!)) exactly: bit width of c! - 1 (src/internal.hpp:173-183).
uint32_t factoradic_bits(uint32_t c) {
    unsigned __int128 f = 1;
    for (uint32_t i = 2; i <= c; ++i) {
        f *= i;
    }
    f -= 1;
    uint32_t bits = 0;
    while (f != 0) {
        ++bits;
        f >>= 1;
    }
    return bits;
}

// Memoised subtree sizes (FormatSizeCache, src/internal.hpp:225-313).
class Sizes {
public:
    explicit Sizes(uint32_t leaf) : leaf_(leaf) {}

    std::pair<uint64_t, uint64_t> subtree(uint64_t c) {
        if (c <= leaf_) {
            return {0, factoradic_bits((uint32_t)c)};
        }
        auto it = subtree_.find(c);
        if (it != subtree_.end()) {
            return it->second;
        }
        const auto l = subtree(c - c / 2);
        const auto r = subtree(c / 2);
        const std::pair<uint64_t, uint64_t> v{
            add(c / 2, add(l.first, r.first)), add(l.second, r.second)};
        subtree_.emplace(c, v);
        return v;
    }
    uint64_t switches(uint64_t c) { return subtree(c).first; }
    uint64_t middle(uint64_t c) { return subtree(c).second; }

    uint64_t top_switches(uint64_t c, uint32_t depth) {
        if (c <= leaf_ || depth == 0) {
            return 0;
        }
        const auto key = std::make_pair(c, depth);
        auto it = top_.find(key);
        if (it != top_.end()) {
            return it->second;
        }
        const uint64_t v = add(c / 2,
            add(top_switches(c - c / 2, depth - 1), top_switches(c / 2, depth - 1)));
        top_.emplace(key, v);
        return v;
    }

private:
    uint32_t leaf_;
    std::map<uint64_t, std::pair<uint64_t, uint64_t>> subtree_;
    std::map<std::pair<uint64_t, uint32_t>, uint64_t> top_;
};

uint32_t routing_depth(uint64_t count, uint32_t leaf) {
    uint32_t d = 0;
    while (count > leaf) {
        count = count - count / 2;
        ++d;
    }
    return d;
}

uint8_t balanced_clusters(uint32_t depth, uint8_t* out) {
    if (depth == 0) {
        return 0;
    }
    if (depth == 1) {
        out[0] = 1;
        return 1;
    }
    out[0] = (uint8_t)((depth + 1) / 2);
    out[1] = (uint8_t)(depth / 2);
    return 2;
}

void check_clusters(const uint8_t* c, uint32_t n, uint32_t depth) {
    uint32_t sum = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (c[i] == 0) {
            throw Fail{kInvalidArgument, "cluster depths must be positive"};
        }
        sum += c[i];
    }
    if (sum != depth) {
        throw Fail{kInvalidArgument, "cluster depths do not span every routing level"};
    }
}

uint64_t bytes_of(uint64_t bits) { return bits / 8 + (bits % 8 != 0 ? 1 : 0); }

void layout_or_throw(uint64_t count, const Format& in, Layout* out) {
    Format f = in;
    if (f.middle_group_log2 == 0 || f.middle_group_log2 > 5) {
        throw Fail{kInvalidArgument, "middle_group_log2 must be between 1 and 5"};
    }
    if (f.middle_placement > 2) {
        throw Fail{kInvalidArgument, "invalid middle placement"};
    }
    if (f.input_cluster_count > 64 || f.output_cluster_count > 64) {
        throw Fail{kInvalidArgument, "cluster depths do not span every routing level"};
    }
    const uint32_t leaf = 1u << f.middle_group_log2;
    const uint32_t depth = routing_depth(count, leaf);
    if (f.input_cluster_count == 0) {
        f.input_cluster_count = balanced_clusters(depth, f.input_clusters);
    }
    if (f.output_cluster_count == 0) {
        f.output_cluster_count = balanced_clusters(depth, f.output_clusters);
    }
    check_clusters(f.input_clusters, f.input_cluster_count, depth);
    check_clusters(f.output_clusters, f.output_cluster_count, depth);
    if (depth == 0) {
        f.middle_placement = 0;
    }
    Sizes sizes(leaf);
    Layout L;
    L.format = f;
    L.size = count;
    L.depth = depth;
    L.switch_bits = sizes.switches(count);
    L.middle_bits = sizes.middle(count);
    L.header_bytes = add(20, (uint64_t)f.input_cluster_count + f.output_cluster_count);
    const uint64_t in_bytes = add(bytes_of(L.switch_bits),
        f.middle_placement == 1 ? bytes_of(L.middle_bits) : 0);
    const uint64_t out_bytes = add(bytes_of(L.switch_bits),
        f.middle_placement == 2 ? bytes_of(L.middle_bits) : 0);
    const uint64_t mid_bytes = f.middle_placement == 0 ? bytes_of(L.middle_bits) : 0;
    if (count > (1ull << 63)) {
        throw Fail{kOverflow, "logical network size is too large"};
    }
    uint64_t width = leaf;
    while (width < count) {
        width <<= 1;
    }
    L.network_size = width;
    L.input_offset = L.header_bytes;
    L.output_offset = add(L.header_bytes, in_bytes);
    L.middle_offset = add(L.output_offset, out_bytes);
    L.end_offset = add(L.middle_offset, mid_bytes);
    *out = L;
}

} // namespace

Error make_layout(uint64_t count, const Format& format, Layout* out) {
    try {
        layout_or_throw(count, format, out);
        return {};
    } catch (const Fail& f) {
        return {f.code, f.message};
    }
}

void write_header(const Layout& L, uint8_t* out) {
    static const uint8_t magic[8] = {'B', 'E', 'N', 'E', 'S', '0', '1', 0};
    std::memcpy(out, magic, 8);
    for (int i = 0; i < 8; ++i) {
        out[8 + i] = (uint8_t)(L.size >> (8 * i));
    }
    out[16] = L.format.middle_placement;
    out[17] = L.format.middle_group_log2;
    out[18] = L.format.input_cluster_count;
    out[19] = L.format.output_cluster_count;
    std::memcpy(out + 20, L.format.input_clusters, L.format.input_cluster_count);
    std::memcpy(out + 20 + L.format.input_cluster_count, L.format.output_clusters,
        L.format.output_cluster_count);
}

Error make_plan(const Layout& L, uint64_t tile_max, Plan* out) {
    try {
        Plan& p = *out;
        std::memset(&p, 0, sizeof p);
        const uint64_t n = L.size;
        const uint32_t leaf = 1u << L.format.middle_group_log2;
        if (L.depth > kMaxLevels - 1) {
            throw Fail{kLength, "permutation is too large for the B200 backend"};
        }
        Sizes sizes(leaf);
        p.n = n;
        p.leaf = leaf;
        p.depth = L.depth;
        p.placement = L.format.middle_placement;
        p.section_offset[0] = L.input_offset;
        p.section_offset[1] = L.output_offset;
        p.section_offset[2] = L.middle_offset;
        p.end_offset = L.end_offset;
        p.switch_bits = L.switch_bits;
        p.middle_bits = L.middle_bits;

        for (uint32_t l = 0; l <= L.depth; ++l) {
            LevelInfo& lv = p.levels[l];
            lv.q = n >> l;
            lv.r = n & ((1ull << l) - 1);
            lv.cap = lv.q + (lv.r != 0 ? 1 : 0);
            lv.pcap = (lv.cap + 1) / 2;
            for (int big = 0; big < 2; ++big) {
                const uint64_t c = lv.q + (uint64_t)big;
                lv.middle[big] = sizes.middle(c);
                for (int side = 0; side < 2; ++side) {
                    const bool embeds = L.format.middle_placement == (uint8_t)(side + 1);
                    lv.section[side][big] = sizes.switches(c) + (embeds ? sizes.middle(c) : 0);
                }
            }
        }

        for (int side = 0; side < 2; ++side) {
            const uint8_t* cl = side == 0 ? L.format.input_clusters : L.format.output_clusters;
            const uint32_t gc = side == 0 ? L.format.input_cluster_count : L.format.output_cluster_count;
            p.group_count[side] = gc;
            uint32_t start = 0;
            for (uint32_t g = 0; g < gc; ++g) {
                GroupInfo& gi = p.groups[side][g];
                gi.start = start;
                gi.depth = cl[g];
                for (int big = 0; big < 2; ++big) {
                    const uint64_t root = p.levels[start].q + (uint64_t)big;
                    gi.group_bits[big] = sizes.top_switches(root, gi.depth);
                    uint64_t bits = 0;
                    for (uint32_t l = 0; l < gi.depth; ++l) {
                        bits += packet_path_bits(root, gi.depth, l, 0, 1ull << l, leaf);
                    }
                    gi.packet_bits[big] = bits;
                }
                start += gi.depth;
            }
            for (uint32_t l = 0; l <= L.depth && gc > 0; ++l) {
                uint32_t g = 0;
                while (g + 1 < gc && p.groups[side][g + 1].start <= l) {
                    ++g;
                }
                const GroupInfo& gi = p.groups[side][g];
                LevelSide& ls = p.levels[l].side[side];
                ls.group = g;
                ls.rel = l - gi.start;
                if (ls.rel >= gi.depth) {
                    continue; // leaf level past the last group: no switches
                }
                for (int rb = 0; rb < 2; ++rb) {
                    const uint64_t root = p.levels[gi.start].q + (uint64_t)rb;
                    uint64_t f0 = 0;
                    for (uint32_t up = 0; up < ls.rel; ++up) {
                        f0 += packet_path_bits(root, gi.depth, up, 0, 1ull << up, leaf);
                    }
                    ls.prefix0[rb] = f0;
                    for (int nb = 0; nb < 2; ++nb) {
                        const uint64_t pairs = (p.levels[l].q + (uint64_t)nb) / 2;
                        const uint64_t tail = pairs == 0 ? 0 : (pairs - 1) >> (gi.depth - ls.rel - 1);
                        uint64_t ft = 0;
                        for (uint32_t up = 0; up < ls.rel; ++up) {
                            ft += packet_path_bits(root, gi.depth, up, tail, 1ull << up, leaf);
                        }
                        ls.prefix_tail[rb][nb] = ft;
                    }
                }
            }
        }

        uint32_t tile = 0;
        while (tile < L.depth && p.levels[tile].cap > tile_max) {
            ++tile;
        }
        p.tile_level = tile;
        uint64_t slots = 0, pairs = 0;
        for (uint32_t l = 0; l <= tile; ++l) {
            const uint64_t s = (1ull << l) * p.levels[l].cap;
            const uint64_t q = (1ull << l) * p.levels[l].pcap;
            slots = s > slots ? s : slots;
            pairs = q > pairs ? q : pairs;
        }
        p.max_slots = slots;
        p.max_pairs = pairs;
        for (uint32_t c = 0; c <= 32; ++c) {
            p.fact_bits[c] = factoradic_bits(c);
        }
        return {};
    } catch (const Fail& f) {
        return {f.code, f.message};
    }
}

} // namespace bpb200
