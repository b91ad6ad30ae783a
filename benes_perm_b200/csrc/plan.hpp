// SPDX-License-Identifier: Apache-2.0
//
// Per-call plan for the B200 compact encoder, shared by host and device.
//
// Level-synchronous view of the reference's recursive network
// (src/benes.cpp:189-351): level l holds 2^l nodes in left-to-right order.
// Splitting a count into ceil/floor halves makes every node at level l hold
// q_l = floor(N / 2^l) entries, plus one more when the bit-reversal of its
// left-to-right index is below r_l = N mod 2^l.  Every quantity the
// reference derives by walking SectionAddress::child
// (src/internal.hpp:553-601) therefore has a closed form in (level, node):
// the functions below evaluate those closed forms, so no per-node host
// descriptor tree (the reference's make_compact_tree64,
// src/internal.hpp:908-1003) is ever built.
//
// In device memory a level is stored "padded": node j occupies slots
// [j * cap_l, j * cap_l + size), cap_l = ceil(N / 2^l); its pair-nodes
// (one per input pair, plus the odd tail) occupy [j * pcap_l, ...),
// pcap_l = ceil(cap_l / 2).  Children of node j are nodes 2j and 2j+1 of
// level l+1, so padded offsets need no prefix sums.
#pragma once

#include <cstddef>
#include <cstdint>

#if defined(__CUDACC__)
#define BP_HD __host__ __device__ __forceinline__
#else
#define BP_HD inline
#endif

namespace bpb200 {

constexpr int kMaxLevels = 64;
constexpr int kMaxGroups = 64;

// One cluster group of one section (a run of `depth` routing levels whose
// switches are packed together, README.md:119-123).
struct GroupInfo {
    uint32_t start;           // first routing level of the group
    uint32_t depth;           // levels in the group
    uint64_t group_bits[2];   // switch bits in the group's packets, root small/large
    uint64_t packet_bits[2];  // bits of one full packet, root small/large
};

// Per-level, per-section constants.
struct LevelSide {
    uint32_t group;             // group holding this level (last group for the leaf level)
    uint32_t rel;               // level - group.start
    uint64_t prefix0[2];        // bits of packet 0 from the group's levels above, by root size
    uint64_t prefix_tail[2][2]; // same for the node's tail packet, [root size][node size]
};

struct LevelInfo {
    uint64_t q;            // small node size
    uint64_t r;            // number of large (q + 1) nodes
    uint64_t cap;          // padded slots per node = ceil(N / 2^l)
    uint64_t pcap;         // padded pair-nodes per node = ceil(cap / 2)
    uint64_t middle[2];    // middle bits of a small / large node's subtree
    uint64_t section[2][2];// [section][small/large]: switch bits + embedded middle bits
    LevelSide side[2];     // 0 = input section, 1 = output section
};

struct Plan {
    uint64_t n;
    uint32_t leaf;         // 2^middle_group_log2
    uint32_t depth;        // routing depth D: every node at level D is a leaf
    uint32_t placement;    // 0 separate, 1 embedded_input, 2 embedded_output
    uint32_t tile_level;   // first level processed by the shared-memory tile kernel
    uint32_t group_count[2];
    uint32_t pad_;
    uint64_t section_offset[3]; // byte offsets of input, output and middle sections
    uint64_t end_offset;
    uint64_t switch_bits;
    uint64_t middle_bits;
    uint64_t max_slots;         // max over levels of 2^l * cap_l
    uint64_t max_pairs;         // max over levels of 2^l * pcap_l
    uint32_t fact_bits[33];     // ceil(log2(c!)) for c = 0..32
    // Subtree sharding: with shards = 2^shard_level > 1 this call encodes
    // every node of the levels above shard_level and, from shard_level on,
    // only the subtree of node `shard` of level shard_level (see
    // level_nodes).  0 or 1: the whole permutation.
    uint32_t shards;
    uint32_t shard;
    uint32_t shard_level;
    GroupInfo groups[2][kMaxGroups];
    LevelInfo levels[kMaxLevels + 1];
};

// The nodes of `level` this call encodes: [lo, lo + 2^shift).  Without
// sharding, and above the shard level, every node of the level; from the
// shard level on, the 2^(level - shard_level) descendants of node `shard`
// of the shard level, which are consecutive and aligned.
struct NodeRange {
    uint64_t lo;
    uint32_t shift;
};

BP_HD NodeRange level_nodes(const Plan& p, uint32_t level) {
    if (p.shards <= 1 || level < p.shard_level) {
        return NodeRange{0, level};
    }
    return NodeRange{(uint64_t)p.shard << (level - p.shard_level), level - p.shard_level};
}

// ---------------------------------------------------------------- bit math

BP_HD uint64_t reverse_bits(uint64_t x, uint32_t width) {
    if (width == 0) {
        return 0;
    }
#if defined(__CUDA_ARCH__)
    return __brevll(x) >> (64 - width);
#else
    uint64_t r = 0;
    for (uint32_t i = 0; i < width; ++i) {
        r = (r << 1) | ((x >> i) & 1);
    }
    return r;
#endif
}

BP_HD uint32_t high_bit(uint64_t x) {
#if defined(__CUDA_ARCH__)
    return 63u - (uint32_t)__clzll((long long)x);
#else
    return 63u - (uint32_t)__builtin_clzll(x);
#endif
}

// Number of node indices j in [0, paths) at `width` levels below a root
// whose bit-reversed index is below `large`, i.e. how many of the first
// `paths` nodes are the larger size.  [0, paths) is split into aligned
// blocks by the set bits of `paths`; inside a block the free low bits
// become the high bits of the reversal, so each block's count is one
// ceiling division.
BP_HD uint64_t count_large(uint64_t paths, uint32_t width, uint64_t large) {
    if (paths == 0 || large == 0) {
        return 0;
    }
    uint64_t total = 0;
    uint64_t rest = paths;
    while (rest != 0) {
        const uint32_t b = high_bit(rest);
        rest &= ~(1ull << b);
        const uint32_t fixed = width - b; // bits fixed by the block prefix
        const uint64_t prefix = (paths >> b) & ~1ull;
        const uint64_t low = reverse_bits(prefix, fixed);
        if (large > low) {
            const uint64_t step = 1ull << fixed;
            uint64_t n = (large - low + step - 1) >> fixed;
            const uint64_t block = 1ull << b;
            total += n < block ? n : block;
        }
    }
    return total;
}

BP_HD bool node_is_large(const LevelInfo& lv, uint32_t level, uint64_t node) {
    return reverse_bits(node, level) < lv.r;
}

BP_HD uint64_t node_size(const LevelInfo& lv, uint32_t level, uint64_t node) {
    return lv.q + (node_is_large(lv, level, node) ? 1 : 0);
}

// Bits that the first `paths` nodes at relative level `rel` of a cluster
// group of depth `depth`, rooted at a node of `root` entries, put into
// packet `packet` (src/internal.hpp:611-649).
BP_HD uint64_t packet_path_bits(uint64_t root, uint32_t depth, uint32_t rel,
    uint64_t packet, uint64_t paths, uint32_t leaf) {
    const uint64_t small = root >> rel;
    const uint64_t large = root & ((1ull << rel) - 1);
    const uint64_t span = 1ull << (depth - rel - 1);
    const uint64_t first = packet * span;
    uint64_t share[2];
    for (int big = 0; big < 2; ++big) {
        const uint64_t count = small + (uint64_t)big;
        const uint64_t pairs = count / 2;
        if (count <= leaf || first >= pairs) {
            share[big] = 0;
        } else {
            share[big] = pairs - first < span ? pairs - first : span;
        }
    }
    const uint64_t nl = count_large(paths, rel, large);
    return nl * share[1] + (paths - nl) * share[0];
}

// Separate-placement middle bit offset of the subtree of node `node` at
// `level`: middle bits of every node to its left.  Level l - 1 always holds
// all of its 2^(l-1) nodes, so the parent's level is summed in closed form.
BP_HD uint64_t middle_prefix(const Plan& p, uint32_t level, uint64_t node) {
    if (level == 0) {
        return 0;
    }
    const LevelInfo& up = p.levels[level - 1];
    const uint64_t parent = node >> 1;
    const uint64_t nl = count_large(parent, level - 1, up.r);
    uint64_t bits = parent * up.middle[0] + nl * (up.middle[1] - up.middle[0]);
    if (node & 1) {
        const uint64_t psize = node_size(up, level - 1, parent);
        const uint64_t left = psize - psize / 2;
        const LevelInfo& lv = p.levels[level];
        // the left sibling has either lv.q or lv.q + 1 entries
        bits += lv.middle[left == lv.q ? 0 : 1];
    }
    return bits;
}

// Section bits (switches + embedded middle) of all level-`level` nodes in
// [first, node).  `level` is always a complete level here.
BP_HD uint64_t section_span(const Plan& p, int side, uint32_t level,
    uint64_t first, uint64_t node) {
    const LevelInfo& lv = p.levels[level];
    const uint64_t nl = count_large(node, level, lv.r) - count_large(first, level, lv.r);
    return (node - first) * lv.section[side][0] +
        nl * (lv.section[side][1] - lv.section[side][0]);
}

// First bit of the packets of group `g` for the cluster root that is the
// ancestor of node `node` at `level` (SectionAddress::packet_base after the
// chain of child() calls that reaches that root).
BP_HD uint64_t cluster_base(const Plan& p, int side, uint32_t g, uint32_t level,
    uint64_t node) {
    uint64_t base = 0;
    for (uint32_t h = 1; h <= g; ++h) {
        const GroupInfo& up = p.groups[side][h - 1];
        const uint32_t s = p.groups[side][h].start;
        const uint64_t root = node >> (level - s);        // ancestor at level s
        const uint64_t parent = node >> (level - up.start); // ancestor at up.start
        const bool parent_large = node_is_large(p.levels[up.start], up.start, parent);
        base += up.group_bits[parent_large ? 1 : 0] +
            section_span(p, side, s, parent << up.depth, root);
    }
    return base;
}

// Everything needed to place the switch bits of one internal node.
struct NodeAddress {
    uint64_t base;        // first bit of the node's cluster packets
    uint64_t packet_bits; // bits in one full packet
    uint64_t full_prefix; // offset of the node's run inside a full packet
    uint64_t tail_prefix; // offset of the node's run inside its tail packet
    uint64_t tail_packet;
    uint32_t span_log2;   // pairs of this node per packet = 2^span_log2
    uint32_t pad_;
};

// SectionAddress state of node `node` at routing level `level` for one
// section (src/internal.hpp:475-718), in closed form.
BP_HD NodeAddress node_address(const Plan& p, int side, uint32_t level, uint64_t node) {
    const LevelInfo& lv = p.levels[level];
    const LevelSide& ls = lv.side[side];
    const GroupInfo& gi = p.groups[side][ls.group];
    const uint32_t rel = ls.rel;
    const uint64_t root = node >> rel;
    const uint64_t path = node & ((1ull << rel) - 1);
    const bool root_large = node_is_large(p.levels[gi.start], gi.start, root);
    const int rs = root_large ? 1 : 0;
    const uint64_t root_count = p.levels[gi.start].q + (uint64_t)rs;
    const bool large = node_is_large(lv, level, node);
    const uint64_t size = lv.q + (large ? 1 : 0);
    NodeAddress a;
    a.base = cluster_base(p, side, ls.group, level, node);
    a.packet_bits = gi.packet_bits[rs];
    a.span_log2 = gi.depth - rel - 1;
    const uint64_t pairs = size / 2;
    a.tail_packet = pairs == 0 ? 0 : (pairs - 1) >> a.span_log2;
    a.full_prefix = ls.prefix0[rs] +
        packet_path_bits(root_count, gi.depth, rel, 0, path, p.leaf);
    a.tail_prefix = ls.prefix_tail[rs][large ? 1 : 0] +
        packet_path_bits(root_count, gi.depth, rel, a.tail_packet, path, p.leaf);
    a.pad_ = 0;
    return a;
}

// Section-relative bit of switch `pair` (SwitchBitAddress::bit,
// src/internal.hpp:464-472).
BP_HD uint64_t switch_bit(const NodeAddress& a, uint64_t pair) {
    const uint64_t packet = pair >> a.span_log2;
    return a.base + packet * a.packet_bits +
        (packet == a.tail_packet ? a.tail_prefix : a.full_prefix) +
        (pair & ((1ull << a.span_log2) - 1));
}

// Section-relative first bit of the factoradic rank of leaf `node` at
// `level` (middle_bit_offset for separate placement, or
// SectionAddress::middle_bit, src/internal.hpp:506-517, when embedded).
// Returns the section index through *section.
BP_HD uint64_t leaf_rank_bit(const Plan& p, uint32_t level, uint64_t node, int* section) {
    const uint64_t mid = middle_prefix(p, level, node);
    if (p.placement == 0) {
        *section = 2;
        return mid;
    }
    const int side = p.placement == 1 ? 0 : 1;
    *section = side;
    const uint32_t gcount = p.group_count[side];
    uint32_t g = 0;
    while (g + 1 < gcount && p.groups[side][g + 1].start <= level) {
        ++g;
    }
    const GroupInfo& gi = p.groups[side][g];
    const uint64_t root = node >> (level - gi.start);
    const bool root_large = node_is_large(p.levels[gi.start], gi.start, root);
    uint64_t bit = cluster_base(p, side, g, level, node);
    if (level > gi.start) {
        bit += gi.group_bits[root_large ? 1 : 0];
    }
    return bit + mid - middle_prefix(p, gi.start, root);
}

} // namespace bpb200
