// SPDX-License-Identifier: Apache-2.0
//
// Forward and inverse lookup of one index in a compact blob, shared by the
// device verifier kernel (lookup.inc) and a host test probe.
//
// Restates the reference's read path, lookup() in src/internal.hpp:1035-1124:
// descend from the root reading one switch per level (input section for a
// forward lookup, output section for an inverse one), decode the leaf's
// factoradic rank, then climb back reading the switches of the other
// section.  On the closed-form plan the node reached at level l is the
// string of left/right turns taken so far (children of node j are 2j and
// 2j + 1), so the climb recomputes each ancestor and its turn from the leaf
// node's index instead of keeping the reference's frame stack.
#pragma once

#include "plan.hpp"

namespace bpb200 {

// Status bits of one lookup (ORed over a batch).
enum LookupStatus : uint32_t {
    kLookupOk = 0,
    kLookupOutOfRange = 1u, // index >= size (std::out_of_range in the reference)
    kLookupTruncated = 2u,  // a bit address fell outside the blob
    kLookupBadPlan = 4u,    // descent ran past the routing depth
};

struct BlobBits {
    const uint8_t* data;
    uint64_t len; // bytes
};

// Bit `bit` (LSB-first) of the section starting at byte `offset`
// (read_bit, src/internal.hpp:1005-1013).
BP_HD uint32_t blob_bit(const BlobBits& b, uint64_t offset, uint64_t bit, uint32_t* status) {
    const uint64_t byte = offset + (bit >> 3);
    if (byte >= b.len) {
        *status |= kLookupTruncated;
        return 0;
    }
    return (uint32_t)(b.data[byte] >> (bit & 7)) & 1u;
}

// `bits` (<= 128) bits from bit `first` of the section at byte `offset`,
// LSB-first into lo/hi (read_rank, src/internal.hpp:1015-1033), a byte at
// a time.
BP_HD void blob_rank(const BlobBits& b, uint64_t offset, uint64_t first, uint32_t bits,
    uint64_t* lo, uint64_t* hi, uint32_t* status) {
    *lo = 0;
    *hi = 0;
    uint32_t i = 0;
    while (i < bits) {
        const uint64_t at = first + i;
        const uint64_t byte = offset + (at >> 3);
        if (byte >= b.len) {
            *status |= kLookupTruncated;
            return;
        }
        const uint32_t shift = (uint32_t)(at & 7);
        uint32_t take = 8 - shift;
        if (take > bits - i) {
            take = bits - i;
        }
        const uint64_t v = (uint64_t)((b.data[byte] >> shift) & ((1u << take) - 1));
        if (i < 64) {
            *lo |= v << i;
            if (i + take > 64) {
                *hi |= v >> (64 - i);
            }
        } else {
            *hi |= v << (i - 64);
        }
        i += take;
    }
}

// (lo, hi) /= d in place for 1 <= d <= 32; returns the remainder.  Long
// division over 32-bit limbs: the running remainder stays below d, so each
// step's dividend fits in 37 bits.
BP_HD uint32_t divide_small(uint64_t* lo, uint64_t* hi, uint32_t d) {
    uint64_t rem = 0;
    uint64_t limb[4] = {*hi >> 32, *hi & 0xffffffffull, *lo >> 32, *lo & 0xffffffffull};
    for (int k = 0; k < 4; ++k) {
        const uint64_t cur = (rem << 32) | limb[k];
        limb[k] = cur / d;
        rem = cur % d;
    }
    *hi = (limb[0] << 32) | limb[1];
    *lo = (limb[2] << 32) | limb[3];
    return (uint32_t)rem;
}

// Position of the (k+1)-th lowest set bit of `mask` (k < popcount(mask)).
BP_HD uint32_t nth_set_bit(uint32_t mask, uint32_t k) {
    for (uint32_t i = 0; i < k; ++i) {
        mask &= mask - 1;
    }
#if defined(__CUDA_ARCH__)
    return (uint32_t)__ffs(mask) - 1;
#else
    return (uint32_t)__builtin_ctz(mask);
#endif
}

// Leaf step of the lookup: the local permutation of `size` (<= 32) entries
// encoded by the factoradic rank (lo, hi), applied forward to `index`
// (p[index]) or inverted (the i with p[i] == index).
//
// The rank is the mixed-radix number with digits d[i] = #{k < i : p[k] <
// p[i]}, radix i + 1 (encode_factoradic, src/internal.hpp:148-167), so the
// lowest digit is d[size-1].  Peeling digits from the top entry down, p[i]
// is the d[i]-th smallest value not yet taken by an entry above i; the peel
// stops as soon as the wanted entry is known.
BP_HD uint32_t leaf_apply(uint64_t lo, uint64_t hi, uint32_t size, uint32_t index, bool inverse) {
    uint32_t free_values = size >= 32 ? 0xffffffffu : ((1u << size) - 1);
    for (uint32_t i = size; i-- > 0;) {
        const uint32_t digit = divide_small(&lo, &hi, i + 1);
        const uint32_t value = nth_set_bit(free_values, digit);
        free_values &= ~(1u << value);
        if (!inverse && i == index) {
            return value;
        }
        if (inverse && value == index) {
            return i;
        }
    }
    return 0; // unreachable for index < size
}

// Forward (p[value]) or inverse (p^-1[value]) lookup.  Returns a
// LookupStatus; *out is valid when it is kLookupOk.
BP_HD uint32_t lookup_one(const Plan& p, const BlobBits& blob, uint64_t value, bool inverse,
    uint64_t* out) {
    if (value >= p.n) {
        return kLookupOutOfRange;
    }
    uint32_t status = 0;
    const int down = inverse ? 1 : 0; // section read on the way down
    const int up = 1 - down;
    uint64_t index = value;
    uint64_t node = 0;
    uint64_t size = p.n;
    uint32_t level = 0;
    while (size > p.leaf) {
        if (level >= p.depth) {
            return kLookupBadPlan;
        }
        bool right = false;
        if ((size & 1) == 0 || index != size - 1) { // the odd tail passes straight left
            const uint64_t bit = switch_bit(node_address(p, down, level, node), index >> 1);
            right = blob_bit(blob, p.section_offset[down], bit, &status) != (uint32_t)(index & 1);
        }
        index >>= 1;
        node = 2 * node + (right ? 1 : 0);
        ++level;
        size = node_size(p.levels[level], level, node);
    }
    int section = 0;
    const uint64_t rank_bit = leaf_rank_bit(p, level, node, &section);
    uint64_t lo = 0, hi = 0;
    blob_rank(blob, p.section_offset[section], rank_bit, p.fact_bits[size], &lo, &hi, &status);
    index = leaf_apply(lo, hi, (uint32_t)size, (uint32_t)index, inverse);
    for (uint32_t l = level; l-- > 0;) {
        const uint64_t at = node >> (level - l);
        const uint32_t right = (uint32_t)(node >> (level - 1 - l)) & 1u;
        const uint64_t count = node_size(p.levels[l], l, at);
        if (right == 0 && (count & 1) != 0 && index == count / 2) {
            index = count - 1; // back out through the odd tail
            continue;
        }
        const uint64_t bit = switch_bit(node_address(p, up, l, at), index);
        index = 2 * index + (right ^ blob_bit(blob, p.section_offset[up], bit, &status));
    }
    *out = index;
    return status;
}

} // namespace bpb200
