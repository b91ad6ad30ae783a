// SPDX-License-Identifier: Apache-2.0
//
// sm_100a kernels of the compact encoder.
//
// Level kernels (global memory) run one routing level over every node of
// the level at once; they are used while nodes are larger than a tile.
// The tile kernel takes one node per CTA into shared memory and finishes
// its whole subtree there, down to the middle-group ranks.
//
// Per internal node and level (src/benes.cpp:226-315):
//   inverse      inv[p[i]] = i (node-local)
//   union        one parity union per output pair (inv[2k], inv[2k+1]) on
//                pair-nodes: colour(u) != colour(w) becomes
//                x(u/2) ^ x(w/2) = 1 ^ (u&1) ^ (w&1), x(k) = colour(2k)
//   orient       odd nodes: flip the tail's component so the tail is colour 0
//   resolve      x(k) = parity to the component minimum (the canonical
//                colouring: each component's smallest vertex gets colour 0);
//                children left[k] = p[2k+x]/2, right[k] = p[2k+1-x]/2; the
//                input switch of pair k is x(k)
//   output bits  output switch of pair k is colour(inv[2k])
#pragma once

#include "device.cuh"
#include "plan.hpp"

#include <cstdint>

namespace bpb200 {

constexpr uint32_t kNodeWave = 256;   // node descriptors held in shared memory at once
constexpr uint32_t kTileThreads = 512;

struct TileShape {
    uint32_t slots;   // padded entry slots needed at the deepest level
    uint32_t pairs;   // padded pair-node slots needed
    uint32_t smem;    // dynamic shared memory bytes
};

// ------------------------------------------------------------ level kernels

template <typename T>
__global__ void __launch_bounds__(256) level_inverse(const Plan* __restrict__ plan,
    uint32_t level, const T* __restrict__ src, uint32_t* __restrict__ inv,
    uint32_t* __restrict__ uf, uint32_t* status) {
    const LevelInfo& lv = plan->levels[level];
    const uint32_t cap = (uint32_t)lv.cap;
    const uint32_t pcap = (uint32_t)lv.pcap;
    const uint64_t total = (uint64_t)cap << level;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += stride) {
        const uint32_t j = (uint32_t)(e / cap);
        const uint32_t i = (uint32_t)(e - (uint64_t)j * cap);
        const uint32_t s = (uint32_t)node_size(lv, level, j);
        if (i >= s) {
            continue;
        }
        const uint64_t v = (uint64_t)src[e];
        if (v >= s) {
            atomicOr(status, kErrNotPermutation);
            continue;
        }
        inv[(uint64_t)j * cap + v] = i;
        if ((i & 1u) == 0) {
            const uint32_t id = j * pcap + (i >> 1);
            uf[id] = id << 1;
        }
    }
}

__global__ void __launch_bounds__(256) level_union(const Plan* __restrict__ plan,
    uint32_t level, const uint32_t* __restrict__ inv, uint32_t* uf, uint32_t* status) {
    const LevelInfo& lv = plan->levels[level];
    const uint32_t cap = (uint32_t)lv.cap;
    const uint32_t pcap = (uint32_t)lv.pcap;
    const uint64_t total = (uint64_t)pcap << level;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < total; p += stride) {
        const uint32_t j = (uint32_t)(p / pcap);
        const uint32_t k = (uint32_t)(p - (uint64_t)j * pcap);
        const uint32_t s = (uint32_t)node_size(lv, level, j);
        if (k >= s / 2) {
            continue;
        }
        const uint32_t u = inv[(uint64_t)j * cap + 2 * k];
        const uint32_t w = inv[(uint64_t)j * cap + 2 * k + 1];
        if (u >= s || w >= s) {
            atomicOr(status, kErrNotPermutation);
            continue;
        }
        const uint32_t base = j * pcap;
        uf_union(uf, base + (u >> 1), base + (w >> 1), 1u ^ (u & 1u) ^ (w & 1u), status);
    }
}

__global__ void level_orient(const Plan* __restrict__ plan, uint32_t level,
    const uint32_t* __restrict__ inv, uint32_t* uf, uint32_t* status) {
    const LevelInfo& lv = plan->levels[level];
    const uint32_t cap = (uint32_t)lv.cap;
    const uint32_t pcap = (uint32_t)lv.pcap;
    const uint64_t nodes = 1ull << level;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nodes;
         j += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t s = (uint32_t)node_size(lv, level, j);
        if ((s & 1u) == 0) {
            continue;
        }
        if (inv[j * cap + s - 1] >= s) {
            atomicOr(status, kErrNotPermutation);
            continue;
        }
        const Found f = uf_find(uf, (uint32_t)j * pcap + (s >> 1), status);
        if (f.bit) {
            atomicOr(uf + f.root, 1u);
        }
    }
}

__global__ void level_descriptors(const Plan* __restrict__ plan, uint32_t level,
    NodeAddress* __restrict__ in_addr, NodeAddress* __restrict__ out_addr) {
    const uint64_t nodes = 1ull << level;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nodes;
         j += (uint64_t)gridDim.x * blockDim.x) {
        in_addr[j] = node_address(*plan, 0, level, j);
        out_addr[j] = node_address(*plan, 1, level, j);
    }
}

template <typename T>
__global__ void __launch_bounds__(256) level_resolve(const Plan* __restrict__ plan,
    uint32_t level, const T* __restrict__ src, uint32_t* uf, uint32_t* __restrict__ xbits,
    uint32_t* __restrict__ dst, const NodeAddress* __restrict__ in_addr,
    uint32_t* __restrict__ blob, uint32_t* status) {
    const LevelInfo& lv = plan->levels[level];
    const uint32_t cap = (uint32_t)lv.cap;
    const uint32_t pcap = (uint32_t)lv.pcap;
    const uint32_t ccap = (uint32_t)plan->levels[level + 1].cap;
    const uint64_t total = (uint64_t)pcap << level;
    const uint64_t section_bit = plan->section_offset[0] * 8;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    // Every warp walks whole 32-slot chunks so the ballot covers one word.
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p - (threadIdx.x & 31) < total;
         p += stride) {
        const bool in_range = p < total;
        uint32_t j = 0, k = 0, s = 0;
        bool live = false;
        if (in_range) {
            j = (uint32_t)(p / pcap);
            k = (uint32_t)(p - (uint64_t)j * pcap);
            s = (uint32_t)node_size(lv, level, j);
            live = k < s - s / 2;
        }
        uint32_t x = 0;
        if (live) {
            const Found f = uf_find(uf, (uint32_t)p, status);
            x = f.bit ^ (uf_load(uf, f.root) & 1u);
        }
        const unsigned word = __ballot_sync(0xffffffffu, x != 0);
        if ((threadIdx.x & 31) == 0) {
            xbits[p >> 5] = word;
        }
        const uint32_t half = s / 2;
        if (live) {
            const uint64_t node = (uint64_t)j * cap;
            const uint64_t left = (uint64_t)(2 * j) * ccap;
            const uint64_t right = (uint64_t)(2 * j + 1) * ccap;
            if (k < half) {
                const uint32_t a = (uint32_t)src[node + 2 * k + x];
                const uint32_t b = (uint32_t)src[node + 2 * k + 1 - x];
                dst[left + k] = a >> 1;
                dst[right + k] = b >> 1;
            } else {
                dst[left + k] = (uint32_t)(src[node + s - 1] >> 1);
            }
        }
        const bool has_switch = live && k < half;
        uint64_t bit = 0;
        if (has_switch) {
            bit = section_bit + switch_bit(in_addr[j], k);
        }
        emit_bit(blob, bit, has_switch && x != 0, 0xffffffffu);
    }
}

__global__ void __launch_bounds__(256) level_output_bits(const Plan* __restrict__ plan,
    uint32_t level, const uint32_t* __restrict__ inv, const uint32_t* __restrict__ xbits,
    const NodeAddress* __restrict__ out_addr, uint32_t* __restrict__ blob) {
    const LevelInfo& lv = plan->levels[level];
    const uint32_t cap = (uint32_t)lv.cap;
    const uint32_t pcap = (uint32_t)lv.pcap;
    const uint64_t total = (uint64_t)pcap << level;
    const uint64_t section_bit = plan->section_offset[1] * 8;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p - (threadIdx.x & 31) < total;
         p += stride) {
        bool has_switch = false;
        bool y = false;
        uint64_t bit = 0;
        if (p < total) {
            const uint32_t j = (uint32_t)(p / pcap);
            const uint32_t k = (uint32_t)(p - (uint64_t)j * pcap);
            const uint32_t s = (uint32_t)node_size(lv, level, j);
            if (k < s / 2) {
                const uint32_t u = inv[(uint64_t)j * cap + 2 * k];
                if (u < s) {
                    const uint64_t q = (uint64_t)j * pcap + (u >> 1);
                    y = (((xbits[q >> 5] >> (q & 31)) ^ u) & 1u) != 0;
                    has_switch = true;
                    bit = section_bit + switch_bit(out_addr[j], k);
                }
            }
        }
        emit_bit(blob, bit, has_switch && y, 0xffffffffu);
    }
}

} // namespace bpb200
