// SPDX-License-Identifier: Apache-2.0
//
// Tile kernel: one CTA per node of the tile level; the node's whole subtree
// (every remaining routing level plus the middle-group ranks) is encoded in
// shared memory.  Node-local values fit 16 bits (a tile holds at most a few
// thousand entries), union-find words are 32-bit shared-memory words.
#pragma once

#include "device.cuh"
#include "kernels.cuh"
#include "plan.hpp"

#include <cstdint>

namespace bpb200 {

__host__ __device__ inline uint32_t align_up(uint32_t x, uint32_t a) { return (x + a - 1) / a * a; }

// Division by a per-level constant: floor(n / d) = umulhi(n, ceil(2^32 / d))
// exactly whenever n * d < 2^32 (the rounding error n * (m - 2^32/d) / 2^32
// stays below 1/d), which holds for tile indices: n and d are below 2^16.
struct FastDiv {
    uint32_t d, m;
    __device__ explicit FastDiv(uint32_t div)
        : d(div), m(div > 1 ? (uint32_t)((0x100000000ull + div - 1) / div) : 0u) {}
    __device__ __forceinline__ uint32_t operator()(uint32_t n) const {
        return d > 1 ? __umulhi(n, m) : n;
    }
};

// Byte offsets of the smem arrays; identical on host (sizing) and device.
__host__ __device__ inline uint32_t tile_smem_layout(uint32_t slots, uint32_t pairs,
    uint32_t* off) {
    const uint32_t words = (pairs + 31) / 32 + 1;
    uint32_t o = 0;
    off[0] = o; o = align_up(o + slots * 2, 16);           // vals[0]
    off[1] = o; o = align_up(o + slots * 2, 16);           // vals[1]
    off[2] = o; o = align_up(o + slots * 2, 16);           // inv[0]
    off[3] = o; o = align_up(o + pairs * 4, 16);           // uf
    off[4] = o; o = align_up(o + words * 4, 16);           // xbits (input switches)
    off[5] = o; o = align_up(o + words * 4, 16);           // ybits (output switches)
    off[6] = o; o = align_up(o + 2 * kNodeWave * (uint32_t)sizeof(NodeAddress), 16);
    off[7] = o; o = align_up(o + kNodeWave * 8, 16);       // leafbit
    off[8] = o; o = align_up(o + slots * 2, 16);           // inv[1]
    return o;
}

// Uniform-level fast path for node sizes in the tile (1) or size_at everywhere (0).
#ifndef BPB200_TILE_UNIFORM
#define BPB200_TILE_UNIFORM 1
#endif

// Tile input through one bulk asynchronous copy (1) or batched plain loads (0).
#ifndef BPB200_TILE_BULK_LOAD
#define BPB200_TILE_BULK_LOAD 0
#endif
constexpr uint32_t kBulkWaitCap = 1u << 22; // mbarrier polls before giving up

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Bounded wait for phase 0 of `mbar`; true once the phase has completed.
__device__ __forceinline__ bool bulk_wait(uint32_t mbar) {
    for (uint32_t it = 0; it < kBulkWaitCap; ++it) {
        uint32_t done = 0;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done) : "r"(mbar), "r"(0u) : "memory");
        if (done) return true;
    }
    return false;
}

// Copies the s0 32-bit input values at `in` into `stage` (16-byte aligned,
// at least s0 * 4 + 16 bytes, free until the caller is done with it): the
// 16-byte-aligned interior of the range with one cp.async.bulk counted on an
// mbarrier, the ragged ends (at most three values each) with plain loads, so
// nothing outside the range is read.  Value i lands at stage[lead + i];
// returns lead, or ~0u when the copy did not complete within the poll bound
// (the status word then says so).  Every thread of the block calls it.
__device__ __forceinline__ uint32_t tile_bulk_stage(const uint32_t* in, uint32_t s0,
    uint32_t* stage, uint64_t* mbar, uint32_t* status) {
    const uint64_t g0 = (uint64_t)in;
    const uint64_t g1 = g0 + (uint64_t)s0 * 4;
    const uint64_t a0 = (g0 + 15) & ~15ull;
    const uint64_t a1 = g1 & ~15ull;
    const uint32_t lead = (uint32_t)((g0 & 15) >> 2);
    const bool bulk = a1 > a0;
    const uint32_t mb = smem_addr(mbar);
    if (threadIdx.x == 0 && bulk) {
        const uint32_t bytes = (uint32_t)(a1 - a0);
        const uint32_t dst = smem_addr(stage) + (uint32_t)(a0 - (g0 & ~15ull));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(mb) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                     :: "r"(mb), "r"(bytes) : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
                     "[%0], [%1], %2, [%3];"
                     :: "r"(dst), "l"(a0), "r"(bytes), "r"(mb) : "memory");
    }
    // ragged ends: values before a0 and from a1 on (all of them without bulk)
    const uint32_t head = bulk ? (uint32_t)((a0 - g0) >> 2) : s0;
    const uint32_t tail = bulk ? (uint32_t)((a1 - g0) >> 2) : s0;
    for (uint32_t i = threadIdx.x; i < head; i += blockDim.x) stage[lead + i] = in[i];
    for (uint32_t i = tail + threadIdx.x; i < s0; i += blockDim.x) stage[lead + i] = in[i];
    __syncthreads(); // the mbarrier is initialised before anyone polls it
    const bool ok = !bulk || bulk_wait(mb);
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) atomicOr(status, kErrIterationCap);
        bulk_wait(mb); // give the copy in flight one more bounded chance
        __syncthreads();
        return ~0u;
    }
    return lead;
}

template <typename T>
__device__ __forceinline__ void tile_body(const Plan* __restrict__ plan_ptr,
    const T* __restrict__ src, uint32_t* __restrict__ blob, uint32_t* status, uint32_t slots,
    uint32_t pairs, uint32_t tile, unsigned char* smem) {
    uint32_t off[9];
    tile_smem_layout(slots, pairs, off);
    uint16_t* vals[2] = {(uint16_t*)(smem + off[0]), (uint16_t*)(smem + off[1])};
    uint16_t* invs[2] = {(uint16_t*)(smem + off[2]), (uint16_t*)(smem + off[8])};
    uint32_t* uf = (uint32_t*)(smem + off[3]);
    uint32_t* xbits = (uint32_t*)(smem + off[4]);
    uint32_t* ybits = (uint32_t*)(smem + off[5]);
    NodeAddress* desc = (NodeAddress*)(smem + off[6]);
    uint64_t* leafbit = (uint64_t*)(smem + off[7]);

    const Plan& plan = *plan_ptr;
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31;
    const uint32_t warp = tid >> 5;
    const uint32_t nwarps = blockDim.x >> 5;
    const uint32_t T0 = plan.tile_level;
    const uint32_t D = plan.depth;
    const uint32_t leaf = plan.leaf;
    const uint32_t J = tile;

    if (T0 > 0 && size_at(plan.levels[T0 - 1], T0 - 1, J >> 1) <= leaf) {
        return; // child of a leaf: not part of the tree
    }
    {
        const LevelInfo& l0 = plan.levels[T0];
        const uint32_t s0 = size_at(l0, T0, J);
        const T* in = src + (uint64_t)J * l0.cap;
        bool loaded = false;
#if BPB200_TILE_BULK_LOAD
        if (sizeof(T) == 4 && s0 >= 256) {
            // staged over vals[1], inv[0] and the union-find words, which
            // phase A fills only after the conversion below
            __shared__ uint64_t bulk_bar;
            uint32_t* stage = (uint32_t*)(smem + off[1]);
            const uint32_t lead = tile_bulk_stage((const uint32_t*)in, s0, stage, &bulk_bar,
                status);
            if (lead == ~0u) {
                return;
            }
            for (uint32_t i = tid; i < s0; i += blockDim.x) {
                const uint32_t v = stage[lead + i];
                if (v >= s0) {
                    atomicOr(status, kErrNotPermutation);
                    vals[0][i] = 0;
                } else {
                    vals[0][i] = (uint16_t)v;
                }
            }
            loaded = true;
        }
#endif
        // every load of a batch is issued before any is used: the error
        // atomic below may alias the input as far as the compiler knows, so
        // a plain loop would wait out one HBM round trip per element
        constexpr int kBatch = 8;
        for (uint32_t i0 = tid; !loaded && i0 < s0; i0 += kBatch * blockDim.x) {
            uint64_t v[kBatch];
#pragma unroll
            for (int q = 0; q < kBatch; ++q) {
                const uint32_t i = i0 + q * blockDim.x;
                v[q] = i < s0 ? (uint64_t)__ldcs(in + i) : 0;
            }
#pragma unroll
            for (int q = 0; q < kBatch; ++q) {
                const uint32_t i = i0 + q * blockDim.x;
                if (i >= s0) {
                    break;
                }
                if (v[q] >= s0) {
                    atomicOr(status, kErrNotPermutation);
                    vals[0][i] = 0;
                } else {
                    vals[0][i] = (uint16_t)v[q];
                }
            }
        }
    }
    __syncthreads();

    for (uint32_t t = 0;; ++t) {
        const uint32_t level = T0 + t;
        const LevelInfo& lv = plan.levels[level];
        const uint32_t cap = (uint32_t)lv.cap;
        const uint32_t pcap = (uint32_t)lv.pcap;
        const FastDiv by_cap(cap), by_pcap(pcap);
        const uint32_t nodes = 1u << t;
        const uint32_t first = J << t;
        uint16_t* cur = vals[t & 1];
        uint16_t* nxt = vals[(t + 1) & 1];
        uint16_t* inv = invs[t & 1];        // this level's inverse
        uint16_t* child_inv = invs[(t + 1) & 1];
        // uniform per level: whether every node here exists / is internal
        const bool all_exist = level == 0 || plan.levels[level - 1].q > leaf;
        const bool all_internal = lv.q > leaf && all_exist;
        // node sizes: every node of a level without large nodes (r = 0, all
        // levels of a power-of-two count) has q entries
#if BPB200_TILE_UNIFORM
        const uint32_t q32 = (uint32_t)lv.q;
        const bool uniform = lv.r == 0;
        auto node_size = [&](uint32_t node) {
            return uniform ? q32 : size_at(lv, level, node);
        };
#else
        auto node_size = [&](uint32_t node) { return size_at(lv, level, node); };
#endif
        auto internal_node = [&](uint32_t path, uint32_t s) {
            if (all_internal) return true;
            if (s <= leaf) return false;
            return all_exist || size_at(plan.levels[level - 1], level - 1, (first + path) >> 1) > leaf;
        };

        if (level < D) {
            if (t == 0 && T0 == 0) {
                // the whole permutation is in this tile: mark inverse slots so
                // duplicates show up as never-written entries
                for (uint32_t e = tid; e < cap; e += blockDim.x) {
                    inv[e] = 0xffffu;
                }
                __syncthreads();
            }
            // A (first tile level only; every later level's inverse and
            // union-find roots come from its parent's phase E0): inverse
            // and union-find init
            for (uint32_t e = tid; t == 0 && e < nodes * cap; e += blockDim.x) {
                const uint32_t path = by_cap(e);
                const uint32_t i = e - path * cap;
                const uint32_t s = node_size(first + path);
                if (i >= s || !internal_node(path, s)) {
                    continue;
                }
                if ((i & 1u) == 0) { // every pair-node is a root, whatever its values
                    const uint32_t id = path * pcap + (i >> 1);
                    uf[id] = id << 1;
                }
                const uint32_t v = cur[e];
                if (v >= s) {
                    atomicOr(status, kErrNotPermutation);
                    continue;
                }
                inv[path * cap + v] = (uint16_t)i;
            }
            __syncthreads();
            // B: one union per output pair.  Consecutive threads take the
            // same pair of consecutive nodes, so the unions running at once
            // spread over all nodes of the level instead of crowding one
            // node's few roots (with 16 nodes of 256 pair-nodes, node-major
            // order ran all 256 unions of a node at once; tile time at 2^30
            // entries 157 -> 145 ms).
            for (uint32_t idx = tid; idx < nodes * pcap; idx += blockDim.x) {
                const uint32_t path = idx & (nodes - 1);
                const uint32_t k = idx >> t;
                const uint32_t s = node_size(first + path);
                if (k >= s / 2 || !internal_node(path, s)) {
                    continue;
                }
                const uint32_t u = inv[path * cap + 2 * k];
                const uint32_t w = inv[path * cap + 2 * k + 1];
                if (u >= s || w >= s) {
                    atomicOr(status, kErrNotPermutation);
                    continue;
                }
                const uint32_t base = path * pcap;
                uf_union(uf, base + (u >> 1), base + (w >> 1), 1u ^ (u & 1u) ^ (w & 1u), status);
            }
            __syncthreads();
            // C: orient odd nodes so the unpaired tail gets colour 0
            for (uint32_t path = tid; path < nodes; path += blockDim.x) {
                const uint32_t s = node_size(first + path);
                if ((s & 1u) == 0 || !internal_node(path, s)) {
                    continue;
                }
                if (inv[path * cap + s - 1] >= s) {
                    atomicOr(status, kErrNotPermutation);
                    continue;
                }
                const Found f = uf_find(uf, path * pcap + (s >> 1), status);
                if (f.bit) {
                    atomicOr(uf + f.root, 1u);
                }
            }
            __syncthreads();
            // D: colours, child scatter
            const uint32_t ccap = (uint32_t)plan.levels[level + 1].cap;
            const uint32_t ptotal = nodes * pcap;
            for (uint32_t base = warp * 32; base < ptotal; base += nwarps * 32) {
                const uint32_t p = base + lane;
                uint32_t x = 0;
                if (p < ptotal) {
                    const uint32_t path = by_pcap(p);
                    const uint32_t k = p - path * pcap;
                    const uint32_t s = node_size(first + path);
                    if (k < s - s / 2 && internal_node(path, s)) {
                        const Found f = uf_find(uf, p, status);
                        x = f.bit ^ (uf_load(uf, f.root) & 1u);
                        const uint32_t node = path * cap;
                        const uint32_t half = s / 2;
                        if (k < half) {
                            nxt[2 * path * ccap + k] = (uint16_t)(cur[node + 2 * k + x] >> 1);
                            nxt[(2 * path + 1) * ccap + k] = (uint16_t)(cur[node + 2 * k + 1 - x] >> 1);
                        } else {
                            nxt[2 * path * ccap + k] = (uint16_t)(cur[node + s - 1] >> 1);
                        }
                    }
                }
                const unsigned word = __ballot_sync(0xffffffffu, x != 0);
                if (lane == 0) {
                    xbits[base >> 5] = word;
                }
            }
            __syncthreads();
            // E0: output switch bits in natural order, and the children's
            // inverse and union-find roots (as level_outputs does for the
            // global levels: output pair k's colour-0 input inv[2k + y]
            // goes left with value k, the other right)
            const uint32_t ccpcap = (uint32_t)plan.levels[level + 1].pcap;
            for (uint32_t base = warp * 32; base < ptotal; base += nwarps * 32) {
                const uint32_t p = base + lane;
                bool y = false;
                if (p < ptotal) {
                    const uint32_t path = by_pcap(p);
                    const uint32_t k = p - path * pcap;
                    const uint32_t s = node_size(first + path);
                    const uint32_t half = s / 2;
                    if (k <= half && internal_node(path, s)) {
                        const uint32_t lb = 2 * path * ccap;
                        const uint32_t rb = lb + ccap;
                        if (k < half) {
                            const uint32_t u = inv[path * cap + 2 * k];
                            const uint32_t w = inv[path * cap + 2 * k + 1];
                            uint16_t to_left = 0xffffu, to_right = 0xffffu;
                            if (u < s && w < s) { // an unwritten slot (repeated value) holds anything
                                const uint32_t q = path * pcap + (u >> 1);
                                y = (((xbits[q >> 5] >> (q & 31)) ^ u) & 1u) != 0;
                                to_left = (uint16_t)((y ? w : u) >> 1);
                                to_right = (uint16_t)((y ? u : w) >> 1);
                            }
                            child_inv[lb + k] = to_left;
                            child_inv[rb + k] = to_right;
                        } else if ((s & 1u) != 0) {
                            const uint32_t u = inv[path * cap + s - 1];
                            child_inv[lb + half] = u < s ? (uint16_t)(u >> 1) : (uint16_t)0xffffu;
                        }
                        if ((k & 1u) == 0) {
                            if (k < s - half) {
                                const uint32_t id = 2 * path * ccpcap + (k >> 1);
                                uf[id] = id << 1;
                            }
                            if (k < half) {
                                const uint32_t id = (2 * path + 1) * ccpcap + (k >> 1);
                                uf[id] = id << 1;
                            }
                        }
                    }
                }
                const unsigned word = __ballot_sync(0xffffffffu, y);
                if (lane == 0) {
                    ybits[base >> 5] = word;
                }
            }
            __syncthreads();
            // E: switch bits, packet-major over a wave of node descriptors
            const uint32_t wave_log2 = t < kNodeWaveLog2 ? t : kNodeWaveLog2; // log2(min(nodes, kNodeWave))
            const uint32_t wn = 1u << wave_log2;
            for (uint32_t w0 = 0; w0 < nodes; w0 += wn) {
                if (tid < 2 * wn) {
                    const uint32_t slot = tid >> 1;
                    const int side = (int)(tid & 1);
                    const uint32_t node = first + w0 + slot;
                    const uint32_t s = node_size(node);
                    if (internal_node(w0 + slot, s)) {
                        desc[side * kNodeWave + slot] = node_address(plan, side, level, node);
                    }
                }
                __syncthreads();
                for (int side = 0; side < 2; ++side) {
                    const LevelSide& ls = lv.side[side];
                    const uint32_t span_log2 = plan.groups[side][ls.group].depth - ls.rel - 1;
                    const uint32_t shift = wave_log2 + span_log2;
                    const uint32_t packets = (cap / 2 + (1u << span_log2) - 1) >> span_log2;
                    const uint32_t* bits = side == 0 ? xbits : ybits;
                    const uint64_t sec = plan.section_offset[side] * 8;
                    if (span_log2 >= 5) {
                        // runs of at least 32 switches: word-wise copies as in
                        // level_emit_words (the bit arrays keep a spare word)
                        const uint32_t cshift = span_log2 - 5;
                        const uint32_t cs = wave_log2 + cshift;
                        const uint32_t chunks = packets << cs;
                        for (uint32_t c = tid; c < chunks; c += blockDim.x) {
                            const uint32_t packet = c >> cs;
                            const uint32_t rem = c & ((1u << cs) - 1);
                            const uint32_t slot = rem >> cshift;
                            const uint32_t pair0 =
                                (packet << span_log2) + ((rem & ((1u << cshift) - 1)) << 5);
                            const uint32_t path = w0 + slot;
                            const uint32_t s = node_size(first + path);
                            if (pair0 >= s / 2 || !internal_node(path, s)) {
                                continue;
                            }
                            const uint32_t q = path * pcap + pair0;
                            uint32_t v = __funnelshift_r(bits[q >> 5], bits[(q >> 5) + 1], q & 31);
                            if (s / 2 - pair0 < 32) {
                                v &= (1u << (s / 2 - pair0)) - 1u;
                            }
                            if (v == 0) {
                                continue;
                            }
                            const uint64_t dest =
                                sec + switch_bit(desc[side * kNodeWave + slot], pair0);
                            const uint32_t off = (uint32_t)(dest & 31);
                            atomicOr(blob + (dest >> 5), v << off);
                            if (off != 0 && (v >> (32 - off)) != 0) {
                                atomicOr(blob + (dest >> 5) + 1, v >> (32 - off));
                            }
                        }
                        continue;
                    }
                    // short runs: the packets every node fills go out as
                    // word blocks (see level_emit_blocks), the rest bit by bit
                    uint32_t full = 0;
                    if (all_internal && lv.q / 2 >= 1) {
                        full = (uint32_t)(((lv.q / 2) - 1) >> span_log2);
                    }
                    if (full > packets) {
                        full = packets;
                    }
                    if (full > 0) {
                        const uint32_t rel = ls.rel;
                        // nodes per word: within a word, a cluster root and the wave
                        uint32_t g_log2 = 5 - span_log2;
                        g_log2 = g_log2 < rel ? g_log2 : rel;
                        g_log2 = g_log2 < wave_log2 ? g_log2 : wave_log2;
                        const uint32_t span_mask = (1u << (1u << span_log2)) - 1u;
                        const uint32_t groups_log2 = wave_log2 - g_log2;
                        const uint32_t work = full << groups_log2;
                        for (uint32_t c = tid; c < work; c += blockDim.x) {
                            const uint32_t packet = c >> groups_log2;
                            const uint32_t slot0 = (c & ((1u << groups_log2) - 1)) << g_log2;
                            uint32_t v = 0;
                            for (uint32_t i = 0; i < (1u << g_log2); ++i) {
                                const uint32_t q = (w0 + slot0 + i) * pcap + (packet << span_log2);
                                const uint32_t field =
                                    __funnelshift_r(bits[q >> 5], bits[(q >> 5) + 1], q & 31) &
                                    span_mask;
                                v |= field << (i << span_log2);
                            }
                            if (v == 0) {
                                continue;
                            }
                            const uint64_t dest = sec +
                                switch_bit(desc[side * kNodeWave + slot0], packet << span_log2);
                            const uint32_t off = (uint32_t)(dest & 31);
                            atomicOr(blob + (dest >> 5), v << off);
                            if (off != 0 && (v >> (32 - off)) != 0) {
                                atomicOr(blob + (dest >> 5) + 1, v >> (32 - off));
                            }
                        }
                    }
                    const uint32_t rest = (packets - full) << shift;
                    for (uint32_t base = warp * 32; base < rest; base += nwarps * 32) {
                        const uint32_t tt = base + lane;
                        bool set = false;
                        uint64_t dest = 0;
                        if (tt < rest) {
                            const uint32_t packet = full + (tt >> shift);
                            const uint32_t rem = tt & ((1u << shift) - 1);
                            const uint32_t slot = rem >> span_log2;
                            const uint32_t pair = (packet << span_log2) + (rem & ((1u << span_log2) - 1));
                            const uint32_t path = w0 + slot;
                            const uint32_t s = node_size(first + path);
                            if (pair < s / 2 && internal_node(path, s)) {
                                const uint32_t q = path * pcap + pair;
                                set = ((bits[q >> 5] >> (q & 31)) & 1u) != 0;
                                if (set) {
                                    dest = sec + switch_bit(desc[side * kNodeWave + slot], pair);
                                }
                            }
                        }
                        emit_bit(blob, dest, set, 0xffffffffu);
                    }
                }
                __syncthreads();
            }
        }

        // leaves at this level (all of level D, and the size-`leaf` nodes of a
        // mixed level D - 1)
        if (lv.q <= leaf) {
            for (uint32_t w0 = 0; w0 < nodes; w0 += kNodeWave) {
                const uint32_t wn = nodes - w0 < kNodeWave ? nodes - w0 : kNodeWave;
                if (tid < wn) {
                    const uint32_t node = first + w0 + tid;
                    uint64_t v = ~0ull;
                    const bool exists = all_exist ||
                        size_at(plan.levels[level - 1], level - 1, node >> 1) > leaf;
                    if (node_size(node) <= leaf && exists) {
                        int section = 0;
                        const uint64_t bit = leaf_rank_bit(plan, level, node, &section);
                        v = plan.section_offset[section] * 8 + bit;
                    }
                    leafbit[tid] = v;
                }
                __syncthreads();
                for (uint32_t li = warp; li < wn; li += nwarps) {
                    const uint64_t at = leafbit[li];
                    if (at == ~0ull) {
                        continue;
                    }
                    const uint32_t path = w0 + li;
                    const uint32_t s = node_size(first + path);
                    const uint32_t v = lane < s ? (uint32_t)cur[path * cap + lane] : 0u;
                    if (lane < s && v >= s) {
                        atomicOr(status, kErrNotPermutation);
                    }
                    bool distinct = true;
                    const U128 rank = warp_factoradic_rank(v < s ? v : 0u, s, &distinct);
                    if (!distinct && lane == 0) {
                        atomicOr(status, kErrNotPermutation);
                    }
                    emit_rank(blob, at, plan.fact_bits[s], rank);
                }
                __syncthreads();
            }
        }
        if (level >= D) {
            break;
        }
    }
}

// One permutation: one CTA per node of the tile level.
template <typename T>
__global__ void __launch_bounds__(kTileThreads, 2) tile_encode(const Plan* __restrict__ plan,
    const T* __restrict__ src, uint32_t* __restrict__ blob, uint32_t* status, uint32_t slots,
    uint32_t pairs, uint32_t part_first) {
    extern __shared__ __align__(16) unsigned char smem[];
    // a sharded call encodes only its own tiles (level_nodes); a launch may
    // cover a part of them, from tile part_first on
    const uint32_t first = (uint32_t)level_nodes(*plan, plan->tile_level).lo + part_first;
    tile_body<T>(plan, src, blob, status, slots, pairs, first + blockIdx.x, smem);
}

// Tiles too large for two CTAs per SM (nodes of 16384 entries, up to about
// 200 KB of shared memory): one CTA of twice the threads per SM keeps the
// same number of resident warps.
template <typename T>
__global__ void __launch_bounds__(2 * kTileThreads, 1) tile_encode_wide(
    const Plan* __restrict__ plan, const T* __restrict__ src, uint32_t* __restrict__ blob,
    uint32_t* status, uint32_t slots, uint32_t pairs, uint32_t part_first) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t first = (uint32_t)level_nodes(*plan, plan->tile_level).lo + part_first;
    tile_body<T>(plan, src, blob, status, slots, pairs, first + blockIdx.x, smem);
}

// Tiles of many permutations in one launch (the batched and serving forms):
// job k owns blocks [first_block, first_block + tiles); the launch's dynamic
// shared memory covers the largest job.
// A job whose permutation is a single tile (tile level 0) also clears its
// blob, writes the header and resets its status word first: its CTA is the
// only writer of that blob.
struct TileJob {
    const Plan* plan;
    const void* src;
    uint32_t* blob;
    uint32_t* status;
    uint32_t slots;
    uint32_t pairs;
    uint32_t first_block;
    uint32_t tiles;
    uint32_t blob_words;   // words to clear (single-tile jobs)
    uint32_t header_bytes;
    uint8_t header[84];
};

template <typename T>
__global__ void __launch_bounds__(kTileThreads, 2) tile_encode_batch(
    const TileJob* __restrict__ jobs, uint32_t njobs) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint32_t lo = 0, hi = njobs;
    while (hi - lo > 1) { // last job whose first block is <= blockIdx.x
        const uint32_t mid = (lo + hi) / 2;
        if (jobs[mid].first_block <= blockIdx.x) lo = mid; else hi = mid;
    }
    const TileJob& job = jobs[lo];
    if (job.tiles == 1 && job.blob_words != 0) {
        for (uint32_t i = threadIdx.x; i < job.blob_words; i += blockDim.x) job.blob[i] = 0;
        __syncthreads();
        uint8_t* b = reinterpret_cast<uint8_t*>(job.blob);
        for (uint32_t i = threadIdx.x; i < job.header_bytes; i += blockDim.x) b[i] = job.header[i];
        if (threadIdx.x == 0) *job.status = 0;
        __syncthreads();
    }
    tile_body<T>(job.plan, (const T*)job.src, job.blob, job.status, job.slots, job.pairs,
        blockIdx.x - job.first_block, smem);
}

} // namespace bpb200
