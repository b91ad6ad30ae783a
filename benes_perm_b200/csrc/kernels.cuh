// SPDX-License-Identifier: Apache-2.0
//
// sm_100a kernels of the compact encoder.
//
// Level kernels (global memory) run one routing level over every node of
// the level at once; they are used while nodes are larger than a tile.
// The tile kernel (tile.cuh) takes one node per CTA into shared memory and
// finishes its whole subtree there, down to the middle-group ranks.
//
// Per internal node and level (src/benes.cpp:226-315):
//   inverse      inv[p[i]] = i (node-local)
//   union        one parity union per output pair (inv[2k], inv[2k+1]) on
//                pair-nodes: colour(u) != colour(w) becomes
//                x(u/2) ^ x(w/2) = 1 ^ (u&1) ^ (w&1), x(k) = colour(2k)
//   orient       odd nodes: flip the tail's component so the tail is colour 0
//   finalize     (walk.cuh) x(k) = parity to the component minimum (the
//                canonical colouring: each component's smallest vertex gets
//                colour 0), or the orbit-walk colour on walk levels;
//                children left[k] = p[2k+x]/2, right[k] = p[2k+1-x]/2; the
//                input switch of pair k is x(k)
//   outputs      output switch of output pair k is colour(inv[2k]); the
//                children's inverses follow from the same two reads
//   emit         switch bits into the clustered blob layout: word copies of
//                long packet runs, word blocks of short ones, bits for the
//                rest
//
// The kernels are bound by memory latency and random-access throughput, not
// by instruction issue: their loops keep several independent loads per
// thread in flight.
#pragma once

#include "device.cuh"
#include "plan.hpp"

#include <cstdint>

namespace bpb200 {

constexpr uint32_t kNodeWaveLog2 = 6;
constexpr uint32_t kNodeWave = 1u << kNodeWaveLog2; // tile node descriptors held in shared memory at once
constexpr uint32_t kTileThreads = 512;
// 4 slots per thread measured fastest on B200 at 2^30 uniform entries
// (inverse kernels 207 ms per compress; 8: 227 ms; 16: 243 ms): more
// threads keep more of the scattered inverse stores in flight.
#ifndef BPB200_INVERSE_ITEMS
#define BPB200_INVERSE_ITEMS 4
#endif
constexpr int kInverseItems = BPB200_INVERSE_ITEMS; // slots per thread in level_inverse
// level_union shape: 2 output pairs per thread with at most 64 registers (4
// blocks of 256 per SM) measured fastest on B200 at 2^30 uniform entries
// (union kernels 253 ms per compress; 4 pairs at 100 registers: 304 ms;
// 8 pairs: 420 ms).  More resident warps hide more of the random latency.
#ifndef BPB200_UNION_ITEMS
#define BPB200_UNION_ITEMS 2
#endif
#ifndef BPB200_UNION_MIN_BLOCKS
#define BPB200_UNION_MIN_BLOCKS 4
#endif
constexpr int kUnionItems = BPB200_UNION_ITEMS; // output pairs per thread in level_union
// level_finalize shape: pair-nodes per thread (1, 2, 4 or 8; 32 / items lanes
// assemble one colour word) and the minimum resident blocks of 256 per SM.
// 2 pair-nodes at 8 blocks measured fastest on B200 at 2^30 uniform entries
// (finalize 115 ms per compress; 2 at 6 blocks: 120; 4 at 6 blocks: 144;
// 4 at the compiler's choice of 4 blocks: 134; 8: 286): the finds are
// latency-bound, so more resident warps beat more finds per thread.
#ifndef BPB200_RESOLVE_ITEMS
#define BPB200_RESOLVE_ITEMS 2
#endif
#ifndef BPB200_FINAL_MIN_BLOCKS
#define BPB200_FINAL_MIN_BLOCKS 8
#endif
constexpr int kResolveItems = BPB200_RESOLVE_ITEMS;
static_assert(kResolveItems == 1 || kResolveItems == 2 || kResolveItems == 4 ||
    kResolveItems == 8, "level_finalize assembles colour words from 1, 2, 4 or 8 bits per lane");

struct TileShape {
    uint32_t slots;   // padded entry slots needed at the deepest level
    uint32_t pairs;   // padded pair-node slots needed
    uint32_t smem;    // dynamic shared memory bytes
};

// 32-bit node-size test: every level here has fewer than 2^32 nodes.
__device__ __forceinline__ uint32_t size_at(const LevelInfo& lv, uint32_t level, uint32_t node) {
    const uint32_t rev = level == 0 ? 0u : (__brev(node) >> (32 - level));
    return (uint32_t)lv.q + ((uint64_t)rev < lv.r ? 1u : 0u);
}

// ------------------------------------------------------------ level kernels

template <typename T>
__device__ __forceinline__ void level_inverse_run(Grid grid, const Plan* __restrict__ plan,
    uint32_t level, const T* __restrict__ src, uint32_t* __restrict__ inv,
    uint32_t* __restrict__ uf, uint32_t* __restrict__ owner, uint32_t* claims, uint32_t* status) {
    const LevelInfo& lv = plan->levels[level];
    const uint32_t cap = (uint32_t)lv.cap;
    const uint32_t pcap = (uint32_t)lv.pcap;
    const uint64_t total = (uint64_t)cap << level;
    const bool aligned = ((uintptr_t)src & 15u) == 0;
    uint64_t first;
    while (claim_chunk(claims, (uint64_t)blockDim.x * kInverseItems, total, &first)) {
        const uint64_t e0 = first + (uint64_t)threadIdx.x * kInverseItems;
        if (e0 >= total) {
            continue;
        }
        T v[kInverseItems];
        if (aligned && e0 + kInverseItems <= total) {
            constexpr int kVec = 16 / sizeof(T);
#pragma unroll
            for (int q = 0; q < kInverseItems / kVec; ++q) {
                const uint4 chunk = __ldcs(reinterpret_cast<const uint4*>(src + e0) + q);
                const T* parts = reinterpret_cast<const T*>(&chunk);
#pragma unroll
                for (int r = 0; r < kVec; ++r) v[q * kVec + r] = parts[r];
            }
        } else {
#pragma unroll
            for (int q = 0; q < kInverseItems; ++q) {
                v[q] = e0 + q < total ? src[e0 + q] : (T)0;
            }
        }
        uint32_t j = (uint32_t)(e0 / cap);
        uint32_t i = (uint32_t)(e0 - (uint64_t)j * cap);
        uint32_t s = size_at(lv, level, j);
#pragma unroll
        for (int q = 0; q < kInverseItems; ++q) {
            if (e0 + q < total && i < s) {
                // every pair-node starts as its own root, whatever its values:
                // a stale word could point outside the array; and unowned
                if ((i & 1u) == 0) {
                    const uint32_t id = j * pcap + (i >> 1);
                    uf[id] = id << 1;
                    owner[id] = ~0u;
                }
                const uint64_t val = (uint64_t)v[q];
                if (val >= s) {
                    atomicOr(status, kErrNotPermutation);
                } else {
                    inv[(uint64_t)j * cap + val] = i;
                }
            }
            if (++i == cap) {
                i = 0;
                ++j;
                s = size_at(lv, level, j);
            }
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(256) level_inverse(const Plan* __restrict__ plan,
    uint32_t level, const T* __restrict__ src, uint32_t* __restrict__ inv,
    uint32_t* __restrict__ uf, uint32_t* __restrict__ owner, uint32_t* claims, uint32_t* status) {
    level_inverse_run<T>(launch_grid(), plan, level, src, inv, uf, owner, claims, status);
}

// ---------------------------------------------------------------------------
// Partitioned inverse for levels whose nodes do not fit in L2.  A plain
// scatter inv[p[i]] = i there costs one HBM read-modify-write of a 32-byte
// sector per entry (about 21 G entries/s on B200).  Instead:
//   level_bucket  streams the values once and appends (destination, i)
//                 records to the 2^kPlaceLog2-slot destination window they
//                 land in (block-local counts in shared memory, one global
//                 reservation per block and window);
//   level_place   replays each window's records; the writes of one window
//                 stay inside an L2-resident 32 MB range.
// Windows of 2^23 slots measured fastest on B200 at 2^30 uniform entries
// (2^21: 256 ms of inverse per compress, 2^22: 240, 2^23: 226): larger
// windows give each block longer runs of records per window.
// A window receives at most as many records as it has slots when the input
// is a permutation; an overfull window means a repeated value.
// ---------------------------------------------------------------------------
#ifndef BPB200_PLACE_LOG2
#define BPB200_PLACE_LOG2 24
#endif
constexpr uint32_t kPlaceLog2 = BPB200_PLACE_LOG2; // slots per destination window (log2)
constexpr uint32_t kMaxWindows = 2048;
static_assert((1ull << 31) >> kPlaceLog2 <= kMaxWindows, "windows must cover 2^31 slots");
constexpr int kBucketItems = 16;

#ifndef BPB200_BUCKET_THREADS
#define BPB200_BUCKET_THREADS 256
#endif
constexpr int kBucketThreads = BPB200_BUCKET_THREADS; // block size of level_bucket

template <typename T>
// Slots [e_lo, e_hi) of the level (the whole level, or one part of an input
// still being uploaded; e_lo a multiple of 4 so vector loads stay aligned).
__device__ __forceinline__ void level_bucket_run(Grid grid, const Plan* __restrict__ plan,
    uint32_t level, const T* __restrict__ src, uint2* __restrict__ records,
    uint32_t* __restrict__ cursor, uint32_t* __restrict__ uf, uint32_t* status,
    uint64_t e_lo, uint64_t e_hi) {
    __shared__ uint32_t count[kMaxWindows];
    __shared__ uint32_t start[kMaxWindows];
    const LevelInfo& lv = plan->levels[level];
    const uint32_t cap = (uint32_t)lv.cap;
    const uint32_t pcap = (uint32_t)lv.pcap;
    const uint64_t slots = (uint64_t)cap << level;
    const uint64_t total = e_hi < slots ? e_hi : slots;
    const uint32_t windows = (uint32_t)((slots + (1ull << kPlaceLog2) - 1) >> kPlaceLog2);
    const uint64_t chunk = (uint64_t)blockDim.x * kBucketItems;
    const bool aligned = ((uintptr_t)src & 15u) == 0 && (e_lo & 3u) == 0;
    for (uint64_t c0 = e_lo + (uint64_t)grid.bid * chunk; c0 < total;
         c0 += (uint64_t)grid.nblk * chunk) {
        for (uint32_t b = threadIdx.x; b < windows; b += blockDim.x) count[b] = 0;
        __syncthreads();
        const uint64_t e0 = c0 + (uint64_t)threadIdx.x * kBucketItems;
        uint32_t dest[kBucketItems], idx[kBucketItems];
        T v[kBucketItems];
        if (aligned && e0 + kBucketItems <= total) {
            constexpr int kVec = 16 / sizeof(T);
#pragma unroll
            for (int q = 0; q < kBucketItems / kVec; ++q) {
                const uint4 part = __ldcs(reinterpret_cast<const uint4*>(src + e0) + q);
                const T* parts = reinterpret_cast<const T*>(&part);
#pragma unroll
                for (int r = 0; r < kVec; ++r) v[q * kVec + r] = parts[r];
            }
        } else {
#pragma unroll
            for (int q = 0; q < kBucketItems; ++q) v[q] = e0 + q < total ? src[e0 + q] : (T)0;
        }
        uint32_t j = (uint32_t)(e0 < total ? e0 / cap : 0);
        uint32_t i = (uint32_t)(e0 < total ? e0 - (uint64_t)j * cap : 0);
        uint32_t s = size_at(lv, level, j);
#pragma unroll
        for (int q = 0; q < kBucketItems; ++q) {
            dest[q] = ~0u;
            if (e0 + q < total && i < s) {
                if ((i & 1u) == 0) { // unconditional: see level_inverse
                    const uint32_t id = j * pcap + (i >> 1);
                    uf[id] = id << 1;
                }
                const uint64_t val = (uint64_t)v[q];
                if (val >= s) {
                    atomicOr(status, kErrNotPermutation);
                } else {
                    dest[q] = j * cap + (uint32_t)val;
                    idx[q] = i;
                    atomicAdd(&count[dest[q] >> kPlaceLog2], 1u);
                }
            }
            if (++i == cap) {
                i = 0;
                ++j;
                s = size_at(lv, level, j);
            }
        }
        __syncthreads();
        for (uint32_t b = threadIdx.x; b < windows; b += blockDim.x) {
            if (count[b] != 0) start[b] = atomicAdd(cursor + b, count[b]);
            count[b] = 0;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < kBucketItems; ++q) {
            if (dest[q] == ~0u) continue;
            const uint32_t b = dest[q] >> kPlaceLog2;
            const uint64_t at = ((uint64_t)b << kPlaceLog2) + start[b] + atomicAdd(&count[b], 1u);
            if (at < slots && at < ((uint64_t)(b + 1) << kPlaceLog2)) {
                records[at] = make_uint2(dest[q], idx[q]);
            } else {
                atomicOr(status, kErrNotPermutation); // more values than slots: a repeat
            }
        }
        __syncthreads();
    }
}

template <typename T>
__global__ void __launch_bounds__(BPB200_BUCKET_THREADS) level_bucket(const Plan* __restrict__ plan,
    uint32_t level, const T* __restrict__ src, uint2* __restrict__ records,
    uint32_t* __restrict__ cursor, uint32_t* __restrict__ uf, uint32_t* status,
    uint64_t e_lo, uint64_t e_hi) {
    level_bucket_run<T>(launch_grid(), plan, level, src, records, cursor, uf, status, e_lo, e_hi);
}

constexpr int kPlaceItems = 16;

__device__ __forceinline__ void level_place_run(Grid grid, const Plan* __restrict__ plan,
    uint32_t level, const uint2* __restrict__ records, const uint32_t* __restrict__ cursor,
    uint32_t* __restrict__ inv, uint32_t* claims) {
    const LevelInfo& lv = plan->levels[level];
    const uint64_t total = lv.cap << level;
    const uint64_t chunk = (uint64_t)blockDim.x * kPlaceItems;
    uint64_t first;
    while (claim_chunk(claims, chunk, total, &first)) {
#pragma unroll
        for (int q = 0; q < kPlaceItems; ++q) {
            const uint64_t at = first + (uint64_t)q * blockDim.x + threadIdx.x;
            if (at >= total) break;
            const uint32_t b = (uint32_t)(at >> kPlaceLog2);
            if ((at & ((1ull << kPlaceLog2) - 1)) < cursor[b]) {
                const uint2 r = __ldcs(records + at);
                inv[r.x] = r.y;
            }
        }
    }
}

__global__ void __launch_bounds__(256) level_place(const Plan* __restrict__ plan,
    uint32_t level, const uint2* __restrict__ records, const uint32_t* __restrict__ cursor,
    uint32_t* __restrict__ inv, uint32_t* claims) {
    level_place_run(launch_grid(), plan, level, records, cursor, inv, claims);
}

// Blocks claim chunks of output pairs in address order (claim_chunk), so the
// union-find words being linked at any time belong to the few nodes those
// chunks cover: once a node's words fit in L2 the random finds hit there.
// `hard` was written by earlier launches: all threads see the same value.
__device__ __forceinline__ void level_union_run(Grid grid, const Plan* __restrict__ plan,
    uint32_t level, const uint32_t* __restrict__ inv, uint32_t* uf, const uint32_t* hard,
    uint32_t* claims, uint32_t* status) {
    if (hard != nullptr && *hard == 0) {
        return; // the orbit walks coloured this level
    }
    const LevelInfo& lv = plan->levels[level];
    const uint32_t cap = (uint32_t)lv.cap;
    const uint32_t pcap = (uint32_t)lv.pcap;
    const NodeRange nr = level_nodes(*plan, level);
    const uint64_t begin = nr.lo * pcap;
    const uint64_t total = (uint64_t)pcap << nr.shift;
    const uint64_t end = begin + total;
    uint64_t first;
    auto next = [&]() -> bool {
        return claim_chunk(claims, (uint64_t)blockDim.x * kUnionItems, total, &first);
    };
    while (next()) {
        const uint64_t p0 = begin + first + (uint64_t)threadIdx.x * kUnionItems;
        if (p0 >= end) {
            continue;
        }
        uint32_t j = (uint32_t)(p0 / pcap);
        uint32_t k = (uint32_t)(p0 - (uint64_t)j * pcap);
        uint32_t s = size_at(lv, level, j);
        uint32_t a[kUnionItems], b[kUnionItems], rel[kUnionItems];
        uint32_t u[kUnionItems], w[kUnionItems], base[kUnionItems];
        uint32_t pending = 0;
#pragma unroll
        for (int q = 0; q < kUnionItems; ++q) {
            if (p0 + q < end && k < s / 2) {
                pending |= 1u << q;
                const uint64_t at = (uint64_t)j * cap + 2 * k;
                u[q] = inv[at];
                w[q] = inv[at + 1];
                base[q] = j * pcap;
                rel[q] = s; // stash the node size for the range check below
            }
            if (++k == pcap) {
                k = 0;
                ++j;
                s = size_at(lv, level, j);
            }
        }
#pragma unroll
        for (int q = 0; q < kUnionItems; ++q) {
            if (pending & (1u << q)) {
                if (u[q] >= rel[q] || w[q] >= rel[q]) {
                    atomicOr(status, kErrNotPermutation);
                    pending &= ~(1u << q);
                    continue;
                }
                a[q] = base[q] + (u[q] >> 1);
                b[q] = base[q] + (w[q] >> 1);
                rel[q] = 1u ^ (u[q] & 1u) ^ (w[q] & 1u);
            }
        }
        uf_union_many<kUnionItems>(uf, a, b, rel, pending, status);
    }
}

__global__ void __launch_bounds__(256, BPB200_UNION_MIN_BLOCKS) level_union(const Plan* __restrict__ plan,
    uint32_t level, const uint32_t* __restrict__ inv, uint32_t* uf, const uint32_t* hard,
    uint32_t* claims, uint32_t* status) {
    level_union_run(launch_grid(), plan, level, inv, uf, hard, claims, status);
}

// Walk levels: their pair-nodes start as union-find roots only when the
// walks gave up (the `hard` flag) and the level falls back to union-find;
// the parent's output pass does not set them up for walk levels.
__global__ void __launch_bounds__(256) level_uf_reset(const Plan* __restrict__ plan,
    uint32_t level, uint32_t* __restrict__ uf, const uint32_t* hard) {
    if (*hard == 0) {
        return;
    }
    const LevelInfo& lv = plan->levels[level];
    const NodeRange nr = level_nodes(*plan, level);
    const uint64_t lo = nr.lo * lv.pcap;
    const uint64_t hi = lo + (lv.pcap << nr.shift);
    for (uint64_t id = lo + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; id < hi;
         id += (uint64_t)gridDim.x * blockDim.x) {
        uf[id] = (uint32_t)id << 1;
    }
}

// Test hook: the walks of the level ran, but the level is coloured by the
// union-find fallback anyway, as if a walk had given up.
__global__ void level_force_fallback(uint32_t* hard) {
    *hard = 1;
}

__device__ __forceinline__ void level_orient_run(Grid grid, const Plan* __restrict__ plan, uint32_t level,
    const uint32_t* __restrict__ inv, uint32_t* uf, const uint32_t* hard, uint32_t* status) {
    if (hard != nullptr && *hard == 0) {
        return;
    }
    const LevelInfo& lv = plan->levels[level];
    const uint32_t cap = (uint32_t)lv.cap;
    const uint32_t pcap = (uint32_t)lv.pcap;
    const NodeRange nr = level_nodes(*plan, level);
    const uint64_t nodes_end = nr.lo + (1ull << nr.shift);
    for (uint64_t j = nr.lo + (uint64_t)grid.bid * blockDim.x + threadIdx.x; j < nodes_end;
         j += (uint64_t)grid.nblk * blockDim.x) {
        const uint32_t s = size_at(lv, level, (uint32_t)j);
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

__global__ void level_orient(const Plan* __restrict__ plan, uint32_t level,
    const uint32_t* __restrict__ inv, uint32_t* uf, const uint32_t* hard, uint32_t* status) {
    level_orient_run(launch_grid(), plan, level, inv, uf, hard, status);
}

__device__ __forceinline__ void level_descriptors_run(Grid grid, const Plan* __restrict__ plan, uint32_t level,
    NodeAddress* __restrict__ in_addr, NodeAddress* __restrict__ out_addr) {
    const NodeRange nr = level_nodes(*plan, level);
    const uint64_t nodes_end = nr.lo + (1ull << nr.shift);
    for (uint64_t j = nr.lo + (uint64_t)grid.bid * blockDim.x + threadIdx.x; j < nodes_end;
         j += (uint64_t)grid.nblk * blockDim.x) {
        in_addr[j] = node_address(*plan, 0, level, j);
        out_addr[j] = node_address(*plan, 1, level, j);
    }
}

__global__ void level_descriptors(const Plan* __restrict__ plan, uint32_t level,
    NodeAddress* __restrict__ in_addr, NodeAddress* __restrict__ out_addr) {
    level_descriptors_run(launch_grid(), plan, level, in_addr, out_addr);
}

// Output side of a level, in natural (node, output pair) order: the output
// switch bits and the children's inverses, so no level below the first
// scatters an inverse.  Output pair k of node j joins outputs 2k and 2k+1,
// fed by inputs u0 = inv[2k] and u1 = inv[2k+1], whose colours differ.  Its
// switch bit is y = colour(u0) (src/benes.cpp:306-310: the output bit of
// input i is colour(i) ^ (p[i] & 1), and p[u0] = 2k).  Of the two, the
// colour-0 input inv[2k + y] is routed to the left child, where it sits at
// input pair inv[2k + y] >> 1 and carries value k (src/benes.cpp:313-314);
// the other goes right with the same value.  So
//     left_inv[k] = inv[2k + y] >> 1,  right_inv[k] = inv[2k + 1 - y] >> 1,
// and an odd node's tail output s - 1, whose input is coloured 0, gives
// left_inv[s / 2] = inv[s - 1] >> 1.  The pass reads inv sequentially and
// one colour bit per output pair, and writes the children's inverse
// sequentially.  It also resets the children's walk owners (one word per
// pair-node: the stamp of its even vertex, the only one the walks read) and
// pair-node union-find roots (`child_owner` / `child_uf`, may be null), the
// state the next level's colouring starts from.  A value out of range (only
// possible when the input was not a permutation, which level 0 reports)
// leaves 0xffffffff, which every user range-checks.
__device__ __forceinline__ void level_outputs_run(Grid grid, const Plan* __restrict__ plan,
    uint32_t level, const uint32_t* __restrict__ inv, const uint32_t* __restrict__ xbits,
    uint32_t* __restrict__ ybits, uint32_t* __restrict__ child_inv,
    uint32_t* __restrict__ child_owner, uint32_t* __restrict__ child_uf) {
    const LevelInfo& lv = plan->levels[level];
    const LevelInfo& cl = plan->levels[level + 1];
    const uint32_t cap = (uint32_t)lv.cap;
    const uint32_t pcap = (uint32_t)lv.pcap;
    const uint32_t ccap = (uint32_t)cl.cap;
    const uint32_t cpcap = (uint32_t)cl.pcap;
    // this call's output pairs; the loop starts at a 32-pair boundary so
    // each warp assembles whole bit words (bits before `first` stay zero)
    const NodeRange nr = level_nodes(*plan, level);
    const uint64_t first = nr.lo * pcap;
    const uint64_t end = first + ((uint64_t)pcap << nr.shift);
    const uint64_t begin = first & ~31ull;
    const uint64_t stride = (uint64_t)grid.nblk * blockDim.x;
    for (uint64_t p = begin + (uint64_t)grid.bid * blockDim.x + threadIdx.x;
         p - (threadIdx.x & 31) < end; p += stride) {
        bool y = false;
        if (p >= first && p < end) {
            const uint32_t j = (uint32_t)(p / pcap);
            const uint32_t k = (uint32_t)(p - (uint64_t)j * pcap);
            const uint32_t s = size_at(lv, level, j);
            const uint32_t half = s / 2;
            const uint64_t node = (uint64_t)j * cap;
            const uint64_t lb = (uint64_t)(2 * j) * ccap;
            const uint64_t rb = lb + ccap;
            if (k < half) {
                const uint32_t u0 = inv[node + 2 * k];
                const uint32_t u1 = inv[node + 2 * k + 1];
                uint32_t to_left = ~0u, to_right = ~0u;
                if (u0 < s && u1 < s) {
                    const uint64_t q = (uint64_t)j * pcap + (u0 >> 1);
                    y = (((xbits[q >> 5] >> (q & 31)) ^ u0) & 1u) != 0;
                    to_left = (y ? u1 : u0) >> 1;
                    to_right = (y ? u0 : u1) >> 1;
                }
                if (child_inv != nullptr) {
                    child_inv[lb + k] = to_left;
                    child_inv[rb + k] = to_right;
                }
            } else if (k == half && (s & 1u) != 0) {
                const uint32_t u = inv[node + s - 1];
                if (child_inv != nullptr) child_inv[lb + half] = u < s ? u >> 1 : ~0u;
            }
            // children's pair-nodes start as their own roots: left child of
            // s - s/2 entries, right of s/2; pair-node k/2 for even k
            if (child_uf != nullptr && (k & 1u) == 0) {
                if (k < s - half) {
                    const uint32_t id = 2 * j * cpcap + (k >> 1);
                    child_uf[id] = id << 1;
                }
                if (k < half) {
                    const uint32_t id = (2 * j + 1) * cpcap + (k >> 1);
                    child_uf[id] = id << 1;
                }
            }
            // children's walk owners, one per pair-node, start unset
            if (child_owner != nullptr && (k & 1u) == 0) {
                if (k < s - half) child_owner[2 * j * cpcap + (k >> 1)] = ~0u;
                if (k < half) child_owner[(2 * j + 1) * cpcap + (k >> 1)] = ~0u;
            }
        }
        const unsigned word = __ballot_sync(0xffffffffu, y);
        if ((threadIdx.x & 31) == 0) {
            ybits[p >> 5] = word;
        }
    }
}

__global__ void __launch_bounds__(256) level_outputs(const Plan* __restrict__ plan,
    uint32_t level, const uint32_t* __restrict__ inv, const uint32_t* __restrict__ xbits,
    uint32_t* __restrict__ ybits, uint32_t* __restrict__ child_inv,
    uint32_t* __restrict__ child_owner, uint32_t* __restrict__ child_uf) {
    level_outputs_run(launch_grid(), plan, level, inv, xbits, ybits, child_inv, child_owner, child_uf);
}

// Switch bits of one section at one level, packet-major: thread t maps to
// (packet, node, pair-in-span) with the pair fastest, then the node, so for
// full packets consecutive threads land on consecutive blob bits and a
// warp issues one or two atomics instead of one per bit.
__device__ __forceinline__ void level_emit_run(Grid grid, const Plan* __restrict__ plan,
    uint32_t level, int side, const uint32_t* __restrict__ bits,
    const NodeAddress* __restrict__ addr, uint32_t* __restrict__ blob, uint64_t first_packet) {
    const LevelInfo& lv = plan->levels[level];
    const LevelSide& ls = lv.side[side];
    const GroupInfo& gi = plan->groups[side][ls.group];
    const uint32_t span_log2 = gi.depth - ls.rel - 1;
    const uint32_t pcap = (uint32_t)lv.pcap;
    const uint64_t max_pairs = lv.cap / 2;
    const uint64_t packets = (max_pairs + (1ull << span_log2) - 1) >> span_log2;
    const NodeRange nr = level_nodes(*plan, level);
    const uint32_t shift = nr.shift + span_log2; // log2(nodes * span)
    const uint64_t total = packets > first_packet ? (packets - first_packet) << shift : 0;
    const uint64_t section_bit = plan->section_offset[side] * 8;
    const uint64_t stride = (uint64_t)grid.nblk * blockDim.x;
    for (uint64_t t = (uint64_t)grid.bid * blockDim.x + threadIdx.x;
         t - (threadIdx.x & 31) < total; t += stride) {
        bool set = false;
        uint64_t dest = 0;
        if (t < total) {
            const uint64_t packet = first_packet + (t >> shift);
            const uint64_t rem = t & ((1ull << shift) - 1);
            const uint32_t node = (uint32_t)(nr.lo + (rem >> span_log2));
            const uint64_t pair = (packet << span_log2) + (rem & ((1ull << span_log2) - 1));
            const uint32_t s = size_at(lv, level, node);
            if (pair < s / 2) {
                const uint64_t q = (uint64_t)node * pcap + pair;
                set = ((bits[q >> 5] >> (q & 31)) & 1u) != 0;
                if (set) {
                    dest = section_bit + switch_bit(addr[node], pair);
                }
            }
        }
        emit_bit(blob, dest, set, 0xffffffffu);
    }
}

__global__ void __launch_bounds__(256) level_emit(const Plan* __restrict__ plan,
    uint32_t level, int side, const uint32_t* __restrict__ bits,
    const NodeAddress* __restrict__ addr, uint32_t* __restrict__ blob, uint64_t first_packet) {
    level_emit_run(launch_grid(), plan, level, side, bits, addr, blob, first_packet);
}

// Block form of level_emit for short runs (span_log2 < 5), on the packets
// every node of the level fills (packet < full_packets: below the smallest
// node's tail packet, so every node contributes `span` switches and every
// path's run starts at path * span inside the packet, SectionAddress using
// packet 0's prefix for all non-tail packets).  Inside such a packet the
// level's switches of one cluster root are then one contiguous block,
// path-major: thread per 32-bit word of a block, gathering the `span`-bit
// fields of 32 / span consecutive nodes, one or two atomics per word.
__device__ __forceinline__ void level_emit_blocks_run(Grid grid, const Plan* __restrict__ plan,
    uint32_t level, int side, const uint32_t* __restrict__ bits,
    const NodeAddress* __restrict__ addr, uint32_t* __restrict__ blob, uint64_t full_packets) {
    const LevelInfo& lv = plan->levels[level];
    const LevelSide& ls = lv.side[side];
    const GroupInfo& gi = plan->groups[side][ls.group];
    const uint32_t rel = ls.rel;
    const uint32_t span_log2 = gi.depth - rel - 1;
    const uint32_t span_mask = (1u << (1u << span_log2)) - 1u; // span <= 16 bits
    const uint32_t pcap = (uint32_t)lv.pcap;
    // nodes per word: 32 / span, or all 2^rel nodes of a root when fewer
    const uint32_t per_word_log2 = min(5u - span_log2, rel);
    const uint32_t words_log2 = rel - per_word_log2; // words per block (log2)
    const uint64_t per_root = full_packets << words_log2;
    // this call's nodes hold whole cluster roots (the host uses this form
    // only then)
    const NodeRange nr = level_nodes(*plan, level);
    const uint64_t root_lo = nr.lo >> rel;
    const uint64_t total = (per_root << (nr.shift - rel));
    const uint64_t section_bit = plan->section_offset[side] * 8;
    const uint64_t stride = (uint64_t)grid.nblk * blockDim.x;
    for (uint64_t t = (uint64_t)grid.bid * blockDim.x + threadIdx.x; t < total; t += stride) {
        const uint64_t root = root_lo + t / per_root;
        const uint64_t rem = t - (root - root_lo) * per_root;
        const uint64_t packet = rem >> words_log2;
        const uint32_t word = (uint32_t)(rem & ((1ull << words_log2) - 1));
        const uint32_t node0 = (uint32_t)(root << rel) + (word << per_word_log2);
        uint32_t v = 0;
        for (uint32_t i = 0; i < (1u << per_word_log2); ++i) {
            const uint64_t q = (uint64_t)(node0 + i) * pcap + (packet << span_log2);
            const uint64_t wq = q >> 5;
            const uint32_t field =
                __funnelshift_r(bits[wq], bits[wq + 1], (uint32_t)(q & 31)) & span_mask;
            v |= field << (i << span_log2);
        }
        if (v == 0) {
            continue;
        }
        const uint64_t dest = section_bit +
            switch_bit(addr[(uint32_t)(root << rel)], packet << span_log2) + ((uint64_t)word << 5);
        const uint32_t off = (uint32_t)(dest & 31);
        atomicOr(blob + (dest >> 5), v << off);
        if (off != 0 && (v >> (32 - off)) != 0) {
            atomicOr(blob + (dest >> 5) + 1, v >> (32 - off));
        }
    }
}

__global__ void __launch_bounds__(256) level_emit_blocks(const Plan* __restrict__ plan,
    uint32_t level, int side, const uint32_t* __restrict__ bits,
    const NodeAddress* __restrict__ addr, uint32_t* __restrict__ blob, uint64_t full_packets) {
    level_emit_blocks_run(launch_grid(), plan, level, side, bits, addr, blob, full_packets);
}

// Transposed form of level_emit_blocks for cluster roots of at least 32
// nodes (rel >= 5): a warp takes 32 consecutive nodes of one root and a
// window of 32 / span full packets.  Each lane loads one 32-bit window of
// its node's switches (span bits per packet, consecutive packets adjacent),
// and lane L then assembles output word L with 32 / span shuffles: packet
// L / span of the window, nodes (L % span) * 32 / span onwards.  Two loads
// per lane replace the 2 * 32 / span loads per word of the block form.
__device__ __forceinline__ void level_emit_transpose_run(Grid grid, const Plan* __restrict__ plan,
    uint32_t level, int side, const uint32_t* __restrict__ bits,
    const NodeAddress* __restrict__ addr, uint32_t* __restrict__ blob, uint64_t full_packets) {
    const LevelInfo& lv = plan->levels[level];
    const LevelSide& ls = lv.side[side];
    const GroupInfo& gi = plan->groups[side][ls.group];
    const uint32_t rel = ls.rel;                 // >= 5
    const uint32_t span_log2 = gi.depth - rel - 1; // < 5
    const uint32_t span_mask = (1u << (1u << span_log2)) - 1u;
    const uint32_t per_window_log2 = 5 - span_log2; // packets per lane window
    const uint32_t pcap = (uint32_t)lv.pcap;
    const uint64_t windows = (full_packets + (1ull << per_window_log2) - 1) >> per_window_log2;
    // 32-node groups of this call's nodes (at least 32 of them, aligned)
    const NodeRange nr = level_nodes(*plan, level);
    const uint64_t groups = 1ull << (nr.shift - 5);
    const uint64_t total_warps = groups * windows;
    const uint64_t section_bit = plan->section_offset[side] * 8;
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warps = ((uint64_t)grid.nblk * blockDim.x) >> 5;
    for (uint64_t wi = ((uint64_t)grid.bid * blockDim.x + threadIdx.x) >> 5; wi < total_warps;
         wi += warps) {
        const uint64_t group = wi / windows;
        const uint64_t k0 = (wi - group * windows) << per_window_log2;
        const uint32_t node = (uint32_t)(nr.lo + (group << 5)) + lane;
        const uint64_t q = (uint64_t)node * pcap + (k0 << span_log2);
        const uint64_t wq = q >> 5;
        uint32_t window = __funnelshift_r(bits[wq], bits[wq + 1], (uint32_t)(q & 31));
        // packets at or past full_packets belong to level_emit
        const uint64_t valid = full_packets - k0; // > 0
        if (valid < (1ull << per_window_log2)) {
            window &= (1u << (uint32_t)(valid << span_log2)) - 1u;
        }
        const uint32_t p_local = lane >> span_log2;
        const uint32_t g_out = lane & ((1u << span_log2) - 1u);
        uint32_t v = 0;
        for (uint32_t n = 0; n < (1u << per_window_log2); ++n) {
            const uint32_t w = __shfl_sync(0xffffffffu, window,
                (int)((g_out << per_window_log2) + n));
            v |= ((w >> (p_local << span_log2)) & span_mask) << (n << span_log2);
        }
        const uint64_t packet = k0 + p_local;
        if (v == 0 || packet >= full_packets) {
            continue;
        }
        const uint32_t root_node = node & ~((1u << rel) - 1u);
        const uint32_t n0 = (node & ((1u << rel) - 1u)) & ~31u; // first node of the group
        const uint64_t dest = section_bit + switch_bit(addr[root_node], packet << span_log2) +
            ((uint64_t)n0 << span_log2) + ((uint64_t)g_out << 5);
        const uint32_t off = (uint32_t)(dest & 31);
        atomicOr(blob + (dest >> 5), v << off);
        if (off != 0 && (v >> (32 - off)) != 0) {
            atomicOr(blob + (dest >> 5) + 1, v >> (32 - off));
        }
    }
}

__global__ void __launch_bounds__(256) level_emit_transpose(const Plan* __restrict__ plan,
    uint32_t level, int side, const uint32_t* __restrict__ bits,
    const NodeAddress* __restrict__ addr, uint32_t* __restrict__ blob, uint64_t full_packets) {
    level_emit_transpose_run(launch_grid(), plan, level, side, bits, addr, blob, full_packets);
}

// Word-wise form of level_emit for levels whose packets carry at least 32
// switches of each node (span_log2 >= 5).  The switches of one node inside
// one packet are a contiguous run of the node's bits and land on a
// contiguous run of blob bits (SwitchBitAddress::bit moves by one per pair
// inside a packet), so the level is a set of bit-range copies: thread per
// 32-switch chunk, one funnel shift to align the source and one or two
// atomics for the destination words (neighbouring runs share edge words).
// Chunks start at multiples of 32 pairs, so a chunk never crosses a packet.
__device__ __forceinline__ void level_emit_words_run(Grid grid, const Plan* __restrict__ plan,
    uint32_t level, int side, const uint32_t* __restrict__ bits,
    const NodeAddress* __restrict__ addr, uint32_t* __restrict__ blob) {
    const LevelInfo& lv = plan->levels[level];
    const LevelSide& ls = lv.side[side];
    const GroupInfo& gi = plan->groups[side][ls.group];
    const uint32_t span_log2 = gi.depth - ls.rel - 1;
    const uint32_t pcap = (uint32_t)lv.pcap;
    const uint64_t max_pairs = lv.cap / 2;
    const uint64_t packets = (max_pairs + (1ull << span_log2) - 1) >> span_log2;
    const uint32_t cshift = span_log2 - 5;  // log2(chunks per run)
    const NodeRange nr = level_nodes(*plan, level);
    const uint32_t shift = nr.shift + cshift; // log2(nodes * chunks per run)
    const uint64_t total = packets << shift;
    const uint64_t section_bit = plan->section_offset[side] * 8;
    const uint64_t stride = (uint64_t)grid.nblk * blockDim.x;
    for (uint64_t t = (uint64_t)grid.bid * blockDim.x + threadIdx.x; t < total; t += stride) {
        const uint64_t packet = t >> shift;
        const uint64_t rem = t & ((1ull << shift) - 1);
        const uint32_t node = (uint32_t)(nr.lo + (rem >> cshift));
        const uint64_t pair0 = (packet << span_log2) + ((rem & ((1ull << cshift) - 1)) << 5);
        const uint64_t half = size_at(lv, level, node) / 2;
        if (pair0 >= half) {
            continue;
        }
        const uint64_t q = (uint64_t)node * pcap + pair0;
        // the bit arrays keep one spare word, so bits[w + 1] is always there
        const uint64_t w = q >> 5;
        uint32_t v = __funnelshift_r(bits[w], bits[w + 1], (uint32_t)(q & 31));
        if (half - pair0 < 32) {
            v &= (1u << (uint32_t)(half - pair0)) - 1u;
        }
        if (v == 0) {
            continue;
        }
        const uint64_t dest = section_bit + switch_bit(addr[node], pair0);
        const uint32_t off = (uint32_t)(dest & 31);
        atomicOr(blob + (dest >> 5), v << off);
        if (off != 0 && (v >> (32 - off)) != 0) {
            atomicOr(blob + (dest >> 5) + 1, v >> (32 - off));
        }
    }
}

__global__ void __launch_bounds__(256) level_emit_words(const Plan* __restrict__ plan,
    uint32_t level, int side, const uint32_t* __restrict__ bits,
    const NodeAddress* __restrict__ addr, uint32_t* __restrict__ blob) {
    level_emit_words_run(launch_grid(), plan, level, side, bits, addr, blob);
}

} // namespace bpb200
