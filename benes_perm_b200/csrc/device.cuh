// SPDX-License-Identifier: Apache-2.0
//
// Device building blocks shared by the level kernels and the tile kernel:
// parity union-find, warp-aggregated bit emission and the warp factoradic
// rank.
#pragma once

#include "plan.hpp"

#include <cstdint>

namespace bpb200 {

// The block's place in the grid it works in: the launch's own grid for a
// one-permutation launch, or this permutation's share of the blocks of a
// batched launch over many permutations (serve.inc).  Kernel bodies index
// their work by it instead of blockIdx / gridDim.
struct Grid {
    uint32_t bid;
    uint32_t nblk;
};

__device__ __forceinline__ Grid launch_grid() { return Grid{blockIdx.x, gridDim.x}; }

// Device status word bits (read by the host after each call).
constexpr uint32_t kErrNotPermutation = 1u;  // value out of range or duplicated
constexpr uint32_t kErrIterationCap = 2u;    // a bounded retry loop gave up
constexpr uint32_t kErrInconsistent = 4u;    // colouring constraint violated

// Retry bound for every lock-free loop; far above what a valid input needs.
// Parents strictly decrease along every union-find chain (links go to the
// smaller root, halving jumps to the grandparent), so loops end anyway; the
// bound only caps the cost of a pathological chain.
constexpr uint32_t kSpinCap = 1u << 20;

// ------------------------------------------------------------------------
// Parity union-find over pair-nodes.
//
// Word layout: (parent << 1) | bit.  For a non-root the bit is the colour
// difference between the node and its parent; a root points to itself and
// its bit is the orientation flag set after all unions (it flips the colour
// of the whole component so that the odd tail ends up colour 0).  Linking
// always hangs the larger root under the smaller, so a root is the smallest
// pair-node of its component and parents strictly decrease along any chain.
// Path halving stores (grandparent, accumulated bit); the colour difference
// between a node and any ancestor is fixed by the constraint graph, so such
// racy plain stores can only ever write true facts.
// ------------------------------------------------------------------------

struct Found {
    uint32_t root;
    uint32_t bit;
};

template <typename Word>
__device__ __forceinline__ Word uf_load(Word* uf, uint32_t i) {
    return *((volatile Word*)(uf + i));
}

template <typename Word>
__device__ __forceinline__ Found uf_find(Word* uf, uint32_t x, uint32_t* err) {
    uint32_t acc = 0;
    uint32_t cur = x;
    for (uint32_t it = 0; it < kSpinCap; ++it) {
        const uint32_t w = (uint32_t)uf_load(uf, cur);
        const uint32_t p = w >> 1;
        if (p == cur) {
            return {cur, acc};
        }
        const uint32_t wp = (uint32_t)uf_load(uf, p);
        const uint32_t pp = wp >> 1;
        if (pp == p) {
            return {p, acc ^ (w & 1u)};
        }
        const uint32_t nb = (w ^ wp) & 1u;
        uf[cur] = (Word)((pp << 1) | nb);
        acc ^= nb;
        cur = pp;
    }
    atomicOr(err, kErrIterationCap);
    return {cur, acc};
}

__device__ __forceinline__ uint32_t cas_word(uint32_t* a, uint32_t e, uint32_t v) {
    return atomicCAS(a, e, v);
}

// Record x(a) ^ x(b) == rel.
template <typename Word>
__device__ __forceinline__ void uf_union(Word* uf, uint32_t a, uint32_t b, uint32_t rel,
    uint32_t* err) {
    for (uint32_t it = 0; it < kSpinCap; ++it) {
        const Found fa = uf_find(uf, a, err);
        const Found fb = uf_find(uf, b, err);
        rel ^= fa.bit ^ fb.bit;
        a = fa.root;
        b = fb.root;
        if (a == b) {
            if (rel != 0) {
                atomicOr(err, kErrInconsistent);
            }
            return;
        }
        const uint32_t lo = a < b ? a : b;
        const uint32_t hi = a < b ? b : a;
        if (cas_word((uint32_t*)(uf + hi), hi << 1, (lo << 1) | rel) == (hi << 1)) {
            return;
        }
    }
    atomicOr(err, kErrIterationCap);
}

// K finds advanced in lockstep: every round issues the loads of all
// unfinished finds before using any of them, so one thread keeps up to 2K
// independent loads in flight.  Bits of `pending` name the finds to run.
// `cached`: plain (L1-cached) loads, for finds that run after every union
// of the level is done.  Every find of a big component reads its root's
// word; through L1 those reads stop queueing at the one L2 slice that holds
// it.  No root changes any more, and a stale cached word is an older parent
// pointer, i.e. still an ancestor with its true parity, so cached finds end
// at the same roots with the same bits.  (During the unions a stale word
// could name a former root; the union kernel keeps uncached loads.)
template <typename Word>
__device__ __forceinline__ Word uf_word(Word* uf, uint32_t i, bool cached) {
    return cached ? uf[i] : uf_load(uf, i);
}

template <int K, typename Word>
__device__ __forceinline__ void uf_find_many(Word* uf, const uint32_t (&x)[K], Found (&out)[K],
    uint32_t pending, uint32_t* err, bool cached = false) {
    uint32_t cur[K], acc[K];
#pragma unroll
    for (int i = 0; i < K; ++i) {
        cur[i] = x[i];
        acc[i] = 0;
    }
    for (uint32_t it = 0; pending != 0; ++it) {
        if (it == kSpinCap) {
            atomicOr(err, kErrIterationCap);
#pragma unroll
            for (int i = 0; i < K; ++i) {
                if (pending & (1u << i)) out[i] = {cur[i], acc[i]};
            }
            return;
        }
        uint32_t w[K], wp[K];
#pragma unroll
        for (int i = 0; i < K; ++i) {
            if (pending & (1u << i)) w[i] = (uint32_t)uf_word(uf, cur[i], cached);
        }
#pragma unroll
        for (int i = 0; i < K; ++i) {
            if (pending & (1u << i)) {
                const uint32_t p = w[i] >> 1;
                if (p == cur[i]) {
                    out[i] = {cur[i], acc[i]};
                    pending &= ~(1u << i);
                } else {
                    wp[i] = (uint32_t)uf_word(uf, p, cached);
                }
            }
        }
#pragma unroll
        for (int i = 0; i < K; ++i) {
            if (pending & (1u << i)) {
                const uint32_t p = w[i] >> 1;
                const uint32_t pp = wp[i] >> 1;
                if (pp == p) {
                    out[i] = {p, acc[i] ^ (w[i] & 1u)};
                    pending &= ~(1u << i);
                } else {
                    const uint32_t nb = (w[i] ^ wp[i]) & 1u;
                    uf[cur[i]] = (Word)((pp << 1) | nb);
                    acc[i] ^= nb;
                    cur[i] = pp;
                }
            }
        }
    }
}

// K unions x(a[i]) ^ x(b[i]) == rel[i], with all 2K finds of a round in
// lockstep.  A failed link retries from the two roots it saw.
//
// The first round's finds use L1-cached loads.  Once a component is large,
// most finds end at its root, and uncached they all queue at the one L2
// slice holding that word.  A cached word may be stale, but it still names
// a true ancestor with its true parity, so a find ends at a node X of the
// right component with the right relative colour; X may have stopped being
// a root.  That is harmless: when both finds reach the same X the two nodes
// share a component; otherwise the link is a CAS that requires the larger
// end `hi` to be a root at that moment (it fails on a stale root, and the
// retry rounds then read L2), and hanging a true root hi under any smaller
// node `lo` joins two different components (a root is its component's
// minimum, so lo < hi lies outside hi's component) while keeping parents
// strictly decreasing.
template <int K, typename Word>
__device__ __forceinline__ void uf_union_many(Word* uf, uint32_t (&a)[K], uint32_t (&b)[K],
    uint32_t (&rel)[K], uint32_t pending, uint32_t* err) {
    for (uint32_t it = 0; pending != 0; ++it) {
        if (it == kSpinCap) {
            atomicOr(err, kErrIterationCap);
            return;
        }
        uint32_t x[2 * K];
        Found f[2 * K];
#pragma unroll
        for (int i = 0; i < K; ++i) {
            x[i] = a[i];
            x[K + i] = b[i];
        }
        uint32_t both = 0;
#pragma unroll
        for (int i = 0; i < K; ++i) {
            if (pending & (1u << i)) both |= (1u << i) | (1u << (K + i));
        }
        uf_find_many<2 * K>(uf, x, f, both, err, it == 0);
#pragma unroll
        for (int i = 0; i < K; ++i) {
            if (!(pending & (1u << i))) continue;
            rel[i] ^= f[i].bit ^ f[K + i].bit;
            a[i] = f[i].root;
            b[i] = f[K + i].root;
            if (a[i] == b[i]) {
                if (rel[i] != 0) atomicOr(err, kErrInconsistent);
                pending &= ~(1u << i);
                continue;
            }
            const uint32_t lo = a[i] < b[i] ? a[i] : b[i];
            const uint32_t hi = a[i] < b[i] ? b[i] : a[i];
            if (cas_word((uint32_t*)(uf + hi), hi << 1, (lo << 1) | rel[i]) == (hi << 1)) {
                pending &= ~(1u << i);
            }
        }
    }
}

// Blocks take chunks of `chunk` consecutive items in increasing order from
// *counter, so the items in flight across the whole GPU stay within a few
// chunks of each other.  (A grid-stride loop lets blocks drift apart and
// spreads node-local random accesses over far more memory than L2 holds.)
// Every thread of the block must call it.
__device__ __forceinline__ bool claim_chunk(uint32_t* counter, uint64_t chunk, uint64_t total,
    uint64_t* first) {
    __shared__ uint64_t s_first;
    __syncthreads();
    if (threadIdx.x == 0) {
        s_first = (uint64_t)atomicAdd(counter, 1u) * chunk;
    }
    __syncthreads();
    *first = s_first;
    return s_first < total;
}

// ------------------------------------------------------------------------
// Warp-aggregated emission of single bits into the blob.  Lanes of the
// warp named in `active` call it together; each lane with `set` ORs bit
// `abs_bit` (absolute bit position in the blob).  Lanes that hit the same
// 32-bit word combine first, so one atomic is issued per distinct word.
// ------------------------------------------------------------------------
__device__ __forceinline__ void emit_bit(uint32_t* blob, uint64_t abs_bit, bool set,
    unsigned active) {
    const unsigned writers = __ballot_sync(active, set);
    if (!set) {
        return;
    }
    const unsigned long long word = abs_bit >> 5;
    const unsigned group = __match_any_sync(writers, word);
    const unsigned v = __reduce_or_sync(group, 1u << (abs_bit & 31));
    if ((threadIdx.x & 31) == (unsigned)(__ffs(group) - 1)) {
        atomicOr(blob + word, v);
    }
}

// ------------------------------------------------------------------------
// 128-bit helpers for the factoradic rank.
// ------------------------------------------------------------------------
struct U128 {
    unsigned long long lo, hi;
};

__device__ __forceinline__ U128 mul128(U128 a, U128 b) {
    U128 r;
    r.lo = a.lo * b.lo;
    r.hi = __umul64hi(a.lo, b.lo) + a.lo * b.hi + a.hi * b.lo;
    return r;
}

__device__ __forceinline__ U128 add128(U128 a, U128 b) {
    U128 r;
    r.lo = a.lo + b.lo;
    r.hi = a.hi + b.hi + (r.lo < a.lo ? 1ull : 0ull);
    return r;
}

__device__ __forceinline__ U128 shfl_down128(U128 v, int d) {
    U128 r;
    r.lo = __shfl_down_sync(0xffffffffu, v.lo, d);
    r.hi = __shfl_down_sync(0xffffffffu, v.hi, d);
    return r;
}

// Factoradic rank of one middle group held one entry per lane (lanes
// >= count are idle), as in encode_factoradic (src/internal.hpp:148-167):
// digit j = #{k < j : v[k] < v[j]} and rank = sum_j digit_j * count!/(j+1)!.
// Digits come from five ballots (a one-hot lane mask per value) and a
// prefix-OR over values; the mixed-radix sum is an order-preserving tree
// reduction of (rank, radix product) pairs: (r1,m1)+(r2,m2) = (r1*m2+r2, m1*m2).
// Must be called by all 32 lanes.  Result valid in lane 0.  *distinct is
// false (in every lane) when two lanes hold the same value.
__device__ __forceinline__ U128 warp_factoradic_rank(uint32_t value, uint32_t count,
    bool* distinct) {
    const unsigned lane = threadIdx.x & 31;
    const bool live = lane < count;
    const unsigned active = __ballot_sync(0xffffffffu, live);
    unsigned onehot = active;
    for (int b = 0; b < 5; ++b) {
        const unsigned bits = __ballot_sync(0xffffffffu, live && ((value >> b) & 1));
        onehot &= ((lane >> b) & 1) ? bits : ~bits;
    }
    // with count values below count, every value has exactly one lane iff
    // no value is missing
    *distinct = __ballot_sync(0xffffffffu, live && __popc(onehot) != 1) == 0;
    // onehot (in lane L) = the lane holding value L.  Exclusive prefix OR
    // over values gives the lanes holding a smaller value.
    unsigned below = onehot;
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned t = __shfl_up_sync(0xffffffffu, below, d);
        if ((int)lane >= d) {
            below |= t;
        }
    }
    below = __shfl_up_sync(0xffffffffu, below, 1);
    if (lane == 0) {
        below = 0;
    }
    const unsigned smaller = __shfl_sync(0xffffffffu, below, live ? value : 0);
    const uint32_t digit = live ? (uint32_t)__popc(smaller & ((1u << lane) - 1u)) : 0u;
    // The first three tree levels combine blocks of at most 8 radices, whose
    // product stays below 25 * 26 * ... * 32 < 2^39: 64-bit arithmetic
    // suffices there (and the partial rank is below the product).
    unsigned long long r64 = digit;
    unsigned long long m64 = live ? (unsigned long long)(lane + 1) : 1ull;
    for (int d = 1; d < 8; d <<= 1) {
        const unsigned long long r2 = __shfl_down_sync(0xffffffffu, r64, d);
        const unsigned long long m2 = __shfl_down_sync(0xffffffffu, m64, d);
        if ((lane & (2 * d - 1)) == 0) {
            r64 = r64 * m2 + r2;
            m64 *= m2;
        }
    }
    U128 r = {r64, 0ull};
    U128 m = {m64, 0ull};
    for (int d = 8; d < 32; d <<= 1) {
        const U128 r2 = shfl_down128(r, d);
        const U128 m2 = shfl_down128(m, d);
        if ((lane & (2 * d - 1)) == 0) {
            r = add128(mul128(r, m2), r2);
            m = mul128(m, m2);
        }
    }
    return r;
}

// OR `nbits` (<= 118) bits of `rank` into the blob at absolute bit `abs`.
// Lanes 0..4 each handle one destination word.  All lanes call.
__device__ __forceinline__ void emit_rank(uint32_t* blob, uint64_t abs, uint32_t nbits,
    U128 rank) {
    const unsigned lane = threadIdx.x & 31;
    rank.lo = __shfl_sync(0xffffffffu, rank.lo, 0);
    rank.hi = __shfl_sync(0xffffffffu, rank.hi, 0);
    if (nbits == 0 || lane >= 5) {
        return;
    }
    const uint32_t shift = (uint32_t)(abs & 31);
    const uint64_t word0 = abs >> 5;
    const uint32_t last = (uint32_t)((shift + nbits - 1) >> 5);
    if (lane > last) {
        return;
    }
    // bits of the rank that land in destination word `lane`
    const int lo_bit = (int)lane * 32 - (int)shift; // rank bit at dest bit 0 of this word
    // rank < count! < 2^nbits, so no rank bit at or above nbits is set and
    // the word is a plain 32-bit window of the 128-bit rank
    uint32_t v;
    if (lo_bit < 0) {
        v = (uint32_t)(rank.lo << (uint32_t)(-lo_bit));
    } else {
        const uint32_t sh = (uint32_t)lo_bit; // < 128
        unsigned long long x;
        if (sh >= 64) {
            x = rank.hi >> (sh - 64);
        } else if (sh == 0) {
            x = rank.lo;
        } else {
            x = (rank.lo >> sh) | (rank.hi << (64 - sh));
        }
        v = (uint32_t)x;
    }
    if (v != 0) {
        atomicOr(blob + word0 + lane, v);
    }
}

} // namespace bpb200
