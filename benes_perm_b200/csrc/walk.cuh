// SPDX-License-Identifier: Apache-2.0
//
// Canonical colouring of the global levels by orbit walks.
//
// Within a node of s entries let A(v) = v^1 (input pair partner) and
// B(u) = inv[p[u]^1] (the input whose output is paired with u's output).
// The constraint graph (src/benes.cpp:238-252) alternates A and B edges, so
// each component is a cycle that splits into two orbits of f = B o A,
// f(v) = inv[p[v^1]^1], mirrors of each other (O and O^1); all vertices of
// one orbit share a colour and the mirror has the other.  An odd node gets
// one virtual vertex s with p[s] = s (so inv[s] = s): the reference's tail
// path then closes into a cycle through s, and giving the tail t = s-1 the
// smallest key makes "orbit holding the smallest key gets colour 0" exactly
// the reference's canonical rule (odd tail first, then each component's
// smallest vertex, src/benes.cpp:253-297):
//     colour(v) = [min key(O(v)) > min key(O(v^1))],  key(t) = 0, key(v) = v+1.
//
// Orbits are long for random inputs, so one vertex in every bucket of
// 2^kRulerLog2 slots (at a hashed position) is a ruler.  A ruler walks its
// orbit up to the next ruler, stamping each even vertex it passes with its
// id and keeping the minimum key of the segment and of the segment's
// mirror.  Only even vertices are stamped, into one owner word per
// pair-node: the colour of pair-node k is the colour of vertex 2k, and
// halving the stamps halves the walk's random writes and its owner array.
// Pointer jumping over rulers (stopping after the first round that changes
// nothing, which implies convergence on cycles) turns segment minima into
// orbit minima.  No atomics, no shared roots: every step is two independent
// gathers.  Cycles without any ruler are short for all but contrived inputs
// and are walked whole (level_walk_short); a walk longer than kWalkCap sets
// the `hard` flag and the level falls back to the union-find kernels.
//
// Walks pay off while a node's arrays fit in L2 (random access there is
// 6-8x faster than in HBM on B200); nodes above kWalkMaxNode entries are
// coloured by union-find, which needs fewer HBM round trips per entry.
#pragma once

#include "device.cuh"
#include "kernels.cuh"
#include "plan.hpp"

#include <cstdint>

namespace bpb200 {

// Tuning knobs, overridable at build time.  Measured on B200 over uniform
// 2^30-entry inputs with super-ruler jumping: one ruler per 8 slots, walks
// up to 2^23-entry nodes and 4 walk blocks per SM gave the lowest total
// (1078 ms; rulers per 16 slots: 1094 at 3 blocks per SM; per 32: 1175;
// per 4: 1132; walk limit 2^24: 1112).  Denser rulers give shorter,
// more numerous walk chains, which hide the L2 latency of each step better.
#ifndef BPB200_RULER_LOG2
#define BPB200_RULER_LOG2 3
#endif
#ifndef BPB200_WALK_MAX_LOG2
#define BPB200_WALK_MAX_LOG2 23
#endif
// Union-find levels whose nodes have at most 2^BPB200_FINAL_STRIDE_LOG2
// slots finalize in grid-stride order, larger ones in claimed order (see
// level_finalize); measured on B200 at 2^30 uniform entries (finalize 105 ms
// per compress; limit 2^24: 110 ms; 2^23: 119 ms).
#ifndef BPB200_FINAL_STRIDE_LOG2
#define BPB200_FINAL_STRIDE_LOG2 26
#endif
// Union-find levels: level_finalize writes each pair-node's root back (1),
// measured on B200 at 2^30 uniform entries: finalize 105.0 ms per compress
// against 106.2 without.
#ifndef BPB200_RESOLVE_WRITEBACK
#define BPB200_RESOLVE_WRITEBACK 1
#endif

constexpr uint32_t kRulerLog2 = BPB200_RULER_LOG2; // one ruler per 2^kRulerLog2 slots
constexpr uint32_t kWalkCap = 1u << 16;      // longest ruler walk before giving up
#ifndef BPB200_WALK_CHUNK
#define BPB200_WALK_CHUNK 32
#endif
// rulers claimed per warp at a time: 32 measured fastest on B200 at 2^30
// uniform entries (walks 157 ms per compress; 16: 159 ms; 8: 176 ms)
constexpr uint32_t kWalkChunk = BPB200_WALK_CHUNK;
constexpr uint32_t kJumpItems = 8;           // rulers per thread in a claimed jump chunk
constexpr uint64_t kWalkMaxNode = 1ull << BPB200_WALK_MAX_LOG2; // larger: union-find
static_assert(BPB200_RULER_LOG2 >= 2 && BPB200_RULER_LOG2 <= 8, "ruler density out of range");
static_assert(BPB200_WALK_MAX_LOG2 >= 13 && BPB200_WALK_MAX_LOG2 <= 28, "walk limit out of range");
constexpr uint32_t kUnset = 0xffffffffu;     // owner of a vertex no walk reached
// Walk owners are one word per pair-node: owner[j * pcap + k] is the stamp
// of even vertex 2k of node j (the finalize reads only even vertices), half
// the footprint of a word per slot, which keeps more of a node in L2.
constexpr uint32_t kColourTag = 0x80000000u; // owner value carrying a colour directly
constexpr uint32_t kNoRuler = 0xffffffffu;   // bucket whose hashed slot is padding

// control words of a level
enum : int {
    kCtlHard = 0,
    kCtlChanged = 1,
    kCtlDone = 2,
    kCtlFinal = 3,
    kCtlClaim = 4,       // ruler chunks handed out by level_walk
    kCtlClaimPlace = 5,  // chunks handed out by level_place
    kCtlClaimInverse = 6, // chunks handed out by level_inverse
    kCtlClaimJump = 7,   // ruler chunks handed out by ruler_jump (reset every round)
    kCtlClaimUnion = 8,  // chunks handed out by level_union
    kCtlClaimFinal = 9,  // chunks handed out by level_finalize
    kCtlClaimSuper = 10, // super-ruler chunks handed out by ruler_super_walk
    kCtlWords = 16       // control_reset clears them with one warp
};

__device__ __forceinline__ uint32_t ruler_position(uint32_t bucket) {
    return (bucket * 0x9E3779B1u) >> (32 - kRulerLog2);
}

__device__ __forceinline__ bool is_ruler_slot(uint32_t slot) {
    return (slot & ((1u << kRulerLog2) - 1)) == ruler_position(slot >> kRulerLog2);
}

// The rulers of this call's nodes (level_nodes): buckets [lo, hi) covering
// slots [slot_lo, slot_end).  A bucket at either end may hash its ruler
// into a neighbouring node outside the range; such rulers are marked absent.
struct RulerRange {
    uint32_t lo, hi;
    uint64_t slot_lo, slot_end;
};

BP_HD RulerRange ruler_range(const Plan& p, uint32_t level) {
    const LevelInfo& lv = p.levels[level];
    const NodeRange nr = level_nodes(p, level);
    const uint64_t slot_lo = nr.lo * lv.cap;
    const uint64_t slot_end = slot_lo + (lv.cap << nr.shift);
    return RulerRange{(uint32_t)(slot_lo >> kRulerLog2),
        (uint32_t)((slot_end + (1u << kRulerLog2) - 1) >> kRulerLog2), slot_lo, slot_end};
}

// One node of one level, as seen by a walker.
template <typename T>
struct NodeView {
    const T* p;            // node's values (node-local)
    const uint32_t* inv;   // node's inverse
    uint32_t s;            // entries
    bool odd;

    // f(v) = inv[p[v^1]^1] with the virtual vertex s of an odd node; returns
    // 0xffffffff when a value is out of range (input is not a permutation)
    __device__ __forceinline__ uint32_t f(uint32_t v) const {
        const uint32_t a = v ^ 1u;
        uint32_t o;
        if (odd && a == s) {
            o = s;
        } else {
            const uint64_t value = (uint64_t)p[a];
            if (value >= s) {
                return 0xffffffffu;
            }
            o = (uint32_t)value;
        }
        const uint32_t b = o ^ 1u;
        return (odd && b == s) ? s : inv[b];
    }
    __device__ __forceinline__ uint32_t key(uint32_t v) const {
        return (odd && v == s - 1) ? 0u : v + 1;
    }
};

// Ruler walks.  Warps claim chunks of kWalkChunk rulers in address order
// from a per-level counter, so the walks in flight at any moment touch a
// window of a few tens of MB that stays in L2; within a warp each lane takes
// the next ruler of the chunk as soon as its current walk ends, so walk
// lengths (geometric, mean 2^kRulerLog2) do not leave lanes idle behind the
// longest walk.  state[r] = {next ruler, min key, min mirror key, 0};
// owner[pair-node] = r for every real even vertex the walk passes.
template <typename T>
__device__ __forceinline__ void level_walk_run(Grid grid, const Plan* __restrict__ plan, uint32_t level,
    const T* __restrict__ vals, const uint32_t* __restrict__ inv, uint32_t* __restrict__ owner,
    uint4* __restrict__ state, uint32_t* control) {
    const LevelInfo& lv = plan->levels[level];
    const uint32_t cap = (uint32_t)lv.cap;
    const RulerRange rr = ruler_range(*plan, level);
    const uint32_t lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    uint32_t next_free = 0, hi = 0; // current chunk, warp-uniform
    bool exhausted = false;
    bool active = false;
    uint32_t r = 0, base = 0, own = 0, s = 0, cur = 0, ma = 0, mb = 0, steps = 0;
    bool odd = false;
    for (;;) {
        const unsigned idle = __ballot_sync(0xffffffffu, !active);
        if (idle != 0 && next_free >= hi && !exhausted) {
            uint32_t c = 0;
            if (lane == 0) c = atomicAdd(control + kCtlClaim, 1u);
            c = __shfl_sync(0xffffffffu, c, 0);
            const uint64_t lo = rr.lo + (uint64_t)c * kWalkChunk;
            if (lo >= rr.hi) {
                exhausted = true;
            } else {
                next_free = (uint32_t)lo;
                hi = (uint32_t)(lo + kWalkChunk < rr.hi ? lo + kWalkChunk : rr.hi);
            }
        }
        if (!active) {
            const uint32_t mine = next_free + (uint32_t)__popc(idle & below);
            if (mine < hi) {
                r = mine;
                const uint32_t slot = (r << kRulerLog2) + ruler_position(r);
                const bool in_range = slot >= rr.slot_lo && slot < rr.slot_end;
                const uint32_t j = in_range ? slot / cap : 0u;
                const uint32_t v0 = slot - j * cap;
                s = in_range ? size_at(lv, level, j) : 0u;
                if (!in_range || v0 >= s) {
                    state[r] = make_uint4(kNoRuler, 0, 0, 0);
                } else {
                    base = j * cap;
                    own = j * (uint32_t)lv.pcap;
                    odd = (s & 1u) != 0;
                    const NodeView<T> nv{vals + base, inv + base, s, odd};
                    cur = v0;
                    ma = nv.key(v0);
                    mb = nv.key(v0 ^ 1u);
                    steps = 0;
                    active = true;
                }
            }
        }
        next_free = min(next_free + (uint32_t)__popc(idle), hi);
        if (__ballot_sync(0xffffffffu, active) == 0) {
            if (exhausted) break;
            continue;
        }
        if (active) {
            const NodeView<T> nv{vals + base, inv + base, s, odd};
            const uint32_t w = nv.f(cur);
            bool end = false;
            uint32_t next = r;
            if (w >= s + (odd ? 1u : 0u)) {
                atomicOr(control + kCtlHard, 1u); // not a permutation
                end = true;
            } else if (w < s && is_ruler_slot(base + w)) {
                next = (base + w) >> kRulerLog2;
                end = true;
            } else {
                if (w < s && (w & 1u) == 0) owner[own + (w >> 1)] = r;
                ma = min(ma, nv.key(w));
                mb = min(mb, nv.key(w ^ 1u));
                cur = w;
                if (++steps == kWalkCap) {
                    atomicOr(control + kCtlHard, 1u);
                    end = true;
                }
            }
            if (end) {
                state[r] = make_uint4(next, ma, mb, 0);
                active = false;
            }
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(256) level_walk(const Plan* __restrict__ plan, uint32_t level,
    const T* __restrict__ vals, const uint32_t* __restrict__ inv, uint32_t* __restrict__ owner,
    uint4* __restrict__ state, uint32_t* control) {
    level_walk_run<T>(launch_grid(), plan, level, vals, inv, owner, state, control);
}

// Orbits no ruler reached: thread per pair-node whose even vertex is
// neither a ruler nor stamped, i.e. lies in a ruler-free orbit (its
// mirror orbit may have rulers; the walk folds the mirror's keys as it
// goes, so it needs nothing from them).  Only the walker starting at the
// smallest even vertex of its orbit walks the orbit whole (the others stop
// at the first smaller even vertex, about log L steps), then stamps the
// orbit's colour on every real vertex of it; the cost is O(L log L) per
// orbit, and such orbits are short for all but contrived inputs.
template <typename T>
__device__ __forceinline__ void level_walk_short_run(Grid grid, const Plan* __restrict__ plan,
    uint32_t level, const T* __restrict__ vals, const uint32_t* __restrict__ inv,
    uint32_t* __restrict__ owner, uint32_t* control) {
    const LevelInfo& lv = plan->levels[level];
    const uint32_t cap = (uint32_t)lv.cap;
    const uint32_t pcap = (uint32_t)lv.pcap;
    const NodeRange nr = level_nodes(*plan, level);
    const uint64_t end = (nr.lo + (1ull << nr.shift)) * pcap;
    for (uint64_t pidx = nr.lo * pcap + (uint64_t)grid.bid * blockDim.x + threadIdx.x; pidx < end;
         pidx += (uint64_t)grid.nblk * blockDim.x) {
        const uint32_t j = (uint32_t)(pidx / pcap);
        const uint32_t k = (uint32_t)(pidx - (uint64_t)j * pcap);
        const uint32_t s = size_at(lv, level, j);
        if (k >= s - s / 2) {
            continue;
        }
        const uint32_t base = j * cap;
        const uint32_t own = j * pcap;
        const uint32_t v = 2 * k;
        if (is_ruler_slot(base + v) || owner[own + k] != kUnset) {
            continue;
        }
        const NodeView<T> nv{vals + base, inv + base, s, (s & 1u) != 0};
        const uint32_t mine = nv.key(v);
        uint32_t ma = mine, mb = nv.key(v ^ 1u);
        uint32_t cur = v;
        bool closed = false, smallest = true;
        for (uint32_t step = 0; step < kWalkCap; ++step) {
            const uint32_t w = nv.f(cur);
            if (w >= s + (nv.odd ? 1u : 0u)) {
                break;
            }
            if (w == v) {
                closed = true;
                break;
            }
            if ((w & 1u) == 0 && w < s && nv.key(w) < mine) {
                smallest = false; // that vertex's walker covers this orbit
                closed = true;
                break;
            }
            ma = min(ma, nv.key(w));
            mb = min(mb, nv.key(w ^ 1u));
            cur = w;
        }
        if (!closed) {
            atomicOr(control + kCtlHard, 1u);
            continue;
        }
        if (!smallest) {
            continue;
        }
        const uint32_t colour = kColourTag | (ma > mb ? 1u : 0u);
        cur = v;
        do {
            if (cur < s && (cur & 1u) == 0) owner[own + (cur >> 1)] = colour;
            cur = nv.f(cur);
        } while (cur != v);
    }
}

template <typename T>
__global__ void __launch_bounds__(256) level_walk_short(const Plan* __restrict__ plan,
    uint32_t level, const T* __restrict__ vals, const uint32_t* __restrict__ inv,
    uint32_t* __restrict__ owner, uint32_t* control) {
    level_walk_short_run<T>(launch_grid(), plan, level, vals, inv, owner, control);
}

// One pointer-jumping round over ruler states (src -> dst).  Blocks claim
// chunks of rulers in address order, so the rulers being jumped at any time
// (and, early on, the near successors they read) stay close together.
// The done/hard words were written by earlier launches, so every thread of
// a block sees the same value and the block leaves together.
// States [lo, hi) are this call's super-rulers (all of them unless the
// level is sharded); a successor outside them can only come from a
// non-permutation and sends the level to union-find.
__device__ __forceinline__ void ruler_jump_run(Grid grid, const uint4* __restrict__ src,
    uint4* __restrict__ dst, uint32_t lo, uint32_t hi, uint32_t round, uint32_t* control) {
    if (*(volatile uint32_t*)(control + kCtlDone) != 0 ||
        *(volatile uint32_t*)(control + kCtlHard) != 0) {
        return;
    }
    bool changed = false;
    const uint64_t chunk = (uint64_t)blockDim.x * kJumpItems;
    uint64_t first = 0;
    bool bad = false;
    while (claim_chunk(control + kCtlClaimJump, chunk, hi - lo, &first)) {
        for (uint32_t k = 0; k < kJumpItems; ++k) {
            const uint64_t r = lo + first + (uint64_t)k * blockDim.x + threadIdx.x;
            if (r >= hi) {
                break;
            }
            const uint4 me = src[r];
            if (me.x == kNoRuler || me.x < lo || me.x >= hi) {
                bad |= me.x != kNoRuler;
                dst[r] = me;
                continue;
            }
            const uint4 nx = src[me.x];
            const uint4 out = make_uint4(nx.x, min(me.y, nx.y), min(me.z, nx.z), 0);
            changed |= (out.y != me.y) || (out.z != me.z);
            dst[r] = out;
        }
    }
    if (__any_sync(0xffffffffu, changed) && (threadIdx.x & 31) == 0) {
        atomicOr(control + kCtlChanged, 1u);
    }
    if (bad) {
        atomicOr(control + kCtlHard, 1u);
    }
    (void)round;
}

__global__ void __launch_bounds__(256) ruler_jump(const uint4* __restrict__ src,
    uint4* __restrict__ dst, uint32_t lo, uint32_t hi, uint32_t round, uint32_t* control) {
    ruler_jump_run(launch_grid(), src, dst, lo, hi, round, control);
}

// After a round: a round that changed nothing means every ruler holds its
// orbit's minima; later rounds then return at once.
__device__ __forceinline__ void ruler_check_run(Grid grid, uint32_t round, uint32_t* control) {
    control[kCtlClaimJump] = 0; // the next round claims from the start again
    if (control[kCtlDone] != 0 || control[kCtlHard] != 0) {
        return;
    }
    control[kCtlFinal] = (round + 1) & 1u; // buffer the round just wrote
    if (control[kCtlChanged] == 0) {
        control[kCtlDone] = 1;
    }
    control[kCtlChanged] = 0;
}

__global__ void ruler_check(uint32_t round, uint32_t* control) {
    ruler_check_run(launch_grid(), round, control);
}

// Levels with few super-rulers spend their jumping time on launches, not on
// the rounds: a round over a few thousand states is shorter than the gap
// between two launches.  ruler_jump_block runs all rounds of such a level in
// one CTA, a block barrier between rounds, and leaves the control words as
// the ruler_jump / ruler_check sequence would (kCtlFinal names the buffer
// the last executed round wrote; kCtlDone is set when a round changed
// nothing).  Each thread handles kJumpBlockBatch states at a time, loading
// all of them before their successors so the gathers overlap.
constexpr uint32_t kJumpBlockThreads = 1024;
constexpr uint32_t kJumpBlockBatch = 4;
#ifndef BPB200_JUMP_BLOCK_LOG2
#define BPB200_JUMP_BLOCK_LOG2 14
#endif
constexpr uint32_t kJumpBlockMaxStates = 1u << BPB200_JUMP_BLOCK_LOG2;

__device__ __forceinline__ void ruler_jump_block_run(Grid grid, uint4* s0, uint4* s1,
    uint32_t lo, uint32_t hi, uint32_t rounds, uint32_t* control) {
    // written by earlier launches: every thread reads the same values
    if (*(volatile uint32_t*)(control + kCtlDone) != 0 ||
        *(volatile uint32_t*)(control + kCtlHard) != 0) {
        return;
    }
    __shared__ uint32_t changed[2];
    if (threadIdx.x == 0) {
        changed[0] = 0u;
        changed[1] = 0u;
    }
    __syncthreads();
    uint32_t final_buffer = 0;
    bool done = false;
    bool bad = false;
    for (uint32_t r = 0; r <= rounds; ++r) {
        const uint4* src = (r & 1u) ? s1 : s0;
        uint4* dst = (r & 1u) ? s0 : s1;
        bool ch = false;
        for (uint32_t base = lo; base < hi; base += kJumpBlockThreads * kJumpBlockBatch) {
            uint4 me[kJumpBlockBatch], nx[kJumpBlockBatch];
#pragma unroll
            for (uint32_t k = 0; k < kJumpBlockBatch; ++k) {
                const uint32_t i = base + k * kJumpBlockThreads + threadIdx.x;
                me[k] = i < hi ? __ldcg(src + i) : make_uint4(kNoRuler, 0u, 0u, 0u);
            }
#pragma unroll
            for (uint32_t k = 0; k < kJumpBlockBatch; ++k) {
                const bool inside = me[k].x >= lo && me[k].x < hi;
                const bool live = me[k].x != kNoRuler && inside;
                bad |= me[k].x != kNoRuler && !inside;
                nx[k] = live ? __ldcg(src + me[k].x) : me[k];
            }
#pragma unroll
            for (uint32_t k = 0; k < kJumpBlockBatch; ++k) {
                const uint32_t i = base + k * kJumpBlockThreads + threadIdx.x;
                if (i >= hi) {
                    continue;
                }
                if (me[k].x == kNoRuler || me[k].x < lo || me[k].x >= hi) {
                    dst[i] = me[k];
                    continue;
                }
                const uint4 out = make_uint4(nx[k].x, min(me[k].y, nx[k].y),
                    min(me[k].z, nx[k].z), 0u);
                ch |= (out.y != me[k].y) || (out.z != me[k].z);
                dst[i] = out;
            }
        }
        if (ch) {
            changed[r & 1u] = 1u;
        }
        __syncthreads(); // this round's states and flag are visible to the block
        const bool any = changed[r & 1u] != 0u;
        final_buffer = (r + 1u) & 1u;
        if (threadIdx.x == 0) {
            changed[(r + 1u) & 1u] = 0u; // every thread read it a round ago
        }
        __syncthreads();
        if (!any) {
            done = true;
            break;
        }
    }
    if (bad) {
        atomicOr(control + kCtlHard, 1u); // a successor out of range: fall back to union-find
    }
    if (threadIdx.x == 0) {
        control[kCtlFinal] = final_buffer;
        if (done) {
            control[kCtlDone] = 1u;
        }
        control[kCtlChanged] = 0u;
        control[kCtlClaimJump] = 0u;
    }
}

__global__ void __launch_bounds__(kJumpBlockThreads, 1) ruler_jump_block(uint4* s0, uint4* s1,
    uint32_t lo, uint32_t hi, uint32_t rounds, uint32_t* control) {
    ruler_jump_block_run(launch_grid(), s0, s1, lo, hi, rounds, control);
}

// ---------------------------------------------------------------------------
// Super-rulers.  Jumping over all rulers costs a full pass over their states
// per round (about log2 of the rulers in an orbit rounds).  Instead every
// ruler whose id is a multiple of 2^kSuperLog2 is a super-ruler: it follows
// the ruler chain to the next super-ruler once (ruler_super_walk), folding
// the segment minima and stamping super_of[r] on the rulers it passes; the
// jumping then runs over the 2^kSuperLog2 times smaller super states.  Ruler
// cycles without a super-ruler are closed by ruler_super_short, which stamps
// their colour directly (kColourTag).  super_of[] starts at kUnset.
// ---------------------------------------------------------------------------
constexpr uint32_t kSuperLog2 = 4;

// Rulers [rlo, rhi) are this call's (ruler_range); their super-rulers are
// the multiples of 2^kSuperLog2 among them.
__device__ __forceinline__ void ruler_super_walk_run(Grid grid, const uint4* __restrict__ state,
    uint32_t rlo, uint32_t rhi, uint4* __restrict__ sstate, uint32_t* __restrict__ super_of,
    uint32_t* control) {
    if (*(volatile uint32_t*)(control + kCtlHard) != 0) {
        return; // the level is coloured by union-find
    }
    const uint32_t slo = (rlo + (1u << kSuperLog2) - 1) >> kSuperLog2;
    const uint32_t shi = (rhi + (1u << kSuperLog2) - 1) >> kSuperLog2;
    uint64_t first = 0;
    while (claim_chunk(control + kCtlClaimSuper, blockDim.x, shi - slo, &first)) {
        const uint64_t i = slo + first + threadIdx.x;
        if (i >= shi) {
            continue;
        }
        const uint32_t r = (uint32_t)i << kSuperLog2;
        const uint4 me = state[r];
        if (me.x == kNoRuler) {
            sstate[i] = make_uint4(kNoRuler, 0, 0, 0);
            continue;
        }
        super_of[r] = r;
        uint32_t ma = me.y, mb = me.z, cur = me.x;
        for (uint32_t hop = 0; (cur & ((1u << kSuperLog2) - 1)) != 0; ++hop) {
            if (cur < rlo || cur >= rhi || hop == kWalkCap) {
                atomicOr(control + kCtlHard, 1u);
                break;
            }
            const uint4 st = state[cur];
            super_of[cur] = r;
            ma = min(ma, st.y);
            mb = min(mb, st.z);
            cur = st.x;
        }
        sstate[i] = make_uint4(cur >> kSuperLog2, ma, mb, 0);
    }
}

__global__ void __launch_bounds__(256) ruler_super_walk(const uint4* __restrict__ state,
    uint32_t rlo, uint32_t rhi, uint4* __restrict__ sstate, uint32_t* __restrict__ super_of,
    uint32_t* control) {
    ruler_super_walk_run(launch_grid(), state, rlo, rhi, sstate, super_of, control);
}

// Ruler cycles that contain no super-ruler: thread per ruler no super walk
// reached; the ruler with the smallest id of its cycle folds the cycle's
// minima and stamps the colour on every ruler of it.
__device__ __forceinline__ void ruler_super_short_run(Grid grid, const uint4* __restrict__ state,
    uint32_t rlo, uint32_t rhi, uint32_t* __restrict__ super_of, uint32_t* control) {
    if (*(volatile uint32_t*)(control + kCtlHard) != 0) {
        return;
    }
    for (uint32_t r = rlo + grid.bid * blockDim.x + threadIdx.x; r < rhi;
         r += grid.nblk * blockDim.x) {
        if (super_of[r] != kUnset) {
            continue;
        }
        const uint4 me = state[r];
        if (me.x == kNoRuler) {
            continue;
        }
        uint32_t ma = me.y, mb = me.z, cur = me.x;
        bool smallest = true, closed = false;
        for (uint32_t hop = 0; hop < kWalkCap; ++hop) {
            if (cur < rlo || cur >= rhi) {
                break;
            }
            if (cur == r) {
                closed = true;
                break;
            }
            if (cur < r) {
                smallest = false; // that ruler's thread closes this cycle
                closed = true;
                break;
            }
            const uint4 st = state[cur];
            ma = min(ma, st.y);
            mb = min(mb, st.z);
            cur = st.x;
        }
        if (!closed) {
            atomicOr(control + kCtlHard, 1u);
            continue;
        }
        if (!smallest) {
            continue;
        }
        const uint32_t colour = kColourTag | (ma > mb ? 1u : 0u);
        cur = r;
        for (uint32_t hop = 0; hop < kWalkCap; ++hop) {
            super_of[cur] = colour;
            cur = state[cur].x;
            if (cur == r || cur < rlo || cur >= rhi) {
                break;
            }
        }
    }
}

__global__ void __launch_bounds__(256) ruler_super_short(const uint4* __restrict__ state,
    uint32_t rlo, uint32_t rhi, uint32_t* __restrict__ super_of, uint32_t* control) {
    ruler_super_short_run(launch_grid(), state, rlo, rhi, super_of, control);
}

// After the jumping: every ruler's colour, stamped into super_of in place
// of its super-ruler (kColourTag | colour, the form ruler cycles without a
// super-ruler already have), so level_finalize resolves a vertex's owner
// with one dependent load instead of two.  The super-ruler states read here
// are the buffer the last jumping round wrote (kCtlFinal).
__device__ __forceinline__ void ruler_colour_run(Grid grid, uint32_t rlo, uint32_t rhi,
    uint32_t* __restrict__ super_of, const uint4* __restrict__ s0, const uint4* __restrict__ s1,
    const uint32_t* control) {
    if (*(volatile const uint32_t*)(control + kCtlHard) != 0) {
        return; // the level is coloured by union-find
    }
    const uint4* state = control[kCtlFinal] ? s1 : s0;
    for (uint32_t r = rlo + grid.bid * blockDim.x + threadIdx.x; r < rhi;
         r += grid.nblk * blockDim.x) {
        const uint32_t so = super_of[r];
        if (so == kUnset || (so & kColourTag) != 0) {
            continue;
        }
        const uint4 st = state[so >> kSuperLog2];
        super_of[r] = kColourTag | (st.y > st.z ? 1u : 0u);
    }
}

__global__ void __launch_bounds__(256) ruler_colour(uint32_t rlo, uint32_t rhi,
    uint32_t* super_of, const uint4* s0, const uint4* s1, const uint32_t* control) {
    ruler_colour_run(launch_grid(), rlo, rhi, super_of, s0, s1, control);
}

// Clears the level's control words; `force_union_find` pre-sets the hard
// flag so the level is coloured by union-find (a test hook for that path).
__device__ __forceinline__ void control_reset_run(Grid grid, uint32_t* control, uint32_t force_union_find) {
    if (threadIdx.x < kCtlWords) {
        control[threadIdx.x] = threadIdx.x == kCtlHard ? force_union_find : 0u;
    }
}

__global__ void control_reset(uint32_t* control, uint32_t force_union_find) {
    control_reset_run(launch_grid(), control, force_union_find);
}

// Colours (from the walks, or from union-find when the level fell back),
// children and the colour bitmap: kResolveItems pair-nodes per thread.
// Blocks claim chunks in address order so the finds (or ruler-state reads)
// of a chunk stay within the nodes it covers.  Every thread of a block runs
// every claimed chunk (the colour bitmap is assembled with warp shuffles).
template <typename T>
__device__ __forceinline__ void level_finalize_run(Grid grid, const Plan* __restrict__ plan,
    uint32_t level, const T* __restrict__ src, const uint32_t* __restrict__ owner,
    const uint32_t* __restrict__ super_of, const uint4* __restrict__ state0,
    const uint4* __restrict__ state1, uint32_t* uf,
    uint32_t* __restrict__ xbits, uint32_t* __restrict__ dst, uint32_t* control,
    uint32_t* status) {
    const LevelInfo& lv = plan->levels[level];
    const uint32_t cap = (uint32_t)lv.cap;
    const uint32_t pcap = (uint32_t)lv.pcap;
    const uint32_t ccap = (uint32_t)plan->levels[level + 1].cap;
    // this call's pair-nodes [lo_pair, end); chunks start at a 32-pair
    // boundary at or below lo_pair so colour words are written whole
    const NodeRange nr = level_nodes(*plan, level);
    const uint64_t lo_pair = nr.lo * pcap;
    const uint64_t end = lo_pair + ((uint64_t)pcap << nr.shift);
    const uint64_t begin = lo_pair & ~31ull;
    const uint64_t total = end - begin;
    const bool hard = control[kCtlHard] != 0;
    const uint4* state = control[kCtlFinal] ? state1 : state0;
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t chunk = (uint64_t)blockDim.x * kResolveItems;
    // Walk levels claim chunks in order (ruler states of the nodes in flight
    // stay in L2), and so do union-find levels with nodes far above L2 size
    // (the finds of neighbouring chunks share the top of their trees).  On
    // union-find levels with nodes near L2 size, claimed chunks would crowd
    // every find in flight onto the root chains of one or two nodes' large
    // components, which then serialise: those stride over the whole level
    // (at 2^30 uniform entries, claimed order took 18.5 -> 12.5 ms on the
    // 2^30-slot level but 14 -> 19 ms on 2^24-slot nodes).
    uint64_t first = (uint64_t)grid.bid * chunk;
    bool started = false;
    const bool claimed = !hard || cap > (1ull << BPB200_FINAL_STRIDE_LOG2);
    auto next_chunk = [&]() -> bool {
        if (claimed) {
            return claim_chunk(control + kCtlClaimFinal, chunk, total, &first);
        }
        if (started) {
            first += (uint64_t)grid.nblk * chunk;
        }
        started = true;
        return first < total;
    };
    while (next_chunk()) {
        const uint64_t p0 = begin + first + (uint64_t)threadIdx.x * kResolveItems;
        uint32_t j = (uint32_t)(p0 / pcap);
        uint32_t k = (uint32_t)(p0 - (uint64_t)j * pcap);
        uint32_t s = size_at(lv, level, j);
        uint32_t jj[kResolveItems], kk[kResolveItems], ss[kResolveItems], c[kResolveItems];
        uint32_t live = 0;
#pragma unroll
        for (int q = 0; q < kResolveItems; ++q) {
            jj[q] = j;
            kk[q] = k;
            ss[q] = s;
            c[q] = 0;
            if (p0 + q >= lo_pair && p0 + q < end && k < s - s / 2) live |= 1u << q;
            if (++k == pcap) {
                k = 0;
                ++j;
                s = size_at(lv, level, j);
            }
        }
        if (hard) {
            uint32_t x[kResolveItems];
            Found f[kResolveItems];
#pragma unroll
            for (int q = 0; q < kResolveItems; ++q) x[q] = (uint32_t)(p0 + q);
            uf_find_many<kResolveItems>(uf, x, f, live, status, true);
#pragma unroll
            for (int q = 0; q < kResolveItems; ++q) {
                if (live & (1u << q)) c[q] = f[q].bit ^ (uf[f[q].root] & 1u);
#if BPB200_RESOLVE_WRITEBACK
                // point the pair-node at its root (a true fact), so the
                // finds of the pair-nodes below it end one step later
                if ((live & (1u << q)) && f[q].root != x[q]) {
                    uf[x[q]] = (f[q].root << 1) | f[q].bit;
                }
#endif
            }
        } else {
            // ruler id (or direct colour) of vertex 2k: every even vertex is
            // a ruler, stamped by the ruler walk that passes it, or stamped
            // by the short walk of its ruler-free orbit
            uint32_t id[kResolveItems];
#pragma unroll
            for (int q = 0; q < kResolveItems; ++q) {
                if (!(live & (1u << q))) continue;
                const uint32_t slot = jj[q] * cap + 2 * kk[q];
                id[q] = is_ruler_slot(slot) ? slot >> kRulerLog2 : owner[jj[q] * pcap + kk[q]];
            }
#pragma unroll
            for (int q = 0; q < kResolveItems; ++q) {
                if (!(live & (1u << q))) continue;
                uint32_t colour;
                if (id[q] == kUnset) {
                    atomicOr(status, kErrInconsistent); // a walk must have reached it
                    colour = 0;
                } else if (id[q] & kColourTag) {
                    colour = id[q] & 1u;
                } else {
                    // ruler -> its super-ruler's orbit minima (or a colour
                    // stamped on a super-free ruler cycle)
                    const uint32_t so = super_of[id[q]];
                    if (so == kUnset) {
                        atomicOr(status, kErrInconsistent);
                        colour = 0;
                    } else if (so & kColourTag) {
                        colour = so & 1u;
                    } else {
                        const uint4 st = state[so >> kSuperLog2];
                        colour = st.y > st.z ? 1u : 0u;
                    }
                }
                c[q] = colour;
            }
        }
        uint32_t mine = 0; // this lane's kResolveItems colour bits
#pragma unroll
        for (int q = 0; q < kResolveItems; ++q) {
            if (!(live & (1u << q))) continue;
            mine |= c[q] << q;
            const uint64_t node = (uint64_t)jj[q] * cap;
            const uint64_t left = (uint64_t)(2 * jj[q]) * ccap;
            const uint64_t right = (uint64_t)(2 * jj[q] + 1) * ccap;
            const uint32_t half = ss[q] / 2;
            if (kk[q] < half) {
                const uint32_t va = (uint32_t)src[node + 2 * kk[q] + c[q]];
                const uint32_t vb = (uint32_t)src[node + 2 * kk[q] + 1 - c[q]];
                dst[left + kk[q]] = va >> 1;
                dst[right + kk[q]] = vb >> 1;
            } else {
                dst[left + kk[q]] = (uint32_t)(src[node + ss[q] - 1] >> 1);
            }
        }
        // 32 / kResolveItems lanes hold one 32-pair colour word
        constexpr uint32_t kWordLanes = 32 / kResolveItems;
        uint32_t v = mine << ((lane & (kWordLanes - 1)) * kResolveItems);
#pragma unroll
        for (uint32_t d = 1; d < kWordLanes; d <<= 1) {
            v |= __shfl_xor_sync(0xffffffffu, v, d);
        }
        if ((lane & (kWordLanes - 1)) == 0 && p0 < end) {
            xbits[p0 >> 5] = v;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(256, BPB200_FINAL_MIN_BLOCKS) level_finalize(const Plan* __restrict__ plan,
    uint32_t level, const T* __restrict__ src, const uint32_t* __restrict__ owner,
    const uint32_t* __restrict__ super_of, const uint4* __restrict__ state0,
    const uint4* __restrict__ state1, uint32_t* uf,
    uint32_t* __restrict__ xbits, uint32_t* __restrict__ dst, uint32_t* control,
    uint32_t* status) {
    level_finalize_run<T>(launch_grid(), plan, level, src, owner, super_of, state0, state1, uf, xbits, dst, control, status);
}

} // namespace bpb200
