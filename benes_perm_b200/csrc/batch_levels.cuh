// SPDX-License-Identifier: Apache-2.0
//
// Batched level kernels: one launch runs one kernel step of one routing
// level for a whole group of permutations.
//
// The host builds, per routing level, a device work list of LevelJob
// entries, one per permutation whose level is still above its tile level:
// the permutation's plan and scratch, and for every kernel step the range
// of the launch's blocks that work on it (first[kind], blocks[kind]).  A
// block finds its job by binary search on `first`, then runs the same body
// as the one-permutation kernel over the job's share of the blocks (a Grid
// in place of blockIdx / gridDim).  Kernels that claim work from
// per-level counters keep claiming from the job's own control words, so
// the work in flight at any moment still covers a few nodes of one or two
// permutations.  A group of R permutations therefore needs one launch per
// kernel step per level instead of R, and the steps of short, latency-bound
// levels of different permutations (pointer-jumping rounds, small walks)
// run side by side on different SMs.
#pragma once

#include "kernels.cuh"
#include "tile.cuh"
#include "walk.cuh"

#include <cstdint>

namespace bpb200 {

enum BatchKind : int {
    kBReset = 0,
    kBInverse,
    kBDescriptors,
    kBWalk,
    kBWalkShort,
    kBSuperWalk,
    kBSuperShort,
    kBJumpBlock,
    kBJump,
    kBCheck,
    kBColour,
    kBUnion,
    kBOrient,
    kBFinalize,
    kBOutputs,
    kBatchKinds
};

// One permutation at one routing level of a batched launch sequence.
struct LevelJob {
    const Plan* plan;
    const void* src;         // this level's values (the caller's input at level 0)
    uint32_t* dst;           // children's values
    uint32_t* inv;           // this level's inverse
    uint32_t* child_inv;     // children's inverse (null when the children are tiles)
    uint32_t* owner;
    uint32_t* uf;
    uint32_t* xbits;
    uint32_t* ybits;
    uint4* state;            // ruler states
    uint4* sstate;           // super-ruler states: two buffers of `supers`
    uint32_t* super_of;
    uint32_t* control;       // the permutation's per-level control words
    uint32_t* status;
    NodeAddress* addr[2];
    uint32_t* blob;          // level 0 only: the blob whose header the reset writes
    uint32_t level;
    uint32_t src_bytes;      // 8 only at level 0 of a uint64 input
    uint32_t buckets;        // rulers
    uint32_t supers;         // super-rulers
    uint32_t rounds;         // jumping rounds (multi-launch form)
    uint32_t force_union_find;
    uint32_t header_bytes;   // level 0 only
    uint8_t header[84];
    uint32_t first[kBatchKinds];
    uint32_t blocks[kBatchKinds];
};

// One section's switch emission of one permutation at one level.
struct EmitJob {
    const Plan* plan;
    const uint32_t* bits;
    const NodeAddress* addr;
    uint32_t* blob;
    uint64_t full;           // full packets (block forms) or first packet (per-bit form)
    uint32_t level;
    int32_t side;
    uint32_t first;
    uint32_t blocks;
};

// Word fills (blob clearing, validation sentinels, super-ruler marks).
struct FillJob {
    uint32_t* ptr;
    uint64_t words;
    uint32_t value;
    uint32_t first;
    uint32_t blocks;
    uint32_t pad_;
};

// The job whose block range holds this block: the last job with
// first <= blockIdx.x (jobs that own no blocks share the next job's first
// and are skipped by taking the last).
template <typename Job, typename First>
__device__ __forceinline__ const Job* batch_job(const Job* jobs, uint32_t n, First first_of,
    Grid* g) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (first_of(jobs[mid]) <= blockIdx.x) lo = mid; else hi = mid;
    }
    return jobs + lo;
}

__device__ __forceinline__ const LevelJob* level_job(const LevelJob* jobs, uint32_t n, int kind,
    Grid* g) {
    const LevelJob* j = batch_job(jobs, n, [kind](const LevelJob& x) { return x.first[kind]; }, g);
    g->bid = blockIdx.x - j->first[kind];
    g->nblk = j->blocks[kind];
    return j;
}

__global__ void __launch_bounds__(256) batch_fill(const FillJob* jobs, uint32_t n) {
    Grid g;
    const FillJob* j = batch_job(jobs, n, [](const FillJob& x) { return x.first; }, &g);
    g.bid = blockIdx.x - j->first;
    g.nblk = j->blocks;
    if (g.bid >= g.nblk) return;
    for (uint64_t i = (uint64_t)g.bid * blockDim.x + threadIdx.x; i < j->words;
         i += (uint64_t)g.nblk * blockDim.x) {
        j->ptr[i] = j->value;
    }
}

// Control words of the level; at level 0 also the status word and the
// blob header (after the blob was cleared by batch_fill).
__global__ void __launch_bounds__(32) batch_reset(const LevelJob* jobs, uint32_t n) {
    Grid g;
    const LevelJob* j = level_job(jobs, n, kBReset, &g);
    if (g.bid >= g.nblk) return;
    control_reset_run(g, j->control, j->force_union_find);
    if (j->blob != nullptr) {
        if (threadIdx.x == 0) *j->status = 0;
        uint8_t* b = reinterpret_cast<uint8_t*>(j->blob);
        for (uint32_t i = threadIdx.x; i < j->header_bytes; i += blockDim.x) b[i] = j->header[i];
    }
}

__global__ void __launch_bounds__(256) batch_inverse(const LevelJob* jobs, uint32_t n) {
    Grid g;
    const LevelJob* j = level_job(jobs, n, kBInverse, &g);
    if (g.bid >= g.nblk) return;
    if (j->src_bytes == 8) {
        level_inverse_run<uint64_t>(g, j->plan, j->level, (const uint64_t*)j->src, j->inv, j->uf,
            j->owner, j->control + kCtlClaimInverse, j->status);
    } else {
        level_inverse_run<uint32_t>(g, j->plan, j->level, (const uint32_t*)j->src, j->inv, j->uf,
            j->owner, j->control + kCtlClaimInverse, j->status);
    }
}

__global__ void __launch_bounds__(256) batch_descriptors(const LevelJob* jobs, uint32_t n) {
    Grid g;
    const LevelJob* j = level_job(jobs, n, kBDescriptors, &g);
    if (g.bid >= g.nblk) return;
    level_descriptors_run(g, j->plan, j->level, j->addr[0], j->addr[1]);
}

__global__ void __launch_bounds__(256) batch_walk(const LevelJob* jobs, uint32_t n) {
    Grid g;
    const LevelJob* j = level_job(jobs, n, kBWalk, &g);
    if (g.bid >= g.nblk) return;
    if (j->src_bytes == 8) {
        level_walk_run<uint64_t>(g, j->plan, j->level, (const uint64_t*)j->src, j->inv, j->owner,
            j->state, j->control);
    } else {
        level_walk_run<uint32_t>(g, j->plan, j->level, (const uint32_t*)j->src, j->inv, j->owner,
            j->state, j->control);
    }
}

__global__ void __launch_bounds__(256) batch_walk_short(const LevelJob* jobs, uint32_t n) {
    Grid g;
    const LevelJob* j = level_job(jobs, n, kBWalkShort, &g);
    if (g.bid >= g.nblk) return;
    if (j->src_bytes == 8) {
        level_walk_short_run<uint64_t>(g, j->plan, j->level, (const uint64_t*)j->src, j->inv,
            j->owner, j->control);
    } else {
        level_walk_short_run<uint32_t>(g, j->plan, j->level, (const uint32_t*)j->src, j->inv,
            j->owner, j->control);
    }
}

__global__ void __launch_bounds__(256) batch_super_walk(const LevelJob* jobs, uint32_t n) {
    Grid g;
    const LevelJob* j = level_job(jobs, n, kBSuperWalk, &g);
    if (g.bid >= g.nblk) return;
    ruler_super_walk_run(g, j->state, 0u, j->buckets, j->sstate, j->super_of, j->control);
}

__global__ void __launch_bounds__(256) batch_super_short(const LevelJob* jobs, uint32_t n) {
    Grid g;
    const LevelJob* j = level_job(jobs, n, kBSuperShort, &g);
    if (g.bid >= g.nblk) return;
    ruler_super_short_run(g, j->state, 0u, j->buckets, j->super_of, j->control);
}

__global__ void __launch_bounds__(kJumpBlockThreads, 1) batch_jump_block(const LevelJob* jobs,
    uint32_t n) {
    Grid g;
    const LevelJob* j = level_job(jobs, n, kBJumpBlock, &g);
    if (g.bid >= g.nblk) return;
    ruler_jump_block_run(g, j->sstate, j->sstate + j->supers, 0u, j->supers, j->rounds,
        j->control);
}

__global__ void __launch_bounds__(256) batch_jump(const LevelJob* jobs, uint32_t n,
    uint32_t round) {
    Grid g;
    const LevelJob* j = level_job(jobs, n, kBJump, &g);
    if (g.bid >= g.nblk || round > j->rounds) return;
    uint4* s0 = j->sstate;
    uint4* s1 = j->sstate + j->supers;
    ruler_jump_run(g, (round & 1u) ? s1 : s0, (round & 1u) ? s0 : s1, 0u, j->supers, round,
        j->control);
}

__global__ void __launch_bounds__(32) batch_check(const LevelJob* jobs, uint32_t n,
    uint32_t round) {
    Grid g;
    const LevelJob* j = level_job(jobs, n, kBCheck, &g);
    if (g.bid >= g.nblk || round > j->rounds || threadIdx.x != 0) return;
    ruler_check_run(g, round, j->control);
}

__global__ void __launch_bounds__(256) batch_colour(const LevelJob* jobs, uint32_t n) {
    Grid g;
    const LevelJob* j = level_job(jobs, n, kBColour, &g);
    if (g.bid >= g.nblk) return;
    ruler_colour_run(g, 0u, j->buckets, j->super_of, j->sstate, j->sstate + j->supers,
        j->control);
}

__global__ void __launch_bounds__(256, BPB200_UNION_MIN_BLOCKS) batch_union(const LevelJob* jobs,
    uint32_t n) {
    Grid g;
    const LevelJob* j = level_job(jobs, n, kBUnion, &g);
    if (g.bid >= g.nblk) return;
    level_union_run(g, j->plan, j->level, j->inv, j->uf, j->control + kCtlHard,
        j->control + kCtlClaimUnion, j->status);
}

__global__ void __launch_bounds__(256) batch_orient(const LevelJob* jobs, uint32_t n) {
    Grid g;
    const LevelJob* j = level_job(jobs, n, kBOrient, &g);
    if (g.bid >= g.nblk) return;
    level_orient_run(g, j->plan, j->level, j->inv, j->uf, j->control + kCtlHard, j->status);
}

// Resident blocks per SM of batch_finalize (its job lookup costs registers
// that level_finalize does not need).
#ifndef BPB200_BATCH_FINAL_MIN_BLOCKS
#define BPB200_BATCH_FINAL_MIN_BLOCKS 4
#endif

__global__ void __launch_bounds__(256, BPB200_BATCH_FINAL_MIN_BLOCKS) batch_finalize(const LevelJob* jobs, uint32_t n) {
    Grid g;
    const LevelJob* j = level_job(jobs, n, kBFinalize, &g);
    if (g.bid >= g.nblk) return;
    if (j->src_bytes == 8) {
        level_finalize_run<uint64_t>(g, j->plan, j->level, (const uint64_t*)j->src, j->owner,
            j->super_of, j->sstate, j->sstate + j->supers, j->uf, j->xbits, j->dst, j->control,
            j->status);
    } else {
        level_finalize_run<uint32_t>(g, j->plan, j->level, (const uint32_t*)j->src, j->owner,
            j->super_of, j->sstate, j->sstate + j->supers, j->uf, j->xbits, j->dst, j->control,
            j->status);
    }
}

__global__ void __launch_bounds__(256) batch_outputs(const LevelJob* jobs, uint32_t n) {
    Grid g;
    const LevelJob* j = level_job(jobs, n, kBOutputs, &g);
    if (g.bid >= g.nblk) return;
    const bool global_child = j->child_inv != nullptr;
    level_outputs_run(g, j->plan, j->level, j->inv, j->xbits, j->ybits, j->child_inv,
        global_child ? j->owner : nullptr, global_child ? j->uf : nullptr);
}

// Emission forms (kernels.cuh), one launch per form over every (permutation,
// section) that uses it at this level.
enum EmitForm : int { kEmitWords = 0, kEmitTranspose, kEmitBlocks, kEmitBits, kEmitForms };

__global__ void __launch_bounds__(256) batch_emit(const EmitJob* jobs, uint32_t n, int form) {
    Grid g;
    const EmitJob* j = batch_job(jobs, n, [](const EmitJob& x) { return x.first; }, &g);
    g.bid = blockIdx.x - j->first;
    g.nblk = j->blocks;
    if (g.bid >= g.nblk) return;
    switch (form) {
    case kEmitWords:
        level_emit_words_run(g, j->plan, j->level, j->side, j->bits, j->addr, j->blob);
        break;
    case kEmitTranspose:
        level_emit_transpose_run(g, j->plan, j->level, j->side, j->bits, j->addr, j->blob,
            j->full);
        break;
    case kEmitBlocks:
        level_emit_blocks_run(g, j->plan, j->level, j->side, j->bits, j->addr, j->blob, j->full);
        break;
    default:
        level_emit_run(g, j->plan, j->level, j->side, j->bits, j->addr, j->blob, j->full);
        break;
    }
}

} // namespace bpb200
