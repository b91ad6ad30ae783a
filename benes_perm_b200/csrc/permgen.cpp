// SPDX-License-Identifier: Apache-2.0
//
// Seeded synthetic permutations for the benchmark and tests.
//
// Randomness: xoshiro256** (Blackman and Vigna), state seeded with four
// successive splitmix64 outputs starting from `seed`.  Bounded draws in
// [0, range) use Lemire's multiply-shift with rejection ("Fast Random Integer
// Generation in an Interval", 2019).  Shuffles run i = n-1 down to 1:
// Fisher-Yates swaps a[i] with a[j], j uniform in [0, i]; Sattolo's variant
// draws j in [0, i - 1] and yields a single n-cycle.
//
// The swap loop is sequential, but the draws do not depend on the array, so
// the draws for the next block of steps are made first and their target
// slots prefetched; that keeps many cache misses in flight and makes a 2^30
// shuffle take seconds instead of minutes.
#include "../../include/benes_b200.h"

#include <cstdint>
#include <cstring>

namespace {

struct Xoshiro {
    uint64_t s[4];

    static uint64_t splitmix(uint64_t& x) {
        uint64_t z = (x += 0x9e3779b97f4a7c15ull);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return z ^ (z >> 31);
    }
    explicit Xoshiro(uint64_t seed) {
        for (auto& v : s) {
            v = splitmix(seed);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t out = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return out;
    }
    // uniform in [0, range), range >= 1
    uint64_t below(uint64_t range) {
        unsigned __int128 m = (unsigned __int128)next() * range;
        uint64_t low = (uint64_t)m;
        if (low < range) {
            const uint64_t floor = (0 - range) % range;
            while (low < floor) {
                m = (unsigned __int128)next() * range;
                low = (uint64_t)m;
            }
        }
        return (uint64_t)(m >> 64);
    }
};

template <typename T>
void shuffle(T* a, uint64_t n, uint64_t seed, bool single_cycle) {
    for (uint64_t i = 0; i < n; ++i) {
        a[i] = (T)i;
    }
    if (n < 2) {
        return;
    }
    Xoshiro rng(seed);
    constexpr uint64_t kBlock = 64;
    uint64_t draws[kBlock];
    uint64_t i = n - 1;
    while (i >= 1) {
        const uint64_t steps = i < kBlock ? i : kBlock;
        for (uint64_t t = 0; t < steps; ++t) {
            const uint64_t at = i - t;
            draws[t] = rng.below(single_cycle ? at : at + 1);
            __builtin_prefetch(a + draws[t], 1, 0);
        }
        for (uint64_t t = 0; t < steps; ++t) {
            const uint64_t at = i - t;
            const T tmp = a[at];
            a[at] = a[draws[t]];
            a[draws[t]] = tmp;
        }
        i -= steps;
    }
}

template <typename T>
int fill(uint32_t kind, uint64_t seed, uint64_t n, T* out) {
    switch (kind) {
    case 0:
        shuffle(out, n, seed, false);
        return 0;
    case 1:
        shuffle(out, n, seed, true);
        return 0;
    case 2:
        for (uint64_t i = 0; i < n; ++i) out[i] = (T)i;
        return 0;
    case 3:
        for (uint64_t i = 0; i < n; ++i) out[i] = (T)(n - 1 - i);
        return 0;
    case 4: {
        if (n == 0 || (n & (n - 1)) != 0) {
            return BPB200_INVALID_ARGUMENT;
        }
        uint32_t bits = 0;
        while ((1ull << bits) < n) ++bits;
        for (uint64_t i = 0; i < n; ++i) {
            uint64_t r = 0;
            for (uint32_t b = 0; b < bits; ++b) r |= ((i >> b) & 1ull) << (bits - 1 - b);
            out[i] = (T)r;
        }
        return 0;
    }
    default:
        return BPB200_INVALID_ARGUMENT;
    }
}

} // namespace

extern "C" int bpb200_fill_permutation(uint32_t kind, uint64_t seed, uint64_t count,
    uint32_t entry_bytes, void* out) {
    if (entry_bytes == 4) {
        if (count > 0xffffffffull + 1) return BPB200_INVALID_ARGUMENT;
        return fill(kind, seed, count, static_cast<uint32_t*>(out));
    }
    if (entry_bytes == 8) {
        return fill(kind, seed, count, static_cast<uint64_t*>(out));
    }
    return BPB200_INVALID_ARGUMENT;
}
