/* SPDX-License-Identifier: Apache-2.0
 *
 * CPU oracle for the benes-perm compact encoder.  TEST INFRASTRUCTURE ONLY:
 * tests, the smoke check and the benchmark's CPU-baseline leg use it as the
 * checker.  The B200 library never links, loads or calls it.
 *
 * It restates, in plain C, the reference's single-threaded portable encoder
 * (src/benes.cpp:150-416 of bramcohen/benes-perm), the format core it
 * depends on (src/internal.hpp:148-718) and the lookup used to verify blobs
 * (src/internal.hpp:1035-1124).  Its bytes are pinned against the
 * reference's golden blobs and against the reference compiled from its own
 * sources (oracle/_ref, see oracle/Makefile).
 */
#ifndef BENES_ORACLE_H
#define BENES_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes; they mirror the C++ exception types the reference throws. */
enum {
    ORACLE_OK = 0,
    ORACLE_INVALID_ARGUMENT = 1, /* std::invalid_argument */
    ORACLE_OVERFLOW = 2,         /* std::overflow_error */
    ORACLE_LENGTH = 3,           /* std::length_error */
    ORACLE_RUNTIME = 4,          /* std::runtime_error / out_of_range */
    ORACLE_LOGIC = 5             /* std::logic_error */
};

/* FormatOptions (include/benes/benes.hpp:32-39).  Empty cluster lists select
 * the balanced default, exactly like the reference. */
typedef struct oracle_format {
    uint8_t middle_group_log2;
    uint8_t middle_placement; /* 0 separate, 1 embedded_input, 2 embedded_output */
    uint8_t input_cluster_count;
    uint8_t output_cluster_count;
    uint8_t input_clusters[64];
    uint8_t output_clusters[64];
} oracle_format;

/* Layout (src/internal.hpp:22-33) after normalize_format. */
typedef struct oracle_layout {
    uint64_t size;
    uint64_t network_size;
    uint64_t switch_bits;
    uint64_t middle_bits;
    uint64_t input_offset;
    uint64_t output_offset;
    uint64_t middle_offset;
    uint64_t end_offset;
    oracle_format format; /* normalized */
} oracle_layout;

int oracle_make_layout(uint64_t count, const oracle_format* format,
    oracle_layout* layout, char* err, size_t err_len);

/* benes::compress(perm, {portable_cpu, threads = 1, format}).
 * entry_bytes is 4 or 8.  The blob buffer must hold layout.end_offset bytes. */
int oracle_compress(const void* permutation, uint64_t count,
    uint32_t entry_bytes, const oracle_format* format,
    uint8_t* blob, uint64_t blob_capacity, uint64_t* blob_len,
    char* err, size_t err_len);

/* CompressedPermutationView construction checks (header + padding). */
int oracle_validate(const uint8_t* blob, uint64_t blob_len,
    char* err, size_t err_len);

/* CompressedPermutationView::forward / inverse. */
int oracle_lookup(const uint8_t* blob, uint64_t blob_len, uint64_t value,
    int inverse, uint64_t* result, char* err, size_t err_len);

/* Address probes used to test the device-side address formulas.  The node
 * is reached from the root by `depth` turns (0 = left/ceil, 1 = right/floor).
 * side 0 = input section, 1 = output section.  Bits are section relative. */
int oracle_switch_bit(uint64_t count, const oracle_format* format, int side,
    int depth, const uint8_t* turns, uint64_t pair, uint64_t* bit);
int oracle_middle_bit(uint64_t count, const oracle_format* format,
    int depth, const uint8_t* turns, uint64_t* bit);

/* factoradic_bit_count (src/internal.hpp:173-183). */
uint32_t oracle_factoradic_bits(uint32_t size);

/* Seeded workload permutations of the benchmark configs (not part of the
 * reference): kind 0 Fisher-Yates, 1 Sattolo single cycle, 2 identity,
 * 3 reverse, 4 bit reversal.  xoshiro256** seeded by splitmix64(seed),
 * Lemire bounded draws.  `out` holds count values of entry_bytes (4 or 8). */
int oracle_fill_permutation(uint32_t kind, uint64_t seed, uint64_t count,
    uint32_t entry_bytes, void* out);

#ifdef __cplusplus
}
#endif

#endif
