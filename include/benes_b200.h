/* SPDX-License-Identifier: Apache-2.0
 *
 * C ABI of the B200 compression backend for benes-perm.
 *
 * Every entry point is plain C: pointers, sizes and status codes, no C++ or
 * torch types.  The reference library binds these from a thin C++ shim that
 * plugs in beside its other accelerated backends (src/internal.hpp:1190-1197,
 * src/backends_stub.cpp:25-40); the status codes map one-to-one onto the
 * exception types the reference throws.
 */
#ifndef BENES_B200_H
#define BENES_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  Reference exception each one becomes in the C++ shim. */
#define BPB200_OK 0
#define BPB200_INVALID_ARGUMENT 1 /* std::invalid_argument (bad input or format) */
#define BPB200_OVERFLOW 2         /* std::overflow_error (checked size arithmetic) */
#define BPB200_LENGTH 3           /* std::length_error (does not fit) */
#define BPB200_RUNTIME 4          /* std::runtime_error (CUDA or device status) */
#define BPB200_OUT_OF_RANGE 5     /* std::out_of_range (lookup index >= size) */
#define BPB200_UNAVAILABLE 6      /* std::runtime_error("b200 backend is unavailable") */

/* benes::FormatOptions (include/benes/benes.hpp:32-39).  A cluster count of
 * zero selects the reference's balanced default (src/internal.hpp:328-338). */
typedef struct bpb200_format {
    uint8_t middle_group_log2;    /* 1..5; the reference default is 5 */
    uint8_t middle_placement;     /* 0 separate, 1 embedded_input, 2 embedded_output */
    uint8_t input_cluster_count;  /* entries used in input_clusters */
    uint8_t output_cluster_count; /* entries used in output_clusters */
    uint8_t input_clusters[64];
    uint8_t output_clusters[64];
} bpb200_format;

/* Replaces detail::cuda_available() (src/internal.hpp:1190; stub pattern
 * src/backends_stub.cpp:25-26): nonzero when a B200-class (sm_100) device is
 * visible and the kernels of this library can run on it. */
int bpb200_available(void);

/* Replaces backend_name(Backend::cuda) (src/benes.cpp:772-780): "b200". */
const char* bpb200_backend_name(void);

/* make_layout(count, format).end_offset (src/internal.hpp:389-429): the
 * exact blob size in bytes.  Same validation and error kinds as the
 * reference (invalid format -> INVALID_ARGUMENT, overflow -> OVERFLOW). */
int bpb200_encoded_size(uint64_t count, const bpb200_format* format,
    uint64_t* blob_bytes, char* err, size_t err_len);

/* Replaces detail::compress_compact_cuda(span<const uint32_t|uint64_t>,
 * FormatOptions) (src/internal.hpp:1192-1197; src/cuda/benes_cuda.cu:1155,
 * 1334).  `entries` is host memory holding `count` little-endian values of
 * `entry_bytes` (4 or 8) bytes.  Writes exactly `blob_len` bytes (which must
 * equal bpb200_encoded_size) into `blob`, byte-identical to the reference's
 * portable encoder.  `device_seconds` (may be NULL) receives the on-device
 * time, the value the reference stores with set_last_device_seconds (for
 * inputs of 2^25 entries and more, from the first level-0 kernel on, which
 * starts while the input is still being uploaded).
 * Errors: INVALID_ARGUMENT "input must contain every value from zero through
 * size minus one" for a non-permutation, exactly like validate_permutation
 * (src/benes.cpp:152-173).  Parts of the blob are copied into `blob` while
 * the encode still runs, so after an error its contents are unspecified. */
int bpb200_compress(const void* entries, uint64_t count, uint32_t entry_bytes,
    const bpb200_format* format, uint8_t* blob, uint64_t blob_len,
    double* device_seconds, char* err, size_t err_len);

/* Device-resident form of bpb200_compress (no reference counterpart; the
 * reference copies host spans, src/cuda/benes_cuda.cu:1397-1409).
 * `d_entries` and `d_blob` are device pointers on the current device;
 * `d_entries` must be aligned to entry_bytes and `d_blob` 4-byte aligned
 * with room for blob_len rounded up to a multiple of 4 bytes (misaligned
 * pointers return BPB200_INVALID_ARGUMENT before any device work; the same
 * holds for the batched form).  Work is queued on `stream` (a cudaStream_t, NULL for
 * the legacy default stream); the call returns after the work completes and
 * the device status word has been checked. */
int bpb200_compress_device(const void* d_entries, uint64_t count, uint32_t entry_bytes,
    const bpb200_format* format, uint8_t* d_blob, uint64_t blob_len, void* stream,
    double* device_seconds, char* err, size_t err_len);

/* Subtree sharding of one permutation over `shards` (a power of two) GPUs
 * or calls; no reference counterpart (the reference splits the same
 * recursion across host threads, src/benes.cpp:317-350).  With k =
 * log2(shards), every shard runs routing levels 0..k-1 in full (they need
 * the whole permutation; no exchange step) and, from level k on, only the
 * subtree of level-k node `shard`, the 2^(l-k) consecutive nodes of each
 * level l below it, through to their middle-group ranks.  Shard 0 alone
 * writes levels 0..k-1's switches and the header; every other bit of the
 * blob belongs to exactly one shard, so the byte-wise sum (or OR) of the
 * shards' blobs is the whole blob, byte-identical to bpb200_compress_device.
 * Same arguments as bpb200_compress_device otherwise; INVALID_ARGUMENT when
 * shards is not a power of two, shard >= shards, or the permutation has
 * fewer global routing levels than k. */
int bpb200_compress_device_shard(const void* d_entries, uint64_t count, uint32_t entry_bytes,
    const bpb200_format* format, uint8_t* d_blob, uint64_t blob_len, uint32_t shard,
    uint32_t shards, void* stream, double* device_seconds, char* err, size_t err_len);

/* Allocation-free form of bpb200_compress_device.  No counterpart in the
 * reference: its backends all allocate per call.  For callers that cannot
 * call cudaMalloc: processes whose device memory belongs to a pooling
 * allocator that must account for every byte, and latency-critical paths
 * that must not pay for the device-wide synchronisation cudaMalloc/cudaFree
 * can imply.  Same arguments and result bytes as bpb200_compress_device
 * (device input and blob, work queued on `stream`), but every byte of
 * scratch comes from one fixed device array inside this library (under
 * 8 MB, present on every GPU that loads the library until the process
 * exits), so it accepts at most 262144 (2^18) entries and returns
 * BPB200_LENGTH above that.  It calls no cudaMalloc/cudaFree.  Like
 * bpb200_compress_device, each call uploads its plan from host memory,
 * waits for `stream` to finish the work and reads the device status word
 * back before it returns.  The first call on each device looks up the
 * array's device address (cudaGetSymbolAddress); make that first call
 * before capturing any stream.  All calls share the one array: calls whose
 * GPU work overlaps (different streams or host threads without ordering)
 * race and corrupt each other's results.  Each call clears what it needs
 * cleared (blob, status word, validation sentinels). */
int bpb200_compress_device_noalloc(const void* d_entries, uint64_t count,
    uint32_t entry_bytes, const bpb200_format* format, uint8_t* d_blob, uint64_t blob_len,
    void* stream, char* err, size_t err_len);

/* Replaces benes::compress_file (src/benes.cpp:498-553) for the b200
 * backend: encodes the raw little-endian permutation file `input_path`
 * (values of `input_width` = 4 or 8 bytes, the InputValueWidth values) and
 * writes the blob to `output_path`, byte-identical to compress_file with the
 * portable backend.  The file is streamed to the device through pinned
 * chunks (reads overlap the upload; there is no host decode pass) and the
 * blob streamed back the same way.  Errors, in the reference's order:
 * RUNTIME "cannot open permutation input file"; INVALID_ARGUMENT
 * "permutation input has an invalid element width or size" (width not 4/8,
 * empty file, size not a multiple of the width, not a regular file);
 * UNAVAILABLE without a
 * usable GPU; RUNTIME "failed to read permutation input file"; then every
 * error of bpb200_compress; RUNTIME "failed to write compressed permutation
 * file".  The output file is created only after the encode succeeded. */
int bpb200_compress_file(const char* input_path, const char* output_path,
    uint32_t input_width, const bpb200_format* format, double* device_seconds,
    char* err, size_t err_len);

/* ---------------------------------------------------------------- batched
 * No reference counterpart (the reference compresses one permutation per
 * call).  Compresses many device-resident permutations of uneven sizes in
 * one call: every permutation of at most 8192 entries is encoded by a single
 * batched launch (one CTA each); larger ones run their level kernels
 * concurrently on pooled workspaces.  Each request's output bytes equal
 * bpb200_compress_device's.  Per-request results land in `status`/`error`;
 * the return value is the first failing status or BPB200_OK.
 * `kernel_launches` (may be NULL) receives the number of kernel launches. */
typedef struct bpb200_request {
    const void* d_entries;  /* device input: count values of entry_bytes */
    uint64_t count;
    uint32_t entry_bytes;   /* 4 or 8 */
    uint32_t reserved;
    bpb200_format format;
    uint8_t* d_blob;        /* device output, 4-byte aligned, rounded-up size */
    uint64_t blob_len;      /* bpb200_encoded_size */
    int status;             /* out: BPB200_* */
    char error[124];        /* out: message when status != 0 */
} bpb200_request;

int bpb200_compress_batch(bpb200_request* requests, uint32_t count, void* stream,
    uint32_t* kernel_launches);

/* ---------------------------------------------------------------- serving
 * No reference counterpart.  A request loop on its own threads: requests
 * (host input, host blob) are admitted in arrival order while their device
 * footprint fits `hbm_budget_bytes`; single-tile requests admitted together
 * are encoded by one batched launch (up to `max_batch` per launch), larger
 * ones by up to `workers` concurrent worker threads; admission resumes as
 * requests complete.  Input and blob memory must stay valid until
 * bpb200_server_wait returns for the ticket.  Latency runs from submit to
 * the blob being written. */
typedef struct bpb200_server bpb200_server;

typedef struct bpb200_server_stats {
    uint64_t submitted;
    uint64_t completed;
    uint64_t failed;
    uint64_t entries;          /* entries of completed requests */
    uint64_t kernel_launches;
    double p50_seconds;        /* latency percentiles of completed requests */
    double p99_seconds;
    double mean_seconds;
} bpb200_server_stats;

bpb200_server* bpb200_server_create(uint64_t hbm_budget_bytes, uint32_t max_batch,
    uint32_t workers, char* err, size_t err_len);
int bpb200_server_submit(bpb200_server* server, const void* entries, uint64_t count,
    uint32_t entry_bytes, const bpb200_format* format, uint8_t* blob, uint64_t blob_len,
    uint64_t* ticket);
int bpb200_server_wait(bpb200_server* server, uint64_t ticket, double* latency_seconds,
    char* err, size_t err_len);
int bpb200_server_get_stats(bpb200_server* server, bpb200_server_stats* stats);
void bpb200_server_destroy(bpb200_server* server);

/* Seeded synthetic permutations used by the benchmark and the tests
 * (workload generator, not part of the reference).  kind: 0 Fisher-Yates
 * uniform, 1 Sattolo single cycle, 2 identity, 3 reverse, 4 bit reversal
 * (count must be a power of two).  Randomness: xoshiro256** seeded from
 * splitmix64(seed), bounded draws by Lemire's multiply-shift with rejection.
 * `out` holds count values of entry_bytes (4 or 8). */
int bpb200_fill_permutation(uint32_t kind, uint64_t seed, uint64_t count,
    uint32_t entry_bytes, void* out);

/* Releases cached device workspaces (no reference counterpart). */
void bpb200_shutdown(void);

/* Per-kernel device timing (tracing hook; the reference only records total
 * device seconds, src/benes.cpp:119-125).  When enabled, every kernel launch
 * of later calls is bracketed by CUDA events.  bpb200_last_profile reports,
 * for the calling thread's last call, seconds and launch counts per kernel
 * kind (0 prologue, 1 inverse, 2 descriptors, 3 union, 4 orient, 5 resolve,
 * 6 output bits, 7 tile, 8 emit, 9 walk, 10 jump, 11 partitioned inverse)
 * and the total number of kernel launches; it returns the number of kinds. */
void bpb200_set_profiling(int enabled);

/* Launch tuning per size class (no reference counterpart; the reference's
 * CUDA backend has one fixed launch shape, src/cuda/benes_cuda.cu:16).  None
 * of these changes a byte of output.  The library reads its table from
 * tuning.json beside the shared object (made by benes_perm_b200/tune.py;
 * BPB200_TUNING_FILE names another file, "none" disables it); a class of
 * ceil(log2 count) the table lacks takes its nearest class. */
typedef struct bpb200_tuning {
    uint32_t walk_blocks_per_sm; /* persistent orbit-walk blocks per SM, 1..8 */
    uint32_t walk_max_log2;      /* largest node coloured by orbit walks (log2 entries) */
    uint32_t jump_block_log2;    /* largest super-ruler count jumped inside one CTA (log2) */
    uint32_t tile_max_log2;      /* largest node encoded by the shared-memory tile (log2), 9..14 */
} bpb200_tuning;

/* The setting calls with `count` entries use. */
int bpb200_get_tuning(uint64_t count, bpb200_tuning* out);

/* Tuner and test hook: a non-null setting is used by every later call
 * (values clamped to their ranges); NULL returns to the table. */
int bpb200_set_tuning(const bpb200_tuning* forced);

/* Test hook: 1 makes later calls colour every global level with the
 * union-find kernels instead of the orbit walks (the path the walks fall
 * back to on contrived inputs); 2 runs the walks and then colours each walk
 * level with that fallback anyway, as if a walk had given up (single-call
 * paths; the batched groups treat 2 as 0); 0 restores the default.  Output
 * bytes are identical in every mode. */
void bpb200_set_colouring(int union_find_only);

/* Geometry of the encode the library would run for (count, format): the
 * routing depth and the first level handled by the shared-memory tile
 * kernel (levels above it run as global-memory level kernels). */
int bpb200_describe(uint64_t count, const bpb200_format* format, uint32_t* depth,
    uint32_t* tile_level);
int bpb200_last_profile(double* seconds, uint32_t* launches, int kinds,
    uint32_t* total_launches);

/* Per-launch detail of the same profile: kernel kind, routing level and
 * seconds of each timed launch, in launch order (up to `capacity`); returns
 * the number of timed launches of the last call. */
int bpb200_last_profile_launches(int* kinds, int* levels, double* seconds, int capacity);

/* Address probes of the closed-form layout (test hooks, no device work):
 * section-relative bit of switch `pair` of node `node` at routing level
 * `level` (side 0 input, 1 output), and the first rank bit of leaf `node`
 * with its section (0 input, 1 output, 2 middle).  They restate
 * SectionAddress::switch_bit / middle_bit (src/internal.hpp:486-517). */
int bpb200_probe_switch_bit(uint64_t count, const bpb200_format* format, int side,
    uint32_t level, uint64_t node, uint64_t pair, uint64_t* bit);
int bpb200_probe_rank_bit(uint64_t count, const bpb200_format* format, uint32_t level,
    uint64_t node, int* section, uint64_t* bit);

/* Batch lookup verifier: a read-only device twin of the reference's lookup
 * (src/internal.hpp:1035-1124, behind CompressedPermutationView::forward /
 * inverse), for checking every entry of blobs too large to re-encode on the
 * host.  The library's own lookup is not replaced.  For each i <
 * query_count, d_out[i] = p[q] (inverse = 0) or p^-1[q] (inverse != 0),
 * q = d_queries[i], or q = i when d_queries is NULL; p is the permutation
 * of `count` entries encoded in the device blob of blob_len bytes with
 * `format`.  Queued on `stream`; returns after it completes.  A query >=
 * count returns BPB200_OUT_OF_RANGE ("permutation lookup is out of range",
 * std::out_of_range in the reference) with that entry set to UINT64_MAX. */
int bpb200_lookup_device(const void* d_blob, uint64_t blob_len, uint64_t count,
    const bpb200_format* format, const uint64_t* d_queries, uint64_t query_count, int inverse,
    uint64_t* d_out, void* stream, char* err, size_t err_len);

/* Roofline probe (no reference counterpart): random 4-byte access rates
 * of the current GPU over an array of 2^log2_words words (10..31; resident
 * in L2 or not): independent random reads, independent random writes and
 * dependent read chains, in accesses per second.  Allocates and frees its
 * own buffer.  The encoder's kernels are bound by such accesses, so these
 * rates, not the streaming copy bandwidth, bound them. */
int bpb200_probe_random_access(uint32_t log2_words, double* reads_per_s,
    double* writes_per_s, double* chain_steps_per_s);

/* Host evaluation of the verifier's per-query walk (test hook, no device
 * work): one forward or inverse lookup in a host blob. */
int bpb200_probe_lookup(uint64_t count, const bpb200_format* format, const uint8_t* blob,
    uint64_t blob_len, uint64_t value, int inverse, uint64_t* out);

#ifdef __cplusplus
}
#endif

#endif /* BENES_B200_H */
