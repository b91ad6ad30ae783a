/* SPDX-License-Identifier: Apache-2.0
 *
 * CPU oracle for the benes-perm compact encoder.  TEST INFRASTRUCTURE ONLY:
 * the B200 library never links, loads or calls this file.  It is a plain-C
 * restatement of the reference's single-threaded portable encoder; every
 * function names the reference file:line it follows.  The bytes it produces
 * are pinned against the reference's golden blobs and against the reference
 * built from its own sources (oracle/_ref).
 */
#include "benes_oracle.h"

#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

/* ------------------------------------------------------------------ errors */

typedef struct {
    jmp_buf jump;
    int code;
    char message[160];
} failure_t;

static void fail(failure_t* f, int code, const char* fmt, ...) {
    va_list args;
    va_start(args, fmt);
    vsnprintf(f->message, sizeof f->message, fmt, args);
    va_end(args);
    f->code = code;
    longjmp(f->jump, 1);
}

static void copy_error(const failure_t* f, char* err, size_t err_len) {
    if (err != NULL && err_len > 0) {
        snprintf(err, err_len, "%s", f->message);
    }
}

/* checked_add, src/internal.hpp:206-213 */
static uint64_t add_checked(failure_t* f, uint64_t a, uint64_t b) {
    if (b > UINT64_MAX - a) {
        fail(f, ORACLE_OVERFLOW, "compressed permutation is too large");
    }
    return a + b;
}

/* ------------------------------------------------------------- factoradic */

/* factoradic_bit_count, src/internal.hpp:173-183: bit width of size! - 1. */
uint32_t oracle_factoradic_bits(uint32_t size) {
    u128 factorial = 1;
    for (uint32_t i = 2; i <= size; ++i) {
        factorial *= i;
    }
    factorial -= 1;
    uint32_t bits = 0;
    while (factorial != 0) {
        ++bits;
        factorial >>= 1;
    }
    return bits;
}

/* encode_factoradic, src/internal.hpp:148-167.  Digit j counts the earlier
 * entries that are smaller than entry j; the rank is the mixed-radix number
 * with radices 1, 2, ..., size read by Horner's rule. */
static u128 factoradic_rank(const uint32_t* values, uint32_t size) {
    u128 rank = 0;
    for (uint32_t j = 0; j < size; ++j) {
        uint32_t digit = 0;
        for (uint32_t k = 0; k < j; ++k) {
            digit += values[k] < values[j];
        }
        rank = rank * (u128)(j + 1) + digit;
    }
    return rank;
}

/* decode_factoradic, src/internal.hpp:189-204. */
static void factoradic_unrank(u128 rank, uint32_t size, uint32_t* out) {
    uint32_t digits[32];
    for (uint32_t j = size; j-- > 0;) {
        digits[j] = (uint32_t)(rank % (j + 1));
        rank /= (j + 1);
    }
    /* Rebuild values from "number of smaller earlier entries": the last entry
     * takes the digit-th smallest of all values, and so on backwards. */
    uint8_t used[32] = {0};
    for (uint32_t j = size; j-- > 0;) {
        uint32_t want = digits[j];
        for (uint32_t v = 0; v < size; ++v) {
            if (used[v]) {
                continue;
            }
            if (want == 0) {
                out[j] = v;
                used[v] = 1;
                break;
            }
            --want;
        }
    }
}

/* ------------------------------------------------------------ size cache */

/* FormatSizeCache, src/internal.hpp:225-313.  Memoised recursive counts of
 * switch bits, middle bits and the switch bits in the top `depth` levels. */
#define SIZE_SLOTS 16384
typedef struct {
    uint64_t count;
    uint32_t depth; /* 0xffffffff = whole-subtree metrics */
    uint32_t used;
    uint64_t a, b;
} size_slot_t;

typedef struct {
    uint32_t leaf;
    failure_t* failure;
    size_slot_t* slots;
} sizes_t;

static size_slot_t* size_slot(sizes_t* s, uint64_t count, uint32_t depth) {
    uint64_t h = (count * 0x9E3779B97F4A7C15ULL) ^ ((uint64_t)depth * 0xC2B2AE3D27D4EB4FULL);
    for (uint32_t probe = 0; probe < SIZE_SLOTS; ++probe) {
        size_slot_t* slot = &s->slots[(h + probe) % SIZE_SLOTS];
        if (!slot->used || (slot->count == count && slot->depth == depth)) {
            return slot;
        }
    }
    fail(s->failure, ORACLE_LOGIC, "oracle size cache exhausted");
    return NULL;
}

static void subtree_metrics(sizes_t* s, uint64_t count, uint64_t* sw, uint64_t* mid) {
    if (count <= s->leaf) {
        *sw = 0;
        *mid = oracle_factoradic_bits((uint32_t)count);
        return;
    }
    size_slot_t* slot = size_slot(s, count, 0xffffffffu);
    if (slot->used) {
        *sw = slot->a;
        *mid = slot->b;
        return;
    }
    uint64_t lsw, lmid, rsw, rmid;
    subtree_metrics(s, count / 2 + count % 2, &lsw, &lmid);
    subtree_metrics(s, count / 2, &rsw, &rmid);
    slot = size_slot(s, count, 0xffffffffu);
    slot->count = count;
    slot->depth = 0xffffffffu;
    slot->a = add_checked(s->failure, count / 2, add_checked(s->failure, lsw, rsw));
    slot->b = add_checked(s->failure, lmid, rmid);
    slot->used = 1;
    *sw = slot->a;
    *mid = slot->b;
}

static uint64_t switch_bits(sizes_t* s, uint64_t count) {
    uint64_t sw, mid;
    subtree_metrics(s, count, &sw, &mid);
    return sw;
}

static uint64_t middle_bits(sizes_t* s, uint64_t count) {
    uint64_t sw, mid;
    subtree_metrics(s, count, &sw, &mid);
    return mid;
}

static uint64_t packet_switch_bits(sizes_t* s, uint64_t count, uint32_t depth) {
    if (count <= s->leaf || depth == 0) {
        return 0;
    }
    size_slot_t* slot = size_slot(s, count, depth);
    if (slot->used) {
        return slot->a;
    }
    uint64_t left = packet_switch_bits(s, count / 2 + count % 2, depth - 1);
    uint64_t right = packet_switch_bits(s, count / 2, depth - 1);
    slot = size_slot(s, count, depth);
    slot->count = count;
    slot->depth = depth;
    slot->a = add_checked(s->failure, count / 2, add_checked(s->failure, left, right));
    slot->used = 1;
    return slot->a;
}

static void sizes_init(sizes_t* s, uint8_t log2, failure_t* f) {
    s->leaf = 1u << log2;
    s->failure = f;
    s->slots = (size_slot_t*)calloc(SIZE_SLOTS, sizeof(size_slot_t));
    if (s->slots == NULL) {
        fail(f, ORACLE_RUNTIME, "oracle out of memory");
    }
}

static void sizes_free(sizes_t* s) {
    free(s->slots);
    s->slots = NULL;
}

/* ------------------------------------------------------------ format core */

/* routing_depth, src/internal.hpp:315-326 */
static uint32_t routing_depth(uint64_t count, uint8_t log2) {
    uint64_t leaf = 1ull << log2;
    uint32_t depth = 0;
    while (count > leaf) {
        count = count / 2 + count % 2;
        ++depth;
    }
    return depth;
}

/* default_clusters, src/internal.hpp:328-338 */
static uint8_t default_clusters(uint32_t depth, uint8_t* out) {
    if (depth == 0) {
        return 0;
    }
    if (depth == 1) {
        out[0] = 1;
        return 1;
    }
    out[0] = (uint8_t)((depth + 1) / 2);
    out[1] = (uint8_t)(depth / 2);
    return 2;
}

/* validate_clusters, src/internal.hpp:340-355 */
static void check_clusters(failure_t* f, const uint8_t* c, uint8_t n, uint32_t depth) {
    uint32_t sum = 0;
    for (uint8_t i = 0; i < n; ++i) {
        if (c[i] == 0) {
            fail(f, ORACLE_INVALID_ARGUMENT, "cluster depths must be positive");
        }
        sum += c[i];
    }
    if (sum != depth) {
        fail(f, ORACLE_INVALID_ARGUMENT, "cluster depths do not span every routing level");
    }
}

/* normalize_format, src/internal.hpp:357-383 */
static oracle_format normalize(failure_t* f, uint64_t count, const oracle_format* in) {
    oracle_format out = *in;
    if (out.middle_group_log2 == 0 || out.middle_group_log2 > 5) {
        fail(f, ORACLE_INVALID_ARGUMENT, "middle_group_log2 must be between 1 and 5");
    }
    if (out.middle_placement > 2) {
        fail(f, ORACLE_INVALID_ARGUMENT, "invalid middle placement");
    }
    if (out.input_cluster_count > 64 || out.output_cluster_count > 64) {
        fail(f, ORACLE_INVALID_ARGUMENT, "too many clusters");
    }
    uint32_t depth = routing_depth(count, out.middle_group_log2);
    if (out.input_cluster_count == 0) {
        out.input_cluster_count = default_clusters(depth, out.input_clusters);
    }
    if (out.output_cluster_count == 0) {
        out.output_cluster_count = default_clusters(depth, out.output_clusters);
    }
    check_clusters(f, out.input_clusters, out.input_cluster_count, depth);
    check_clusters(f, out.output_clusters, out.output_cluster_count, depth);
    if (depth == 0) {
        out.middle_placement = 0;
    }
    return out;
}

static uint64_t bytes_for(uint64_t bits) {
    return bits / 8 + (bits % 8 != 0);
}

/* make_layout, src/internal.hpp:389-429 */
static oracle_layout layout_of(failure_t* f, uint64_t count, const oracle_format* format) {
    oracle_layout L;
    memset(&L, 0, sizeof L);
    L.format = normalize(f, count, format);
    sizes_t s;
    sizes_init(&s, L.format.middle_group_log2, f);
    /* The cache is freed before any failure can escape below only when the
     * arithmetic succeeds; a failure longjmps out and leaks one small table,
     * which is acceptable for a test oracle. */
    L.switch_bits = switch_bits(&s, count);
    L.middle_bits = middle_bits(&s, count);
    sizes_free(&s);
    uint64_t header = add_checked(f, 20,
        (uint64_t)L.format.input_cluster_count + L.format.output_cluster_count);
    int in_embeds = L.format.middle_placement == 1;
    int out_embeds = L.format.middle_placement == 2;
    uint64_t in_bytes = add_checked(f, bytes_for(L.switch_bits),
        in_embeds ? bytes_for(L.middle_bits) : 0);
    uint64_t out_bytes = add_checked(f, bytes_for(L.switch_bits),
        out_embeds ? bytes_for(L.middle_bits) : 0);
    uint64_t mid_bytes = L.format.middle_placement == 0 ? bytes_for(L.middle_bits) : 0;
    if (count > (1ull << 63)) {
        fail(f, ORACLE_OVERFLOW, "logical network size is too large");
    }
    uint64_t width = 1ull << L.format.middle_group_log2;
    if (count > width) {
        width = 1;
        while (width < count) {
            width <<= 1;
        }
    }
    L.size = count;
    L.network_size = width;
    L.input_offset = header;
    L.output_offset = add_checked(f, header, in_bytes);
    L.middle_offset = add_checked(f, L.output_offset, out_bytes);
    L.end_offset = add_checked(f, L.middle_offset, mid_bytes);
    return L;
}

int oracle_make_layout(uint64_t count, const oracle_format* format,
    oracle_layout* layout, char* err, size_t err_len) {
    failure_t f;
    if (setjmp(f.jump)) {
        copy_error(&f, err, err_len);
        return f.code;
    }
    *layout = layout_of(&f, count, format);
    return ORACLE_OK;
}

/* write_header, src/internal.hpp:431-454 */
static void write_header(uint8_t* out, const oracle_layout* L) {
    static const uint8_t magic[8] = {'B', 'E', 'N', 'E', 'S', '0', '1', 0};
    memcpy(out, magic, 8);
    for (int i = 0; i < 8; ++i) {
        out[8 + i] = (uint8_t)(L->size >> (8 * i));
    }
    out[16] = L->format.middle_placement;
    out[17] = L->format.middle_group_log2;
    out[18] = L->format.input_cluster_count;
    out[19] = L->format.output_cluster_count;
    memcpy(out + 20, L->format.input_clusters, L->format.input_cluster_count);
    memcpy(out + 20 + L->format.input_cluster_count, L->format.output_clusters,
        L->format.output_cluster_count);
}

/* ------------------------------------------------------ section addresses */

/* How many of the first `paths` nodes at `level` levels below a root whose
 * count leaves remainder `large` modulo 2^level are one entry larger than
 * the rest.  A node is large when the bit-reversal of its path is below
 * `large`; split by the first turn and recurse (left turns keep the even
 * reversed paths, right turns the odd ones). */
static uint64_t large_before(uint64_t paths, uint32_t level, uint64_t large) {
    uint64_t total = 0;
    while (paths > 0 && large > 0) {
        if (level == 0) {
            total += 1; /* the single remaining node is a large one */
            break;
        }
        uint64_t half = 1ull << (level - 1);
        uint64_t left_large = (large + 1) / 2;
        if (paths <= half) {
            large = left_large;
        } else {
            total += left_large < half ? left_large : half;
            paths -= half;
            large = large / 2;
        }
        --level;
    }
    return total;
}

/* SectionAddress, src/internal.hpp:475-718 */
typedef struct {
    const uint8_t* clusters;
    int embeds;
    sizes_t* sizes;
    uint32_t cluster_index;
    uint32_t group_depth;
    uint32_t relative_level;
    uint64_t path;
    uint64_t root_count;
    uint64_t node_count;
    uint64_t packet_base;
    uint64_t residual_before;
    uint64_t group_bits;
    uint64_t full_packet_bits;
    uint64_t pair_span;
    uint64_t full_prefix;
    uint64_t tail_packet;
    uint64_t tail_prefix;
} section_t;

static uint64_t section_bits(const section_t* a, uint64_t count) {
    return switch_bits(a->sizes, count) + (a->embeds ? middle_bits(a->sizes, count) : 0);
}

/* Bits that the first `paths` nodes at `level` put into packet `packet`
 * (packet_path_prefix_bits, src/internal.hpp:611-649). */
static uint64_t packet_path_bits(const section_t* a, uint64_t packet, uint32_t level, uint64_t paths) {
    uint64_t nodes = 1ull << level;
    uint64_t small = a->root_count / nodes;
    uint64_t large = a->root_count % nodes;
    uint64_t span = 1ull << (a->group_depth - level - 1);
    uint64_t first = packet * span;
    uint64_t share[2];
    for (int big = 0; big < 2; ++big) {
        uint64_t count = small + (uint64_t)big;
        uint64_t pairs = count / 2;
        if (count <= a->sizes->leaf || first >= pairs) {
            share[big] = 0;
        } else {
            share[big] = pairs - first < span ? pairs - first : span;
        }
    }
    uint64_t big_paths = large_before(paths, level, large);
    return big_paths * share[1] + (paths - big_paths) * share[0];
}

static uint64_t packet_prefix(const section_t* a, uint64_t packet) {
    uint64_t bits = 0;
    for (uint32_t level = 0; level < a->relative_level; ++level) {
        bits += packet_path_bits(a, packet, level, 1ull << level);
    }
    return bits + packet_path_bits(a, packet, a->relative_level, a->path);
}

static void refresh_group(section_t* a) {
    a->group_bits = packet_switch_bits(a->sizes, a->root_count, a->group_depth);
    uint64_t bits = 0;
    for (uint32_t level = 0; level < a->group_depth; ++level) {
        bits += packet_path_bits(a, 0, level, 1ull << level);
    }
    a->full_packet_bits = bits;
}

static void refresh_node(section_t* a) {
    a->pair_span = 1ull << (a->group_depth - a->relative_level - 1);
    a->full_prefix = packet_prefix(a, 0);
    uint64_t pairs = a->node_count / 2;
    a->tail_packet = pairs == 0 ? 0 : (pairs - 1) / a->pair_span;
    a->tail_prefix = packet_prefix(a, a->tail_packet);
}

static section_t section_root(uint64_t count, const uint8_t* clusters, int embeds, sizes_t* sizes) {
    section_t a;
    memset(&a, 0, sizeof a);
    a.clusters = clusters;
    a.embeds = embeds;
    a.sizes = sizes;
    a.root_count = count;
    a.node_count = count;
    if (count > sizes->leaf) {
        a.group_depth = clusters[0];
        refresh_group(&a);
        refresh_node(&a);
    }
    return a;
}

static uint64_t section_switch_bit(const section_t* a, uint64_t pair) {
    uint64_t packet = pair / a->pair_span;
    return a->packet_base + packet * a->full_packet_bits +
        (packet == a->tail_packet ? a->tail_prefix : a->full_prefix) +
        pair % a->pair_span;
}

static uint64_t section_middle_bit(const section_t* a) {
    if (a->root_count <= a->sizes->leaf) {
        return a->packet_base;
    }
    return a->packet_base + a->group_bits + a->residual_before;
}

static section_t section_child(const section_t* a, int right, uint64_t count) {
    section_t c = *a;
    uint64_t left_count = count / 2 + count % 2;
    uint64_t child_count = right ? count / 2 : left_count;
    uint32_t remaining = a->group_depth - a->relative_level;
    if (remaining > 1) {
        if (right) {
            c.residual_before += section_bits(a, left_count) -
                packet_switch_bits(a->sizes, left_count, remaining - 1);
        }
        c.relative_level += 1;
        c.path = a->path * 2 + (uint64_t)right;
        c.node_count = child_count;
        refresh_node(&c);
        return c;
    }
    uint64_t before = a->residual_before + (right ? section_bits(a, left_count) : 0);
    c.packet_base = a->packet_base + a->group_bits + before;
    c.residual_before = 0;
    c.root_count = child_count;
    c.node_count = child_count;
    c.relative_level = 0;
    c.path = 0;
    if (child_count > a->sizes->leaf) {
        c.cluster_index += 1;
        c.group_depth = a->clusters[c.cluster_index];
        refresh_group(&c);
        refresh_node(&c);
    } else {
        c.group_depth = 0;
        c.group_bits = 0;
        c.full_packet_bits = 0;
        c.pair_span = 0;
        c.full_prefix = 0;
        c.tail_packet = 0;
        c.tail_prefix = 0;
    }
    return c;
}

/* ---------------------------------------------------------------- encoder */

typedef struct {
    uint8_t* blob;
    const oracle_layout* layout;
    sizes_t* sizes;
    failure_t* failure;
} encoder_t;

static void set_bit(uint8_t* blob, uint64_t section, uint64_t bit) {
    blob[section + bit / 8] |= (uint8_t)(1u << (bit & 7));
}

static void* must_alloc(failure_t* f, size_t count, size_t size) {
    void* p = calloc(count ? count : 1, size);
    if (p == NULL) {
        fail(f, ORACLE_RUNTIME, "oracle out of memory");
    }
    return p;
}

/* encode_compact_node, src/benes.cpp:189-351 (threads = 1). */
static void encode_node(encoder_t* E, const uint32_t* perm, uint64_t count,
    section_t in, section_t out, uint64_t middle_offset) {
    const oracle_layout* L = E->layout;
    if (count <= E->sizes->leaf) {
        /* leaf: exact factoradic rank, src/benes.cpp:201-225 */
        u128 rank = factoradic_rank(perm, (uint32_t)count);
        uint64_t section = L->middle_offset;
        uint64_t bit0 = middle_offset;
        if (L->format.middle_placement == 1) {
            section = L->input_offset;
            bit0 = section_middle_bit(&in);
        } else if (L->format.middle_placement == 2) {
            section = L->output_offset;
            bit0 = section_middle_bit(&out);
        }
        uint32_t nbits = oracle_factoradic_bits((uint32_t)count);
        for (uint32_t b = 0; b < nbits; ++b) {
            if ((rank >> b) & 1) {
                set_bit(E->blob, section, bit0 + b);
            }
        }
        return;
    }

    uint64_t pairs = count / 2;
    uint64_t left_count = count - pairs;
    uint32_t* left = (uint32_t*)must_alloc(E->failure, left_count, 4);
    uint32_t* right = (uint32_t*)must_alloc(E->failure, pairs, 4);
    {
        /* inverse and the degree-2 constraint graph, src/benes.cpp:232-252 */
        uint32_t* inv = (uint32_t*)must_alloc(E->failure, count, 4);
        for (uint64_t i = 0; i < count; ++i) {
            inv[perm[i]] = (uint32_t)i;
        }
        uint32_t* nbr = (uint32_t*)must_alloc(E->failure, count * 2, 4);
        uint8_t* deg = (uint8_t*)must_alloc(E->failure, count, 1);
#define LINK(a, b)                        \
    do {                                  \
        nbr[2 * (a) + deg[a]++] = (b);    \
        nbr[2 * (b) + deg[b]++] = (a);    \
    } while (0)
        for (uint64_t k = 0; k < pairs; ++k) {
            LINK((uint32_t)(2 * k), (uint32_t)(2 * k + 1));
            LINK(inv[2 * k], inv[2 * k + 1]);
        }
#undef LINK
        /* canonical BFS 2-colouring, src/benes.cpp:253-297: the odd tail and
         * its output partner get colour 0 first, then every other component
         * gives colour 0 to its smallest vertex. */
        int8_t* color = (int8_t*)must_alloc(E->failure, count, 1);
        memset(color, -1, count);
        uint32_t* queue = (uint32_t*)must_alloc(E->failure, count, 4);
        uint64_t seeds[2];
        int nseeds = 0;
        if (count % 2 == 1) {
            seeds[nseeds++] = count - 1;
            seeds[nseeds++] = inv[count - 1];
        }
        for (uint64_t scan = 0; scan < count + (uint64_t)nseeds; ++scan) {
            uint64_t start = scan < (uint64_t)nseeds ? seeds[scan] : scan - (uint64_t)nseeds;
            if (color[start] >= 0) {
                if (scan < (uint64_t)nseeds && color[start] != 0) {
                    fail(E->failure, ORACLE_LOGIC, "compact odd endpoints have incompatible colors");
                }
                continue;
            }
            color[start] = 0;
            uint64_t head = 0, tail = 0;
            queue[tail++] = (uint32_t)start;
            while (head < tail) {
                uint32_t v = queue[head++];
                for (uint8_t e = 0; e < deg[v]; ++e) {
                    uint32_t w = nbr[2 * v + e];
                    int8_t want = (int8_t)(color[v] ^ 1);
                    if (color[w] < 0) {
                        color[w] = want;
                        queue[tail++] = w;
                    } else if (color[w] != want) {
                        fail(E->failure, ORACLE_LOGIC, "compact network coloring failed");
                    }
                }
            }
        }
        /* switch bits and child permutations, src/benes.cpp:298-315 */
        for (uint64_t i = 0; i < count; ++i) {
            int branch = color[i] != 0;
            if (i != count - 1 || count % 2 == 0) {
                if (branch != (int)(i & 1)) {
                    set_bit(E->blob, L->input_offset, section_switch_bit(&in, i / 2));
                }
            }
            uint64_t o = perm[i];
            if (o != count - 1 || count % 2 == 0) {
                if (branch != (int)(o & 1)) {
                    set_bit(E->blob, L->output_offset, section_switch_bit(&out, o / 2));
                }
            }
            (branch ? right : left)[i / 2] = (uint32_t)(o / 2);
        }
        free(queue);
        free(color);
        free(deg);
        free(nbr);
        free(inv);
    }
    uint64_t right_middle = middle_offset + middle_bits(E->sizes, left_count);
    section_t lin = section_child(&in, 0, count), lout = section_child(&out, 0, count);
    section_t rin = section_child(&in, 1, count), rout = section_child(&out, 1, count);
    encode_node(E, left, left_count, lin, lout, middle_offset);
    free(left);
    encode_node(E, right, pairs, rin, rout, right_middle);
    free(right);
}

int oracle_compress(const void* permutation, uint64_t count,
    uint32_t entry_bytes, const oracle_format* format,
    uint8_t* blob, uint64_t blob_capacity, uint64_t* blob_len,
    char* err, size_t err_len) {
    failure_t f;
    sizes_t sizes = {0, NULL, NULL};
    uint32_t* root = NULL;
    if (setjmp(f.jump)) {
        sizes_free(&sizes);
        free(root);
        copy_error(&f, err, err_len);
        return f.code;
    }
    if (entry_bytes != 4 && entry_bytes != 8) {
        fail(&f, ORACLE_INVALID_ARGUMENT, "entry width must be 4 or 8 bytes");
    }
    /* validate_permutation, src/benes.cpp:152-173 */
    if (count == 0) {
        fail(&f, ORACLE_INVALID_ARGUMENT, "permutation size is out of range");
    }
    if (entry_bytes == 4 && count > 0xffffffffull) {
        fail(&f, ORACLE_INVALID_ARGUMENT, "permutation size requires 64-bit source values");
    }
    if (count > 0xffffffffull) {
        fail(&f, ORACLE_LENGTH, "oracle handles fewer than 2^32 entries");
    }
    oracle_layout L = layout_of(&f, count, format);
    if (blob_capacity < L.end_offset) {
        fail(&f, ORACLE_LENGTH, "blob buffer is too small");
    }
    root = (uint32_t*)must_alloc(&f, count, 4);
    {
        uint8_t* seen = (uint8_t*)must_alloc(&f, count, 1);
        for (uint64_t i = 0; i < count; ++i) {
            uint64_t v = entry_bytes == 4 ? ((const uint32_t*)permutation)[i]
                                          : ((const uint64_t*)permutation)[i];
            if (v >= count || seen[v]) {
                free(seen);
                fail(&f, ORACLE_INVALID_ARGUMENT,
                    "input must contain every value from zero through size minus one");
            }
            seen[v] = 1;
            root[i] = (uint32_t)v;
        }
        free(seen);
    }
    memset(blob, 0, L.end_offset);
    write_header(blob, &L);
    sizes_init(&sizes, L.format.middle_group_log2, &f);
    section_t in = section_root(count, L.format.input_clusters, L.format.middle_placement == 1, &sizes);
    section_t out = section_root(count, L.format.output_clusters, L.format.middle_placement == 2, &sizes);
    encoder_t E = {blob, &L, &sizes, &f};
    encode_node(&E, root, count, in, out, 0);
    sizes_free(&sizes);
    free(root);
    *blob_len = L.end_offset;
    return ORACLE_OK;
}

/* ------------------------------------------------------------ probes */

static int walk_to(failure_t* f, uint64_t count, const oracle_format* format,
    int depth, const uint8_t* turns, oracle_layout* L, sizes_t* s,
    section_t* in, section_t* out, uint64_t* node_count, uint64_t* middle) {
    *L = layout_of(f, count, format);
    sizes_init(s, L->format.middle_group_log2, f);
    *in = section_root(count, L->format.input_clusters, L->format.middle_placement == 1, s);
    *out = section_root(count, L->format.output_clusters, L->format.middle_placement == 2, s);
    *middle = 0;
    for (int d = 0; d < depth; ++d) {
        if (count <= s->leaf) {
            fail(f, ORACLE_INVALID_ARGUMENT, "path descends below a leaf");
        }
        uint64_t left_count = count / 2 + count % 2;
        if (turns[d]) {
            *middle += middle_bits(s, left_count);
        }
        *in = section_child(in, turns[d], count);
        *out = section_child(out, turns[d], count);
        count = turns[d] ? count / 2 : left_count;
    }
    *node_count = count;
    return 0;
}

int oracle_switch_bit(uint64_t count, const oracle_format* format, int side,
    int depth, const uint8_t* turns, uint64_t pair, uint64_t* bit) {
    failure_t f;
    sizes_t s = {0, NULL, NULL};
    if (setjmp(f.jump)) {
        sizes_free(&s);
        return f.code;
    }
    oracle_layout L;
    section_t in, out;
    uint64_t n, middle;
    walk_to(&f, count, format, depth, turns, &L, &s, &in, &out, &n, &middle);
    if (n <= s.leaf || pair >= n / 2) {
        fail(&f, ORACLE_INVALID_ARGUMENT, "no such switch");
    }
    *bit = section_switch_bit(side ? &out : &in, pair);
    sizes_free(&s);
    return ORACLE_OK;
}

int oracle_middle_bit(uint64_t count, const oracle_format* format,
    int depth, const uint8_t* turns, uint64_t* bit) {
    failure_t f;
    sizes_t s = {0, NULL, NULL};
    if (setjmp(f.jump)) {
        sizes_free(&s);
        return f.code;
    }
    oracle_layout L;
    section_t in, out;
    uint64_t n, middle;
    walk_to(&f, count, format, depth, turns, &L, &s, &in, &out, &n, &middle);
    if (n > s.leaf) {
        fail(&f, ORACLE_INVALID_ARGUMENT, "not a leaf");
    }
    if (L.format.middle_placement == 1) {
        *bit = section_middle_bit(&in);
    } else if (L.format.middle_placement == 2) {
        *bit = section_middle_bit(&out);
    } else {
        *bit = middle;
    }
    sizes_free(&s);
    return ORACLE_OK;
}

/* ------------------------------------------------------ parse and lookup */

static int get_bit(const uint8_t* blob, uint64_t section, uint64_t bit) {
    return (blob[section + bit / 8] >> (bit & 7)) & 1;
}

/* parse_header + validate_padding, src/benes.cpp:26-117 */
static oracle_layout parse(failure_t* f, const uint8_t* blob, uint64_t len) {
    static const uint8_t magic[8] = {'B', 'E', 'N', 'E', 'S', '0', '1', 0};
    if (len < 20) {
        fail(f, ORACLE_INVALID_ARGUMENT, "compressed permutation header is truncated");
    }
    if (memcmp(blob, magic, 8) != 0) {
        fail(f, ORACLE_INVALID_ARGUMENT, "compressed permutation has invalid magic");
    }
    uint64_t size = 0;
    for (int i = 0; i < 8; ++i) {
        size |= (uint64_t)blob[8 + i] << (8 * i);
    }
    oracle_format fmt;
    memset(&fmt, 0, sizeof fmt);
    fmt.middle_placement = blob[16];
    fmt.middle_group_log2 = blob[17];
    fmt.input_cluster_count = blob[18];
    fmt.output_cluster_count = blob[19];
    uint64_t header = 20ull + fmt.input_cluster_count + fmt.output_cluster_count;
    if (header > 84 || header > len) {
        fail(f, ORACLE_INVALID_ARGUMENT, "unsupported compressed permutation header size");
    }
    if (fmt.middle_placement > 2) {
        fail(f, ORACLE_INVALID_ARGUMENT, "compressed permutation has invalid format parameters");
    }
    memcpy(fmt.input_clusters, blob + 20, fmt.input_cluster_count);
    memcpy(fmt.output_clusters, blob + 20 + fmt.input_cluster_count, fmt.output_cluster_count);
    if (size == 0) {
        fail(f, ORACLE_INVALID_ARGUMENT, "compressed permutation has invalid dimensions");
    }
    oracle_layout L = layout_of(f, size, &fmt);
    if (L.end_offset != len) {
        fail(f, ORACLE_INVALID_ARGUMENT, "compressed permutation has invalid section bounds");
    }
    uint64_t begins[3] = {L.input_offset, L.output_offset, L.middle_offset};
    uint64_t ends[3] = {L.output_offset, L.middle_offset, L.end_offset};
    uint64_t used[3] = {
        L.switch_bits + (L.format.middle_placement == 1 ? L.middle_bits : 0),
        L.switch_bits + (L.format.middle_placement == 2 ? L.middle_bits : 0),
        L.format.middle_placement == 0 ? L.middle_bits : 0};
    for (int k = 0; k < 3; ++k) {
        uint64_t section_bytes = ends[k] - begins[k];
        uint64_t used_bytes = used[k] / 8;
        if (used_bytes > section_bytes || (used_bytes == section_bytes && used[k] % 8 != 0)) {
            fail(f, ORACLE_INVALID_ARGUMENT, "compressed permutation section is too small");
        }
        uint64_t padding = (section_bytes - used_bytes) * 8 - used[k] % 8;
        for (uint64_t b = 0; b < padding; ++b) {
            if (get_bit(blob, begins[k], used[k] + b)) {
                fail(f, ORACLE_INVALID_ARGUMENT, "compressed permutation has nonzero section padding bits");
            }
        }
    }
    return L;
}

int oracle_validate(const uint8_t* blob, uint64_t blob_len, char* err, size_t err_len) {
    failure_t f;
    if (setjmp(f.jump)) {
        copy_error(&f, err, err_len);
        return f.code;
    }
    (void)parse(&f, blob, blob_len);
    return ORACLE_OK;
}

/* lookup, src/internal.hpp:1035-1124 */
int oracle_lookup(const uint8_t* blob, uint64_t blob_len, uint64_t value,
    int inverse, uint64_t* result, char* err, size_t err_len) {
    failure_t f;
    sizes_t s = {0, NULL, NULL};
    if (setjmp(f.jump)) {
        sizes_free(&s);
        copy_error(&f, err, err_len);
        return f.code;
    }
    oracle_layout L = parse(&f, blob, blob_len);
    if (value >= L.size) {
        fail(&f, ORACLE_RUNTIME, "permutation lookup is out of range");
    }
    sizes_init(&s, L.format.middle_group_log2, &f);
    struct frame {
        uint64_t size;
        section_t in, out;
        int right;
    } frames[64];
    int depth = 0;
    uint64_t count = L.size, index = value, middle = 0;
    section_t in = section_root(count, L.format.input_clusters, L.format.middle_placement == 1, &s);
    section_t out = section_root(count, L.format.output_clusters, L.format.middle_placement == 2, &s);
    while (count > s.leaf) {
        int odd_tail = count % 2 == 1 && index == count - 1;
        int right = 0;
        if (!odd_tail) {
            uint64_t bit = section_switch_bit(inverse ? &out : &in, index / 2);
            uint64_t section = inverse ? L.output_offset : L.input_offset;
            right = get_bit(blob, section, bit) != (int)(index & 1);
        }
        frames[depth].size = count;
        frames[depth].in = in;
        frames[depth].out = out;
        frames[depth].right = right;
        ++depth;
        uint64_t left_count = count / 2 + count % 2;
        if (right) {
            middle += middle_bits(&s, left_count);
        }
        in = section_child(&in, right, count);
        out = section_child(&out, right, count);
        index /= 2;
        count = right ? count / 2 : left_count;
    }
    uint64_t section = L.middle_offset, bit0 = middle;
    if (L.format.middle_placement == 1) {
        section = L.input_offset;
        bit0 = section_middle_bit(&in);
    } else if (L.format.middle_placement == 2) {
        section = L.output_offset;
        bit0 = section_middle_bit(&out);
    }
    uint32_t nbits = oracle_factoradic_bits((uint32_t)count);
    u128 rank = 0;
    for (uint32_t b = 0; b < nbits; ++b) {
        if (get_bit(blob, section, bit0 + b)) {
            rank |= (u128)1 << b;
        }
    }
    uint32_t leaf[32];
    factoradic_unrank(rank, (uint32_t)count, leaf);
    if (!inverse) {
        index = leaf[index];
    } else {
        uint64_t found = count;
        for (uint64_t i = 0; i < count; ++i) {
            if (leaf[i] == index) {
                found = i;
                break;
            }
        }
        if (found == count) {
            fail(&f, ORACLE_RUNTIME, "invalid compact factorial code");
        }
        index = found;
    }
    while (depth != 0) {
        const struct frame* fr = &frames[--depth];
        uint64_t pairs = fr->size / 2;
        if (!fr->right && fr->size % 2 == 1 && index == pairs) {
            index = fr->size - 1;
            continue;
        }
        uint64_t section2 = inverse ? L.input_offset : L.output_offset;
        uint64_t bit = section_switch_bit(inverse ? &fr->in : &fr->out, index);
        index = index * 2 + (uint64_t)(fr->right ^ get_bit(blob, section2, bit));
    }
    sizes_free(&s);
    *result = index;
    return ORACLE_OK;
}

/* --------------------------------------------------------- workload inputs
 *
 * The configs' seeded permutations, restated here so that the CPU baseline
 * and the fixture generators need nothing from the B200 library.  Not part
 * of the reference (its tests shuffle with std::shuffle,
 * tests/test_benes.cpp:60-68); the configs name the published generators:
 * xoshiro256** (Blackman and Vigna, 2018) whose four state words are
 * successive splitmix64 outputs from the seed, bounded draws in [0, range)
 * by Lemire's multiply-shift with rejection (2019), and shuffles from the
 * top index down: Fisher-Yates draws j in [0, i], Sattolo j in [0, i - 1]
 * (one n-cycle).  Kinds: 0 Fisher-Yates, 1 Sattolo, 2 identity, 3 reverse,
 * 4 bit reversal (power-of-two counts only). */

typedef struct {
    uint64_t s[4];
} xoshiro_t;

static uint64_t splitmix_next(uint64_t* x) {
    uint64_t z = (*x += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

static uint64_t rotate_left(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static uint64_t xoshiro_next(xoshiro_t* g) {
    uint64_t* s = g->s;
    const uint64_t result = rotate_left(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotate_left(s[3], 45);
    return result;
}

static uint64_t xoshiro_below(xoshiro_t* g, uint64_t range) {
    u128 m = (u128)xoshiro_next(g) * range;
    if ((uint64_t)m < range) {
        const uint64_t threshold = (0 - range) % range;
        while ((uint64_t)m < threshold) {
            m = (u128)xoshiro_next(g) * range;
        }
    }
    return (uint64_t)(m >> 64);
}

#define ORACLE_SHUFFLE(T)                                                          \
    static void shuffle_##T(T* a, uint64_t n, uint64_t seed, int cycle) {          \
        for (uint64_t i = 0; i < n; ++i) a[i] = (T)i;                              \
        if (n < 2) return;                                                         \
        xoshiro_t g;                                                               \
        uint64_t x = seed;                                                         \
        for (int k = 0; k < 4; ++k) g.s[k] = splitmix_next(&x);                    \
        /* draws do not depend on the array: draw a block ahead and prefetch */  \
        uint64_t draw[32];                                                         \
        for (uint64_t top = n - 1; top >= 1;) {                                    \
            const uint64_t steps = top < 32 ? top : 32;                            \
            for (uint64_t t = 0; t < steps; ++t) {                                 \
                draw[t] = xoshiro_below(&g, cycle ? top - t : top - t + 1);        \
                __builtin_prefetch(a + draw[t], 1, 0);                             \
            }                                                                      \
            for (uint64_t t = 0; t < steps; ++t) {                                 \
                const T keep = a[top - t];                                         \
                a[top - t] = a[draw[t]];                                           \
                a[draw[t]] = keep;                                                 \
            }                                                                      \
            top -= steps;                                                          \
        }                                                                          \
    }
ORACLE_SHUFFLE(uint32_t)
ORACLE_SHUFFLE(uint64_t)

int oracle_fill_permutation(uint32_t kind, uint64_t seed, uint64_t count,
    uint32_t entry_bytes, void* out) {
    if (entry_bytes != 4 && entry_bytes != 8) return ORACLE_INVALID_ARGUMENT;
    if (entry_bytes == 4 && count > 0x100000000ull) return ORACLE_INVALID_ARGUMENT;
    if (kind == 4 && (count == 0 || (count & (count - 1)) != 0)) return ORACLE_INVALID_ARGUMENT;
    if (kind > 4) return ORACLE_INVALID_ARGUMENT;
    uint32_t* a32 = (uint32_t*)out;
    uint64_t* a64 = (uint64_t*)out;
    if (kind <= 1) {
        if (entry_bytes == 4) {
            shuffle_uint32_t(a32, count, seed, (int)kind);
        } else {
            shuffle_uint64_t(a64, count, seed, (int)kind);
        }
        return ORACLE_OK;
    }
    uint32_t bits = 0;
    while (kind == 4 && (1ull << bits) < count) ++bits;
    for (uint64_t i = 0; i < count; ++i) {
        uint64_t v = i;
        if (kind == 3) {
            v = count - 1 - i;
        } else if (kind == 4) {
            v = 0;
            for (uint32_t b = 0; b < bits; ++b) v |= ((i >> b) & 1ull) << (bits - 1 - b);
        }
        if (entry_bytes == 4) a32[i] = (uint32_t)v; else a64[i] = v;
    }
    return ORACLE_OK;
}
