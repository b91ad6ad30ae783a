// SPDX-License-Identifier: Apache-2.0
//
// Driver for the reference-side integration shim.  TEST INFRASTRUCTURE ONLY.
//
// Compiled (by oracle.oracle.build_shim) together with the backend unit and
// declarations of the integration notes, against the reference's own
// headers and library (oracle/_ref) and libbenes_b200.so.  For each case it
// runs the shim and the reference's portable_cpu path (benes::compress /
// benes::compress_file, src/benes.cpp:422-553) on the same arguments and
// prints one line: case, the shim's outcome, the reference's outcome
// (exception type and message, or "ok"), plus "<case>_bytes same|different"
// when both produced a blob.
#include "b200_decls.hpp"
#include "internal.hpp"
#include <benes_b200.h>

#include <cstdio>
#include <fstream>
#include <functional>
#include <numeric>
#include <string>
#include <typeinfo>
#include <vector>

using namespace benes;

// The enumerator the integration notes append to Backend (its value after
// the reference's five); the reference headers here lack it.
constexpr Backend kB200 = static_cast<Backend>(5);

// The dispatch fragment of the integration notes (section 3), as written
// there, in a function of the shape of benes::compress: the b200 branch,
// then every other backend through the reference's own compress.
template <typename Value>
std::vector<std::byte> dispatch(std::span<const Value> permutation, const CompressOptions& options) {
    const Backend backend = options.backend;
#include "dispatch_fragment.inc"
    return compress(permutation, options);
}

static std::string outcome(const std::function<void()>& fn) {
    try {
        fn();
        return "ok|";
    } catch (const std::out_of_range& e) {
        return std::string("out_of_range|") + e.what();
    } catch (const std::invalid_argument& e) {
        return std::string("invalid_argument|") + e.what();
    } catch (const std::length_error& e) {
        return std::string("length_error|") + e.what();
    } catch (const std::overflow_error& e) {
        return std::string("overflow_error|") + e.what();
    } catch (const std::runtime_error& e) {
        return std::string("runtime_error|") + e.what();
    } catch (const std::exception& e) {
        return std::string("exception|") + e.what();
    }
}

static void report(const char* name, const std::string& shim, const std::string& ref) {
    std::printf("%s\t%s\t%s\n", name, shim.c_str(), ref.c_str());
}

static FormatOptions fmt(std::uint8_t m, std::vector<std::uint8_t> in = {},
    std::vector<std::uint8_t> out = {}, MiddlePlacement pl = MiddlePlacement::separate) {
    FormatOptions f;
    f.middle_group_log2 = m;
    f.input_clusters = std::move(in);
    f.output_clusters = std::move(out);
    f.middle_placement = pl;
    return f;
}

template <typename V>
static void compare(const char* name, const std::vector<V>& p, const FormatOptions& f) {
    std::vector<std::byte> a, b;
    const std::string shim = outcome([&] { a = detail::compress_compact_b200(std::span<const V>(p), f); });
    CompressOptions o;
    o.backend = Backend::portable_cpu;
    o.threads = 1;
    o.format = f;
    const std::string ref = outcome([&] { b = compress(std::span<const V>(p), o); });
    report(name, shim, ref);
    if (shim == "ok|" && ref == "ok|") {
        std::printf("%s_bytes\t%s\t%s\n", name, a == b ? "same" : "different", "same");
    }
}

int main(int argc, char** argv) {
    const std::string dir = argc > 1 ? argv[1] : ".";
    std::printf("available\t%d\n", detail::b200_available() ? 1 : 0);
    std::vector<std::uint32_t> p(1000);
    std::iota(p.begin(), p.end(), 0u);
    for (std::size_t i = p.size() - 1; i > 0; --i) std::swap(p[i], p[(i * 7919u) % (i + 1)]);
    std::vector<std::uint64_t> p64(p.begin(), p.end());

    compare("valid_u32", p, fmt(5));
    compare("valid_u64_embedded", p64, fmt(4, {}, {}, MiddlePlacement::embedded_output));
    {
        // 2^20 uint64 entries, default clusters, embedded_output
        std::vector<std::uint64_t> big(1u << 20);
        std::iota(big.begin(), big.end(), std::uint64_t{0});
        std::uint64_t x = 0x2545F4914F6CDD1Dull;
        for (std::size_t i = big.size() - 1; i > 0; --i) {
            x ^= x << 13; x ^= x >> 7; x ^= x << 17;
            std::swap(big[i], big[x % (i + 1)]);
        }
        compare("valid_u64_2p20", big, fmt(5, {}, {}, MiddlePlacement::embedded_output));
        // the dispatch branch of the integration notes, section 3
        std::vector<std::byte> a, b;
        CompressOptions d;
        d.backend = kB200;
        d.format = fmt(5, {}, {}, MiddlePlacement::embedded_output);
        const std::string shim = outcome([&] { a = dispatch(std::span<const std::uint64_t>(big), d); });
        CompressOptions o;
        o.backend = Backend::portable_cpu;
        o.format = d.format;
        const std::string ref = outcome([&] { b = compress(std::span<const std::uint64_t>(big), o); });
        report("dispatch_u64_2p20", shim, ref);
        if (shim == "ok|" && ref == "ok|") {
            std::printf("dispatch_u64_2p20_bytes\t%s\t%s\n", a == b ? "same" : "different", "same");
        }
    }
    compare("group_log2_zero", p, fmt(0));
    compare("group_log2_six", p, fmt(6));
    compare("clusters_short", p, fmt(5, {1, 1}));
    compare("clusters_long", p64, fmt(5, {}, {9, 9}));
    compare("bad_placement", p, fmt(5, {}, {}, static_cast<MiddlePlacement>(3)));
    compare("empty", std::vector<std::uint32_t>{}, fmt(5));

    // compress_file: argument and file errors come before any device work
    const std::string missing = dir + "/missing.bin";
    const std::string odd = dir + "/odd.bin";
    {
        std::ofstream f(odd, std::ios::binary);
        f.write("abcde", 5);
    }
    CompressOptions o;
    o.backend = Backend::portable_cpu;
    report("file_missing",
        outcome([&] { detail::compress_file_b200(missing, dir + "/a.out", InputValueWidth::bits32, fmt(5)); }),
        outcome([&] { compress_file(missing, dir + "/b.out", InputValueWidth::bits32, o); }));
    report("file_ragged",
        outcome([&] { detail::compress_file_b200(odd, dir + "/a.out", InputValueWidth::bits32, fmt(5)); }),
        outcome([&] { compress_file(odd, dir + "/b.out", InputValueWidth::bits32, o); }));
    report("file_directory",
        outcome([&] { detail::compress_file_b200(dir, dir + "/a.out", InputValueWidth::bits32, fmt(5)); }),
        outcome([&] { compress_file(dir, dir + "/b.out", InputValueWidth::bits32, o); }));
    report("file_bad_width",
        outcome([&] { detail::compress_file_b200(odd, dir + "/a.out", static_cast<InputValueWidth>(3), fmt(5)); }),
        outcome([&] { compress_file(odd, dir + "/b.out", static_cast<InputValueWidth>(3), o); }));
    return 0;
}
