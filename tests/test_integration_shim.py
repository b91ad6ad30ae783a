# SPDX-License-Identifier: Apache-2.0
"""The reference-side shim of INTEGRATION.md, compiled as written.

The two C++ blocks of its section 2 (the backend translation unit and its
declarations) are compiled against the reference's own headers and linked
with the reference library built from its unmodified sources
(oracle/_ref/libbenes_ref.so) and with libbenes_b200.so.  A driver then
feeds the same arguments to the shim and to the reference's portable_cpu
path (benes::compress / benes::compress_file, src/benes.cpp:422-553) and
prints the exception type and message each raised; the two must agree.
Without a GPU the valid call must fail with "b200 backend is unavailable";
with one, the shim's bytes must equal the reference's.  Runs where the
reference sources are present (it reads their headers); skipped elsewhere.
"""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("BENES_REFERENCE_DIR", "/root/reference")

DRIVER = r'''
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
    report("file_bad_width",
        outcome([&] { detail::compress_file_b200(odd, dir + "/a.out", static_cast<InputValueWidth>(3), fmt(5)); }),
        outcome([&] { compress_file(odd, dir + "/b.out", static_cast<InputValueWidth>(3), o); }));
    return 0;
}
'''


def _shim_blocks():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    section = text.split("## 2.", 1)[1].split("\n## 3.", 1)[0]
    blocks = re.findall(r"```cpp\n(.*?)```", section, re.S)
    assert len(blocks) == 2, "section 2 holds the backend unit and its declarations"
    unit = next(b for b in blocks if "#include <benes_b200.h>" in b)
    decls = next(b for b in blocks if b is not unit)
    return unit, decls


@pytest.fixture(scope="module")
def shim_results(tmp_path_factory, reference, b200):
    if not os.path.exists(os.path.join(REF, "src", "internal.hpp")):
        pytest.skip("reference sources are not present")
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ is not available")
    work = tmp_path_factory.mktemp("shim")
    unit, decls = _shim_blocks()
    # the declarations go into internal.hpp beside the CUDA ones; here they
    # follow it in a small header the unit and the driver include
    (work / "b200_decls.hpp").write_text('#pragma once\n#include "internal.hpp"\n' + decls)
    (work / "benes_b200_backend.cpp").write_text('#include "b200_decls.hpp"\n' + unit)
    (work / "driver.cpp").write_text('#include "b200_decls.hpp"\n' + DRIVER)
    ref_dir = os.path.join(ROOT, "oracle", "_ref")
    lib_dir = os.path.join(ROOT, "benes_perm_b200")
    exe = str(work / "driver")
    cmd = [cxx, "-std=c++20", "-O1", "-pthread",
           "-I", str(work), "-I", os.path.join(REF, "src"), "-I", os.path.join(REF, "include"),
           "-I", os.path.join(ROOT, "include"),
           str(work / "benes_b200_backend.cpp"), str(work / "driver.cpp"),
           "-L", ref_dir, "-lbenes_ref", "-L", lib_dir, "-lbenes_b200",
           f"-Wl,-rpath,{ref_dir}:{lib_dir}", "-o", exe]
    build = subprocess.run(cmd, capture_output=True, text=True)
    assert build.returncode == 0, build.stderr[-4000:]
    run = subprocess.run([exe, str(work)], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stderr[-2000:]
    rows = {}
    for line in run.stdout.splitlines():
        name, *rest = line.split("\t")
        rows[name] = rest
    return rows


ERROR_CASES = ["group_log2_zero", "group_log2_six", "clusters_short", "clusters_long",
               "bad_placement", "empty", "file_missing", "file_ragged", "file_bad_width"]


@pytest.mark.parametrize("case", ERROR_CASES)
def test_shim_errors_match_reference(shim_results, case):
    shim, ref = shim_results[case]
    assert not ref.startswith("ok|"), ref
    assert shim == ref


@pytest.mark.parametrize("case", ["valid_u32", "valid_u64_embedded"])
def test_shim_valid_call(shim_results, case):
    shim, ref = shim_results[case]
    assert ref == "ok|"
    if shim_results["available"][0] == "1":
        assert shim == "ok|"
        assert shim_results[case + "_bytes"][0] == "same"
    else:
        assert shim == "runtime_error|b200 backend is unavailable"
