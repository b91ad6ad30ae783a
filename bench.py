#!/usr/bin/env python
# SPDX-License-Identifier: Apache-2.0
"""Benchmark of the B200 compact encoder (one JSON line on rank 0).

Workload: a uniform random permutation of N = 2^30 uint64 entries (Fisher-
Yates driven by xoshiro256** seeded through splitmix64), middle_group_log2 5,
the balanced default clusters and embedded_output middle placement: the
configuration the headline metric is quoted on.  A step is one full compress
of that permutation.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--shard] [--no-serving] [--workload headline|serving]

``value``: entries/s with the input already in HBM (device-resident entry
point), timed with CUDA events on the launching stream over exactly K steps,
max over ranks.  ``e2e``: the same metric through the host entry point,
including the host->device copy of the input from pinned memory and the
device->host copy of the blob.  With N GPUs every rank compresses its own
permutation (replicas, weak scaling); ``--shard`` instead splits one
permutation into N subtree shards summed on rank 0 (strong scaling).  After
the timed regions the measured blob's SHA-256 is compared with the
reference's digest, every entry is checked in both directions through the
device lookup verifier, and the host entry point's blob is compared with
the device one (``verified``); a failed check exits 1.  ``serving``: the
mixed-size request stream through the serving loop against plain
per-request calls (capacity: median of three runs on one warmed server;
latency under Poisson arrivals).  ``cpu_baseline`` and ``--impl reference``
time the reference's portable_cpu encoder (built from its own sources into
oracle/_ref) with all host threads on a bounded 2^24-entry sample of the
same workload, with input from the oracle's generator.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "entries/sec compressed bit-exact at N=2^30; serving p50/p99 latency vs plain"
UNIT = "entries/s"
SEED = 0x5EED_2030
STREAM_TEST_SEED = 0x5EED_0240   # the mixed stream the GPU tests replay


def serving_specs(requests, max_log2, seed):
    """The mixed-size request stream: per request (N, generator kind, dtype,
    middle_group_log2, placement), N = round(2^U(10, max_log2)), Fisher-Yates
    or Sattolo, uint32 or uint64, m in {4, 5}, placement uniform over the
    three, default clusters.  Request i's permutation uses seed + i."""
    rng = np.random.default_rng(seed)
    specs = []
    for _ in range(requests):
        n = int(round(2 ** rng.uniform(10, max_log2)))
        kind = int(rng.integers(0, 2))                   # Fisher-Yates or Sattolo
        dtype = np.uint32 if rng.integers(0, 2) == 0 else np.uint64
        m = int(rng.choice([4, 5]))
        placement = int(rng.integers(0, 3))
        specs.append((n, kind, dtype, m, placement))
    return specs


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=("b200", "reference"))
    ap.add_argument("--log2n", type=int, default=30, help="workload size (default 30)")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-log2n", type=int, default=24,
                    help="size of the CPU sample the reference arm and cpu_baseline time")
    ap.add_argument("--cpu-full", action="store_true",
                    help="reference arm: also time one full 2^30 compress (minutes)")
    ap.add_argument("--workload", default="headline", choices=("headline", "serving"),
                    help="serving: the mixed-size request stream (not the headline metric)")
    ap.add_argument("--requests", type=int, default=4096, help="serving: number of requests")
    ap.add_argument("--no-serving", action="store_true",
                    help="headline run without the serving sub-object")
    ap.add_argument("--max-log2", type=int, default=24, help="serving: largest log2 N")
    ap.add_argument("--hbm-budget", type=int, default=120 * 10**9, help="serving: admission budget")
    ap.add_argument("--shard", action="store_true",
                    help="N>1: one permutation sharded by subtrees over the ranks (strong "
                         "scaling) instead of one replica per rank")
    ap.add_argument("--workers", type=int, default=4,
                    help="serving: concurrent workers for requests above one tile")
    return ap.parse_args()


def workload(log2n):
    import benes_perm_b200 as bp
    fmt = bp.FormatOptions(middle_group_log2=5, middle_placement=bp.MiddlePlacement.embedded_output)
    return 1 << log2n, fmt


def workload_config(n, log2n, world, shard_mode=False):
    return {
        "workload": f"compress uniform random permutation, N=2^{log2n} uint64, m=5, "
                    "default clusters, embedded_output",
        "n": n, "entry_bytes": 8, "middle_group_log2": 5, "clusters": "balanced default",
        "middle_placement": "embedded_output",
        "permutation": "Fisher-Yates, xoshiro256** seeded by splitmix64(0x5EED2030)",
        "l2": "inputs larger than L2 (8 GiB per step), no flush",
        "parallelism": (f"subtree shards x{world} of one permutation (top log2 N levels on "
                        "every rank, shard blobs summed on rank 0)" if shard_mode else
                        f"replicas x{world} (one permutation per rank)"),
    }


def replica_seed(rank):
    """Each replica compresses its own permutation (distinct seeds)."""
    return SEED + rank


def max_over_ranks(seconds, dist, device):
    """The slowest rank's time: the job is done when every replica is."""
    if dist is None:
        return seconds
    import torch
    t = torch.tensor([seconds], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(n, steps, world, seconds):
    """Whole-job entries/s: every rank compresses `steps` permutations of n."""
    return n * steps * world / seconds


def dist_setup(gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ----------------------------------------------------------------- clocks

class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.3)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, mx, reasons = [], None, set()
        for ln in getattr(self, "lines", []):
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------- roofline

def algorithmic_bytes(n, depth, tile, entry_bytes, switch_bits, middle_bits, walk_levels,
                      place_levels=()):
    """Compulsory HBM bytes per kernel kind for one compress: every array a
    kernel must touch, read once and written once at its minimal width.
    Levels in `walk_levels` are coloured by orbit walks (walk + jump), the
    other global levels by union-find (union).  Only level 0 builds an
    inverse from its values (partitioned, kind "place", on the levels in
    `place_levels`; else "inverse"); every later level's inverse is written
    by its parent's output pass ("output_bits")."""
    kinds = ("inverse", "place", "union", "walk", "jump", "resolve", "output_bits", "emit",
             "tile")
    per = {k: 0.0 for k in kinds}
    for lvl in range(tile):
        w = entry_bytes if lvl == 0 else 4
        if lvl == 0:
            per["place" if lvl in place_levels else "inverse"] += (w + 4) * n
        if lvl in walk_levels:
            per["walk"] += 12 * n                  # values, inverse, owner stamp per vertex
            per["jump"] += 2 * n                   # ruler states (16 B per 16 slots) read+written
            per["resolve"] += (4 + w + 4) * n + n / 8  # owners, values, children, bits
        else:
            per["union"] += 8 * n                  # inverse, one word per pair read+written
            per["resolve"] += (2 + w + 4) * n + n / 8  # union-find words, values, children, bits
        # this level's inverse, the children's inverse (when they are global), output bits
        per["output_bits"] += 4 * n + (4 * n if lvl + 1 < tile else 0) + n / 8
        per["emit"] += n / 4                       # bits of both sides, read and placed
    w = entry_bytes if tile == 0 else 4
    per["tile"] = w * n + 2 * (depth - tile) * n / 16 + middle_bits / 8
    pipeline = (entry_bytes * n + 4 * n * max(depth - 1, 0) + 4 * n * depth
                + 2 * switch_bits / 8 + 4 * n + middle_bits / 8)
    return per, pipeline


def random_accesses(n, tile, walk_levels, place_levels):
    """Random 4-byte accesses per step by kernel kind and level, the least
    each kind's algorithm needs (reads, writes): the inverse scatter one
    write per entry (level 0 only; later inverses are written in order); a
    union per output pair at least two finds and a link (a read per entry,
    a write per pair); an orbit-walk step two gathers and an owner stamp
    (two reads and a write per entry); finalize one lookup per pair-node
    (find or owner-to-colour); the output pass one colour bit per output
    pair."""
    acc = {}
    half = n / 2
    for lvl in range(tile):
        if lvl == 0:
            acc[("place" if lvl in place_levels else "inverse", lvl)] = (0.0, float(n))
        if lvl in walk_levels:
            acc[("walk", lvl)] = (2.0 * n, float(n))
        else:
            acc[("union", lvl)] = (float(n), half)
        acc[("resolve", lvl)] = (half, 0.0)
        acc[("output_bits", lvl)] = (half, 0.0)
    return acc


def random_access_roofline(n, depth, tile, walk_levels, place_levels, node_log2, kernel_secs,
                           probe):
    """Per kernel kind: the time the least random accesses of its algorithm
    take at the probed random-access rates, against the measured time.
    Apart from the input and output streams every access of these kernels
    is random, so this, not streaming bandwidth, is the bound that applies.
    ``bound_l2_s`` takes every access at the L2-resident rates: a lower
    bound on the time, hence ``frac`` <= 1.  ``bound_dram_s`` takes the DRAM
    rates for levels whose nodes exceed 2^23 entries (their arrays do not
    fit L2); a kind can beat it where its access order keeps them in L2
    (claim-ordered work, the partitioned inverse)."""
    bound_l2, bound_dram = {}, {}
    l2, dram = probe["l2_32MB"], probe["dram_4GB"]
    for (kind, lvl), (reads, writes) in random_accesses(n, tile, walk_levels,
                                                         place_levels).items():
        fast = reads / l2["reads_per_s"] + writes / l2["writes_per_s"]
        rates = l2 if node_log2[lvl] <= 23 else dram
        slow = reads / rates["reads_per_s"] + writes / rates["writes_per_s"]
        bound_l2[kind] = bound_l2.get(kind, 0.0) + fast
        bound_dram[kind] = bound_dram.get(kind, 0.0) + slow
    kinds = {}
    for kind, t in bound_l2.items():
        measured = kernel_secs.get(kind, 0.0)
        if measured > 0:
            kinds[kind] = {"bound_l2_s": round(t, 6), "bound_dram_s": round(bound_dram[kind], 6),
                           "measured_s": round(measured, 6), "frac": round(t / measured, 3)}
    total_bound = sum(bound_l2.values())
    total = sum(v for k, v in kernel_secs.items() if k in bound_l2)
    return {"probe_accesses_per_s": {k: {kk: round(vv / 1e9, 1) for kk, vv in v.items()}
                                     for k, v in probe.items()},
            "probe_unit": "G accesses/s (4-byte; reads, writes, dependent chain steps)",
            "kinds": kinds, "bound_l2_s": round(total_bound, 6),
            "bound_dram_s": round(sum(bound_dram.values()), 6), "measured_s": round(total, 6),
            "frac": round(total_bound / total, 3) if total else None,
            "note": "least random 4-byte accesses of each kind's algorithm at the probed rates; "
                    "the tile kernel (shared memory) is not included"}


def measured_traffic(kind, n, node_log2s):
    """DRAM bytes per step of `kind` from the committed ncu summary
    (profiles/dram_traffic.json): bytes per entry of each level, measured
    with ncu on a 2^26-entry input and keyed by the level's node size, summed
    here over the levels that run the kind (`node_log2s`), times the entries.
    Node sizes beyond the measured ones take the nearest measured size (a
    node far above L2 size costs the same per entry at any size)."""
    try:
        with open(os.path.join(ROOT, "profiles", "dram_traffic.json")) as f:
            table = json.load(f)
        row = table["kinds"][kind]
    except (OSError, KeyError, ValueError):
        return None
    known = {int(k): v for k, v in row["by_node_log2"].items()}

    def per_entry(lg):
        return known[min(known, key=lambda k: (abs(k - lg), k))]

    return {"bytes_per_step": sum(per_entry(lg) for lg in node_log2s) * n,
            "source": f"{table['source']}; {row['launch']}"}


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# ----------------------------------------------------------------- arms

def cpu_sample_config(n_sample):
    """Config of the CPU sample: the headline workload's format and generator
    at a bounded size."""
    lg = n_sample.bit_length() - 1
    return {
        "workload": f"compress uniform random permutation, N=2^{lg} uint64, m=5, default "
                    "clusters, embedded_output (bounded sample of the N=2^30 workload)",
        "n": n_sample, "entry_bytes": 8, "middle_group_log2": 5, "clusters": "balanced default",
        "middle_placement": "embedded_output", "sample_of_n": 1 << 30,
        "permutation": "Fisher-Yates, xoshiro256** seeded by splitmix64(0x5EED2030)",
    }


def _cpu_setup(n_sample):
    """The reference library (oracle/_ref, built from the reference's own
    sources) and the sample input, made by the oracle's restatement of the
    workload generator: nothing of the B200 library is loaded."""
    from oracle.oracle import Oracle, Reference, make_format
    ref = Reference()
    perm = Oracle().fill_permutation(0, SEED, n_sample, np.uint64)
    fmt = make_format(5, [], [], 2)
    out = np.zeros(ref.encoded_size(n_sample, fmt), dtype=np.uint8)
    return ref, ref.hardware_threads(), perm, fmt, out


def reference_arm(args, world, rank):
    """portable_cpu of the reference on the host cores: each step compresses
    a bounded sample (2^24 entries by default) of the headline workload with
    every host thread; ``config`` names the sample actually timed."""
    if rank != 0:
        return
    n_sample = 1 << args.cpu_log2n
    ref, threads, perm, fmt, out = _cpu_setup(n_sample)
    for _ in range(args.warmup):
        ref.compress(perm, fmt, threads=threads, out=out)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ref.compress(perm, fmt, threads=threads, out=out)
    secs = time.perf_counter() - t0
    value = n_sample * args.steps / secs
    sample = (f"each step compresses a {n_sample}-entry (2^{args.cpu_log2n}) uint64 uniform "
              f"permutation with the headline format, reference portable_cpu, {threads} threads; "
              "a full 2^30 compress per step would not fit the run's time")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": secs / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "uint64", "data": "synthetic",
        "config": cpu_sample_config(n_sample),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if args.cpu_full:
        line["full_2p30"] = cpu_full_run()
    print(json.dumps(line), flush=True)


def cpu_baseline(args):
    n_sample = 1 << args.cpu_log2n
    ref, threads, perm, fmt, out = _cpu_setup(n_sample)
    ref.compress(perm, fmt, threads=threads, out=out)
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        ref.compress(perm, fmt, threads=threads, out=out)
        times.append(time.perf_counter() - t0)
    med = statistics.median(times)
    return {"value": n_sample / med, "unit": UNIT, "cores": threads, "kind": "reference",
            "config": cpu_sample_config(n_sample),
            "sample": f"median of 3 compresses of a 2^{args.cpu_log2n}-entry uint64 uniform "
                      "permutation with the headline format by the reference portable_cpu "
                      f"encoder, {threads} threads"}


def cpu_full_run():
    """One reference portable_cpu compress of the full 2^30 workload with all
    host threads (minutes; about 50 GB of host memory), its bytes checked
    against the committed reference digest."""
    import hashlib
    n = 1 << 30
    ref, threads, perm, fmt, out = _cpu_setup(n)
    t0 = time.perf_counter()
    blob = ref.compress(perm, fmt, threads=threads, out=out)
    secs = time.perf_counter() - t0
    want = reference_digest(n, SEED)
    return {"value": n / secs, "unit": UNIT, "seconds": secs, "cores": threads,
            "kind": "reference", "n": n,
            "sha256_matches_digest": (hashlib.sha256(blob).hexdigest() == want) if want else None}


def reference_digest(n, seed):
    """The committed SHA-256 of the reference's blob for the headline
    workload at (n, seed), if tests/golden/reference_digests.json has it."""
    try:
        with open(os.path.join(ROOT, "tests", "golden", "reference_digests.json")) as f:
            d = json.load(f)["config3"]
    except (OSError, KeyError, ValueError):
        return None
    return d["sha256"] if d["n"] == n and d["seed"] == seed else None


def b200_arm(args, world, rank, local):
    import torch
    import benes_perm_b200 as bp

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    n, fmt = workload(args.log2n)
    size = bp.encoded_size(n, fmt)
    depth, tile = bp.describe(n, fmt)

    # --shard: every rank holds the same permutation and encodes its subtree
    # shard (bpb200_compress_device_shard); the shards are summed on rank 0
    shard_mode = args.shard and world > 1
    seed = SEED if shard_mode else replica_seed(rank)
    host = torch.empty(n, dtype=torch.int64, pin_memory=True)
    perm = host.numpy().view(np.uint64)
    bp.fill_permutation(bp.PermutationKind.uniform, seed, n, np.uint64, out=perm)
    d_in = host.to(f"cuda:{local}", non_blocking=False)
    d_blob = torch.empty((size + 3) // 4 * 4, dtype=torch.uint8, device=f"cuda:{local}")
    stream = torch.cuda.current_stream()

    def step():
        if shard_mode:
            bp.compress_device_shard(d_in.data_ptr(), n, 8, d_blob.data_ptr(), size, rank, world,
                                     fmt, stream.cuda_stream)
            bp.combine_shards(d_blob)
            return None
        return bp.compress_device(d_in.data_ptr(), n, 8, d_blob.data_ptr(), size, fmt,
                                  stream.cuda_stream)

    # random-access rates of this GPU (L2-resident and DRAM arrays), the
    # bound of the encoder's kernels; measured before the timed steps
    probe = {"l2_32MB": bp.probe_random_access(23), "dram_4GB": bp.probe_random_access(30)}
    for _ in range(max(args.warmup, 3)):
        step()
    _, _, launches_per_step = bp.last_profile()

    gpu_index = local
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    if vis and vis.split(",")[local].strip().isdigit():
        gpu_index = int(vis.split(",")[local])
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    # per-kernel device times come from the timed steps themselves: every
    # launch is bracketed by CUDA events on its own stream (two event
    # records per launch, well under 1 ms per step)
    bp.set_profiling(True)
    kernel_secs = {}
    kernel_counts = {}
    walk_levels = set()
    place_levels = set()
    level_ms = {}
    with ClockSampler(gpu_index) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            step()
            ks, kc, _ = bp.last_profile()
            for k in ks:
                kernel_secs[k] = kernel_secs.get(k, 0.0) + ks[k] / args.steps
                kernel_counts[k] = kc[k]
            marks = bp.last_profile_launches()
            walk_levels |= {lvl for kind, lvl, _ in marks if kind == "walk"}
            place_levels |= {lvl for kind, lvl, _ in marks if kind == "place"}
            for kind, lvl, sec in marks:
                row = level_ms.setdefault(lvl, {})
                row[kind] = row.get(kind, 0.0) + sec * 1e3 / args.steps
        stop.record(stream)
        torch.cuda.synchronize()
    bp.set_profiling(False)
    if dist is not None:
        dist.barrier()
    secs = max_over_ranks(start.elapsed_time(stop) / 1e3, dist, f"cuda:{local}")
    jobs = 1 if shard_mode else world  # permutations the whole job compresses per step
    value = replica_throughput(n, args.steps, jobs, secs)

    # end to end through the host entry point: pinned input in, pinned blob out
    host_blob = torch.empty(size, dtype=torch.uint8, pin_memory=True)
    blob_np = host_blob.numpy()
    opts = bp.CompressOptions(format=fmt)
    def host_call():
        if shard_mode:
            got = bp.compress_sharded(perm, opts)
            if got is not None:
                blob_np[:] = np.frombuffer(got, dtype=np.uint8)
        else:
            bp.compress(perm, opts, out=blob_np)

    host_call()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.e2e_steps):
        host_call()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_secs = max_over_ranks(e0.elapsed_time(e1) / 1e3, dist, f"cuda:{local}")
    e2e_value = replica_throughput(n, args.e2e_steps, jobs, e2e_secs)

    if shard_mode and rank != 0:
        verified = {"ok": True, "note": "shard mode: rank 0 holds and checks the combined blob"}
    else:
        verified = verify_output(bp, torch, d_in, d_blob, host_blob, n, size, fmt, stream,
                                 reference_digest(n, seed))
    if not verified["ok"]:
        print(f"rank {rank}: the measured blob failed verification: {verified}",
              file=sys.stderr, flush=True)
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        if not verified["ok"]:
            sys.exit(1)
        return

    # roofline of the dominant kernel kind: its algorithmic bytes over all of
    # its launches in a step, divided by their summed event-timed durations
    switch_bits, middle_bits = _section_bits(n, fmt)
    alg, pipeline_bytes = algorithmic_bytes(n, depth, tile, 8, switch_bits, middle_bits,
                                            walk_levels, place_levels)
    timed = {k: v for k, v in kernel_secs.items() if alg.get(k, 0) > 0 and v > 0}
    dominant = max(timed, key=timed.get)
    peak, peak_kind = load_peaks()
    achieved = alg[dominant] / timed[dominant] / 1e9
    total_kernel = sum(kernel_secs.values())
    node_log2 = {lvl: max(0, (-(-n >> lvl) - 1).bit_length()) for lvl in range(tile + 1)}
    kind_levels = {"union": [node_log2[l] for l in range(tile) if l not in walk_levels],
                   "walk": [node_log2[l] for l in sorted(walk_levels)],
                   "jump": [node_log2[l] for l in sorted(walk_levels)],
                   "tile": [node_log2[tile]]}
    traffic = measured_traffic(dominant, n,
                               kind_levels.get(dominant, [node_log2[l] for l in range(tile)]))
    roofline = {
        "bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak, "unit": "GB/s",
        "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
        "traffic": traffic["bytes_per_step"] if traffic else None,
        "traffic_source": traffic["source"] if traffic else None,
        "algorithmic_bytes_per_step": alg[dominant],
        "kernel_seconds_per_step": timed[dominant],
        "share_of_device_time": timed[dominant] / total_kernel,
        "per_kind_gbs": {k: round(alg[k] / timed[k] / 1e9, 1) for k in timed},
    }
    pipeline = {
        "algorithmic_bytes": pipeline_bytes, "seconds": secs / args.steps,
        "achieved": pipeline_bytes / (secs / args.steps) / 1e9, "peak": peak, "unit": "GB/s",
        "frac": pipeline_bytes / (secs / args.steps) / 1e9 / peak,
    }
    random_roof = random_access_roofline(n, depth, tile, walk_levels, place_levels, node_log2,
                                         kernel_secs, probe)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": secs / args.steps * 1e3,
        "higher_is_better": True, "scaling": "strong" if shard_mode else "weak",
        "vs_baseline": None, "dtype": "uint64",
        "data": "synthetic", "config": workload_config(n, args.log2n, world, shard_mode),
        "clocks": clocks.summary(),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": n * 8,
                "d2h_bytes_per_step": size, "steps": args.e2e_steps},
        "gpu_launches": launches_per_step * args.steps,
        "roofline": roofline,
        "pipeline_roofline": pipeline,
        "random_access_roofline": random_roof,
        "per_level_ms": {str(l): {k: round(v, 3) for k, v in sorted(row.items())}
                         for l, row in sorted(level_ms.items())},
        "kernel_seconds": {k: round(v, 6) for k, v in kernel_secs.items()},
        "kernel_launches": kernel_counts,
        "levels": {"depth": depth, "tile_level": tile, "walk_levels": sorted(walk_levels)},
        "verified": verified,
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args)
    if world == 1 and not args.no_serving:
        # the serving stream runs after the headline's buffers are released
        del d_in, d_blob, host, host_blob, perm, blob_np
        torch.cuda.empty_cache()
        bp.shutdown()
        line["serving"] = serving_run(args)
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    if not verified["ok"]:
        sys.exit(1)


def verify_output(bp, torch, d_in, d_blob, host_blob, n, size, fmt, stream, digest):
    """Checks the measured output after the timed regions: the blob's SHA-256
    equals the reference's own blob's (committed digest of the reference's
    portable encoder on this exact input, when there is one: the canonical
    bytes, not only a decodable blob), every entry of the device blob
    round-trips through the device lookup verifier (p[i] for all i, then
    p^-1[p[i]] == i), and the host entry point's blob equals the
    device-resident one byte for byte."""
    import hashlib
    t0 = time.perf_counter()
    match = None
    if digest is not None:
        match = hashlib.sha256(host_blob.numpy()).hexdigest() == digest
    out = torch.empty(n, dtype=torch.int64, device=d_in.device)
    bp.lookup_device(d_blob.data_ptr(), size, n, fmt, out.data_ptr(), n,
                     stream=stream.cuda_stream)
    forward = bool(torch.equal(out, d_in))
    bp.lookup_device(d_blob.data_ptr(), size, n, fmt, out.data_ptr(), n,
                     d_queries=d_in.data_ptr(), inverse=True, stream=stream.cuda_stream)
    inverse = bool(torch.equal(out, torch.arange(n, dtype=torch.int64, device=d_in.device)))
    del out
    same = bool(torch.equal(host_blob.to(d_blob.device), d_blob[:size]))
    return {"ok": forward and inverse and same and match is not False,
            "reference_sha256_match": match, "forward_lookups": forward,
            "inverse_lookups": inverse, "host_blob_equals_device_blob": same,
            "method": "SHA-256 against the reference's blob (tests/golden/"
                      "reference_digests.json); every entry through bpb200_lookup_device, "
                      "both directions",
            "seconds": round(time.perf_counter() - t0, 3)}


def _section_bits(n, fmt):
    """Switch bits per side and middle bits of the layout (FormatSizeCache)."""
    leaf = 1 << fmt.middle_group_log2
    memo = {}

    def fbits(c):
        f = 1
        for i in range(2, c + 1):
            f *= i
        return (f - 1).bit_length()

    def sizes(c):
        if c <= leaf:
            return 0, fbits(c)
        if c in memo:
            return memo[c]
        a = sizes(c - c // 2)
        b = sizes(c // 2)
        memo[c] = (c // 2 + a[0] + b[0], a[1] + b[1])
        return memo[c]

    return sizes(n)


def stream_digests(requests, max_log2):
    """The reference's per-request SHA-256 prefixes (hex, 128 bits) for the
    mixed stream, from tests/golden/reference_digests.json, or None."""
    try:
        with open(os.path.join(ROOT, "tests", "golden", "reference_digests.json")) as f:
            d = json.load(f)["stream4096"]
    except (OSError, KeyError, ValueError):
        return None
    if d["seed"] != SEED or d["max_log2"] != max_log2 or d["requests"] < requests:
        return None
    return d["sha256_128"][:requests]


def serving_run(args):
    """Mixed-size request stream (the fifth configuration): plain
    per-request calls (bpb200_compress one after another), then the serving
    loop twice: every request submitted at once (capacity) and Poisson
    arrivals at 1.5x the plain path's request rate (paced).  Every blob of
    every run is compared with the plain call's and, where the committed
    reference digests cover the stream, with the reference's own bytes.
    Returns the record (host wall clock, submit to blob in host memory)."""
    import concurrent.futures as futures
    import hashlib
    import threading

    import benes_perm_b200 as bp

    specs = serving_specs(args.requests, args.max_log2, SEED)
    rng = np.random.default_rng(SEED + 1)                # arrival times
    opts = [bp.CompressOptions(format=bp.FormatOptions(middle_group_log2=m,
                                                       middle_placement=bp.MiddlePlacement(pl)))
            for (_, _, _, m, pl) in specs]

    def make(i):
        n, kind, dtype, _, _ = specs[i]
        return bp.fill_permutation(bp.PermutationKind(kind), SEED + i, n, dtype)

    with futures.ThreadPoolExecutor(16) as pool:
        perms = list(pool.map(make, range(len(specs))))
    total = sum(p.size for p in perms)
    for p, o in zip(perms[:8], opts[:8]):                # warm-up
        bp.compress(p, o)

    # plain per-request calls; the byte checks run after the timing
    t0 = time.perf_counter()
    plain_blobs = [bp.compress(p, o) for p, o in zip(perms, opts)]
    t_plain = time.perf_counter() - t0
    plain_rate = total / t_plain
    plain = [hashlib.sha256(b).hexdigest()[:32] for b in plain_blobs]
    del plain_blobs
    want = stream_digests(len(perms), args.max_log2)

    # One long-lived server, as in deployment: before the timed runs it
    # encodes the 16 largest requests and the first 48 once (untimed), so its
    # workspaces and group buffers are already sized when the clock starts.
    server = bp.Server(hbm_budget_bytes=args.hbm_budget, max_batch=256, workers=args.workers)
    warm = sorted(range(len(perms)), key=lambda i: -perms[i].size)[:16] + list(range(48))
    for i in warm:
        server.wait(server.submit(perms[i], opts[i]))

    def serve(arrivals):
        """Runs the stream through the server; arrivals (seconds from the
        start, or None for all at once) pace the submissions.  Returns the
        wall time, the sorted latencies, the blob digests and the kernel
        launches of this run."""
        launches0 = server.stats()["kernel_launches"]
        tickets = [None] * len(perms)
        ready = [threading.Event() for _ in perms]

        def submitter():
            start = time.perf_counter()
            for i, (p, o) in enumerate(zip(perms, opts)):
                if arrivals is not None:
                    delay = arrivals[i] - (time.perf_counter() - start)
                    if delay > 0:
                        time.sleep(delay)
                tickets[i] = server.submit(p, o)
                ready[i].set()

        blobs = [None] * len(perms)
        latencies = []
        t1 = time.perf_counter()
        th = threading.Thread(target=submitter)
        th.start()
        for i in range(len(perms)):
            ready[i].wait()
            blobs[i], lat = server.wait(tickets[i])
            latencies.append(lat)
        t_serve = time.perf_counter() - t1
        th.join()
        launches = server.stats()["kernel_launches"] - launches0
        got = [hashlib.sha256(b).hexdigest()[:32] for b in blobs]
        return t_serve, np.sort(np.array(latencies)), got, launches

    # capacity: every request submitted at once (offered load above capacity),
    # three runs on the warm server; the median run is reported (host-side
    # staging makes single runs vary with the load on the shared host)
    runs = [serve(None) for _ in range(3)]
    capacity_rates = [total / r[0] for r in runs]
    t_serve, lat, got, launches = sorted(runs, key=lambda r: r[0])[1]
    got_all = [r[2] for r in runs]
    # latency under the stated offered load
    rate = 1.5 * len(perms) / t_plain                    # offered load, requests/s
    arrivals = np.cumsum(rng.exponential(1.0 / rate, len(perms)))
    t_paced, lat_paced, got_paced, _ = serve(arrivals)
    server.close()
    identical = all(g == plain for g in got_all) and got_paced == plain
    ref_match = None if want is None else (
        plain == want and all(g == want for g in got_all) and got_paced == want)
    return {
        "metric": "entries/s on the mixed-size serving stream (serving loop vs plain per-request)",
        "value": total / t_serve, "unit": UNIT, "n_gpus": 1, "higher_is_better": True,
        "plain_per_request": plain_rate, "ratio_vs_plain": (total / t_serve) / plain_rate,
        "capacity": {"note": "all requests submitted at once; median of three runs",
                     "runs_entries_per_s": capacity_rates,
                     "p50_latency_s": float(np.percentile(lat, 50)),
                     "p99_latency_s": float(np.percentile(lat, 99))},
        "paced": {"offered_load_requests_per_s": rate,
                  "offered_over_plain_capacity": 1.5,
                  "value": total / t_paced, "ratio_vs_plain": (total / t_paced) / plain_rate,
                  "p50_latency_s": float(np.percentile(lat_paced, 50)),
                  "p99_latency_s": float(np.percentile(lat_paced, 99))},
        "identical_bytes": bool(identical),
        "reference_sha256_match": ref_match,
        "kernel_launches": launches,
        "launches_per_request": launches / len(perms),
        "workers": args.workers, "data": "synthetic",
        "config": {"workload": f"{len(perms)} requests, N = round(2^U(10,{args.max_log2})), "
                               "Fisher-Yates or Sattolo, uint32 or uint64, m in {4,5}, "
                               "placement uniform over 3, default clusters; capacity run with "
                               "every request submitted at once, paced run with Poisson arrivals",
                   "entries": int(total), "hbm_budget_bytes": args.hbm_budget,
                   "timing": "host wall clock (submit to blob in host memory) on one "
                             "server, warmed with 64 of the stream's requests before the "
                             "timed runs; capacity: median of three runs; byte checks after "
                             "the timed runs"},
    }


def serving_arm(args):
    print(json.dumps(serving_run(args)), flush=True)


def main():
    args = parse_args()
    world, rank, local = dist_setup(args.gpus)
    if args.workload == "serving":
        if rank == 0:
            serving_arm(args)
        return
    if args.impl == "reference":
        reference_arm(args, world, rank)
    else:
        b200_arm(args, world, rank, local)


if __name__ == "__main__":
    main()
