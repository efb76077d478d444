#!/usr/bin/env python
"""PairHMM benchmark on one node: GCUPS of the batched engine on the 2,000-region uneven workload.

One step = the whole PairHMM path over one batch of 2,000 active regions (reads U[10,500] of
100-250 bp, 2-32 haplotypes of 150-600 bp; seeded synthetic data): the FP32 wavefront pass over
every read x haplotype pair and the FP64 recompute of the pairs whose FP32 sum falls below 1e-28.

  value      batched GCUPS with the batch already in HBM (device pipeline replayed, CUDA events)
  e2e        the same through phmm_compute_regions from pinned host buffers (H2D of all reads and
             haplotypes and D2H of all likelihoods inside every step)
  plain      one region per call (the one-region-per-launch form), for the batched/plain ratio
  latency    p50/p99 region latency of the serving loop under Poisson arrivals at 80% of capacity
  roofline   the FP32 wavefront pass: 12 FLOP per cell against the device's measured FP32 FMA peak
  cpu_baseline  the reference's own AVX PairHMM (compiled from its sources) on all host cores
  smith_waterman  realignment of every read of the batch to a haplotype of its region on the GPU
             (resident and end to end), checked against the oracle; the reference's aligner on the host

Multi-GPU: one process per GPU (torchrun); every rank runs its own 2,000 regions (regions are
independent: weak scaling, no collective on the data path); value = all ranks' cells / max time.
`--impl reference` times the reference's CPU implementation instead (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
import ctypes as C
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "PairHMM GCUPS batched vs plain per-region, 1 B200, ≤1e-4 log10 err; p99 latency"
WORKLOAD = ("2,000 batched uneven active regions in one launch sequence: reads U[10,500] per region of "
            "length U[100,250], base quality Phred U[2,41], ins/del 45, GCP 10, 1% substitution errors; "
            "haplotypes U[2,32] per region of 150-600 bp (SNP/indel edits of one window); FP32 with "
            "FP64 recompute below 1e-28")
FLOP_PER_CELL = 12  # 8 multiplies + 4 adds per cell (M, I, D updates)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms while active."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(5)

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def traffic_from_profiles(kernel_class: int) -> float | None:
    """DRAM bytes per launch of the dominant FP32 kernel from the committed ncu summary, when that
    summary covers the same kernel class (None otherwise)."""
    for p in sorted((ROOT / "profiles").glob("fwd_f32_*.md")):
        cls, traffic = None, None
        for line in p.read_text().splitlines():
            if line.startswith("class:"):
                cls = int(line.split(":", 1)[1])
            if line.startswith("traffic_bytes_per_launch:"):
                traffic = float(line.split(":", 1)[1])
        if cls == kernel_class and traffic is not None:
            return traffic
    return None


# ---- reference CPU arm -----------------------------------------------------------------------

def reference_gcups(batch, regions, threads: int) -> tuple[float, float]:
    """Runs the reference's schedule_pairhmm (AVX path) over `regions`, one region per worker thread
    like HaplotypeCaller's region pool; returns (GCUPS, seconds)."""
    from oracle import Ref

    ref = Ref()
    cells = sum(batch.subset([g]).cells() for g in regions)

    def work(g):
        return ref.schedule_region(batch, g, 0.02, 0.02)

    with ThreadPoolExecutor(max_workers=threads, initializer=ref.init_thread) as ex:
        t = time.perf_counter()
        list(ex.map(work, regions))
        dt = time.perf_counter() - t
    return cells / dt / 1e9, dt


# The FP32 -> FP64 switch in log10 space: an FP32 sum accepted by the switch (>= 1e-28f) reports at
# least log10(1e-28f) - log10(2^120 as the float constant); a likelihood below this value can only
# have come from the FP64 recompute.
LOG10_SWITCH = float(np.log10(np.float64(np.float32(1e-28))) - np.float64(np.float32(36.1236000061)))
ERR_EDGES = [0.0, 1e-12, 1e-10, 1e-8, 1e-6, 1e-5, 1e-4, np.inf]


def error_report(got: np.ndarray, flags: np.ndarray, f64: np.ndarray) -> dict:
    """|log10 error| of every pair against the all-FP64 model (the pairs with an empty read or
    haplotype, NaN on both sides, are counted apart)."""
    fin = np.isfinite(got) & np.isfinite(f64)
    err = np.abs(got[fin] - f64[fin])
    fl = flags[fin].astype(bool)
    hist = np.histogram(err, bins=ERR_EDGES)[0]
    return {"pairs": int(err.size), "pairs_total": int(got.size),
            "nan_pairs_agree": bool(np.array_equal(np.isnan(got), np.isnan(f64))),
            "max": float(err.max()) if err.size else 0.0,
            "p99": float(np.percentile(err, 99)) if err.size else 0.0,
            "p50": float(np.percentile(err, 50)) if err.size else 0.0,
            "over_1e-4": int(np.sum(err > 1e-4)),
            "max_fp32_pairs": float(err[~fl].max()) if (~fl).any() else 0.0,
            "max_fp64_pairs": float(err[fl].max()) if fl.any() else 0.0,
            "histogram": {f"<{hi:g}" if hi != np.inf else ">=1e-4": int(c) for hi, c in zip(ERR_EDGES[1:], hist)},
            "model": "all-FP64 check arithmetic on the device (phmm_resident_check_fp64), equal to the CPU "
                     "all-FP64 oracle pair for pair in the GPU tests"}


def reference_whole_batch(batch, got: np.ndarray, flags: np.ndarray, threads: int) -> dict:
    """Every region of the batch through the reference's own schedule_pairhmm (oracle/_ref, AVX-512
    path, `threads` host threads), compared with the engine pair by pair; and every pair whose
    reference likelihood lies below the FP32 -> FP64 switch (a value only the FP64 recompute can
    give) checked against the engine's FP64 flag."""
    from oracle import Ref

    ref = Ref()
    offs = batch.out_offsets()
    want = np.empty(batch.out_size, np.float64)

    def work(g):
        want[offs[g]:offs[g + 1]] = ref.schedule_region(batch, g, 0.02, 0.02).reshape(-1)

    t = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads, initializer=ref.init_thread) as ex:
        list(ex.map(work, range(batch.n_regions)))
    dt = time.perf_counter() - t
    fin = np.isfinite(got) & np.isfinite(want)
    d = np.abs(got - want)
    fl = flags.astype(bool)
    only_f64 = fin & (want < LOG10_SWITCH)
    near = fin & (np.abs(want - LOG10_SWITCH) < 1e-5)
    return {"pairs": int(fin.sum()), "nan_pairs_agree": bool(np.array_equal(np.isnan(got), np.isnan(want))),
            "max_abs_diff": float(d[fin].max()) if fin.any() else 0.0,
            "pairs_bit_equal_le_1e-12": int(np.sum(d[fin] <= 1e-12)),
            "pairs_diff_over_1e-12": int(np.sum(d[fin] > 1e-12)),
            "pairs_diff_over_1e-5": int(np.sum(d[fin] > 1e-5)),
            "reference_pairs_only_fp64": int(only_f64.sum()),
            "fp64_flag_disagreements": int(np.sum(only_f64 & ~fl)),
            "engine_fp64_pairs": int(fl.sum()),
            "pairs_within_1e-5_of_switch": int(near.sum()),
            "reference_seconds": round(dt, 2), "reference_gcups": round(batch.cells() / dt / 1e9, 2),
            "threads": threads,
            "note": "pairs differing by more than 1e-12 are pairs the reference leaves to its intra kernel "
                    "(ungrouped by its SIMD packing), which rounds the prior and the log10 once more"}


# ---- ranks --------------------------------------------------------------------------------------

def shard_seed(rank: int) -> int:
    """Each rank computes its own 2,000-region batch of the benchmark's shape (regions are
    independent: weak scaling, no data exchanged between ranks)."""
    return 1 + rank


def rank_reduce(dist, x: float, op: str = "max", device: str = "cpu") -> float:
    """Max or sum of a per-rank number over all ranks (identity with one process).  Every rank calls
    it the same number of times in the same order."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def weak_scaling_value(dist, cells_per_step: float, steps: int, device_ms: float, device: str = "cpu") -> tuple:
    """(GCUPS of the whole job, ms per step): all ranks' cells over the slowest rank's device time."""
    dev_ms = rank_reduce(dist, device_ms, "max", device)
    total = rank_reduce(dist, float(cells_per_step), "sum", device) * steps
    return total / (dev_ms / 1e3) / 1e9, dev_ms / steps


def strong_scaling_regions(batch, rank: int, world: int) -> list[int]:
    """The regions of one shared batch that rank `rank` of `world` computes in the strong-scaling
    leg: the rank's part of phmm_partition_regions (longest-processing-time greedy on region cells,
    the same split on every rank, nothing exchanged)."""
    from rovaca_b200 import partition_regions

    part, _ = partition_regions(batch, world)
    return [int(g) for g in np.nonzero(part == rank)[0]]


def run_reference(args, rank: int, world: int) -> None:
    if rank != 0:
        return
    from oracle import ref_available
    from rovaca_b200 import synth

    if not ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libphmm_ref.so was not built "
                          "(needs the reference sources and oracle/build_ref.sh)"}), flush=True)
        return
    batch = synth.config1(seed=1)
    cores = os.cpu_count() or 1
    sample = list(range(64))
    for _ in range(args.warmup):
        reference_gcups(batch, sample[:8], cores)
    times, cells = [], sum(batch.subset([g]).cells() for g in sample)
    for _ in range(args.steps):
        _, dt = reference_gcups(batch, sample, cores)
        times.append(dt)
    gcups = cells * len(times) / sum(times) / 1e9
    line = {
        "metric": METRIC, "value": round(gcups, 3), "unit": "GCUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * sum(times) / len(times), 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 recompute)", "data": "synthetic (seeded)",
        "impl": "reference",
        "config": {"workload": WORKLOAD, "regions_per_step": len(sample), "cells_per_step": cells},
        "cpu_baseline": {"value": round(gcups, 3), "unit": "GCUPS", "cores": cores, "kind": "reference",
                         "sample": f"regions 0-{len(sample) - 1} of the 2,000-region batch per step, one region "
                                   "per thread, reference schedule_pairhmm (AVX-512 path when available)"},
        "e2e": {"value": round(gcups, 3), "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---- our arm ----------------------------------------------------------------------------------

class RequestPool:
    """Every region of a batch as a request of its own (host structs built once): the serving legs
    draw each arriving request's region uniformly at random from it, i.e. from the batch's size
    distribution."""

    def __init__(self, batch, expected=None):
        self.regions = [batch.subset([g]) for g in range(batch.n_regions)]
        self.structs = [r.as_c() for r in self.regions]
        self.cells = [r.cells() for r in self.regions]
        self.sizes = [r.out_size for r in self.regions]
        # each region's likelihoods from the batched run, for checking every served request
        self.expected = None
        if expected is not None:
            offs = np.concatenate([[0], np.cumsum(self.sizes)])
            self.expected = [expected[offs[g]:offs[g + 1]] for g in range(batch.n_regions)]


def serving_latency(engine, pool: RequestPool, load: float, capacity_regions_per_s: float, seconds: float, seed: int):
    """Poisson arrivals at `load` x capacity, each request a region drawn at random from the pool;
    returns latency percentiles, the sustained GCUPS of the completed requests and the serving
    loop's own counters."""
    from rovaca_b200 import _lib

    lib = _lib.load()
    rng = np.random.default_rng(seed)
    structs, cells, sizes = pool.structs, pool.cells, pool.sizes
    rate = load * capacity_regions_per_s
    n_req = int(rate * seconds * 1.5) + 16
    gaps = rng.exponential(1.0 / rate, n_req)
    picks = rng.integers(0, len(structs), n_req)
    before = engine.server_stats()
    outs, tickets, done_cells = [], [], 0
    t0 = time.perf_counter()
    next_t = t0
    k = 0
    lag = 0.0  # how far submission fell behind the arrival schedule (host-side stalls)
    while next_t - t0 < seconds:
        now = time.perf_counter()
        if now < next_t:
            time.sleep(min(next_t - now, 0.002))
            continue
        lag = max(lag, now - next_t)
        g = int(picks[k % n_req])
        out = np.empty(sizes[g])
        t = C.c_uint64()
        rc = lib.phmm_submit(engine._h, C.byref(structs[g]), out.ctypes.data, None, C.byref(t))
        if rc != 0:
            raise RuntimeError(f"phmm_submit failed: {rc}")
        tickets.append((t.value, g))
        outs.append(out)
        next_t += gaps[k % len(gaps)]
        k += 1
    lat = []
    for t, g in tickets:
        _, total_us = engine.wait(t)
        lat.append(total_us / 1e3)
        done_cells += cells[g]
    elapsed = time.perf_counter() - t0
    after = engine.server_stats()
    lat = np.array(lat)
    batches = after["batches"] - before["batches"]
    # every served request's likelihoods against the same region's in the batched run (bit for bit:
    # a pair's arithmetic does not depend on what it was batched with)
    mismatched = None
    if pool.expected is not None:
        mismatched = sum(not np.array_equal(o, pool.expected[g], equal_nan=True)
                         for o, (_, g) in zip(outs, tickets))
    return {"load": load, "offered_regions_per_s": round(rate, 1), "requests": len(lat),
            "p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3),
            "sustained_gcups": round(done_cells / elapsed / 1e9, 2),
            "batches": batches,
            "mean_batch_regions": round((after["requests_done"] - before["requests_done"]) / max(batches, 1), 1),
            "mean_batch_ms": round((after["batch_ms"] - before["batch_ms"]) / max(batches, 1), 2),
            "mean_batch_device_ms": round((after["device_ms"] - before["device_ms"]) / max(batches, 1), 2),
            "max_batch_ms_so_far": round(after["max_batch_ms"], 2), "max_queue_ms_so_far": round(after["max_queue_ms"], 2),
            "max_submit_lag_ms": round(lag * 1e3, 2),
            "arena_grows": after["arena_grows"] - before["arena_grows"],
            "graph_captures": after["graph_captures"] - before["graph_captures"],
            "max_setup_ms_so_far": round(after["max_setup_ms"], 2), "max_host_ms_so_far": round(after["max_host_ms"], 2),
            "mean_phase_ms": {k: round((after[k + "_ms"] - before[k + "_ms"]) / max(batches, 1), 3)
                              for k in ("gather", "plan", "enqueue", "wait", "scatter")},
            "requests_differing_from_batched": mismatched}


def underflow_stress(engine, steps: int, warmup: int, cpu_threads: int | None, n_regions: int = 500) -> dict:
    """The underflow-stress configuration at its stated size (500 regions x 200 reads of 250 bp, base
    quality U[2,15], 5% errors, 16 haplotypes of 800-1,000 bp with 5-10 indels): FP64 rerun fraction,
    GCUPS resident and end to end, every pair's log10 error against the all-FP64 model, and (rank 0
    of a one-GPU run) every pair against the reference's own schedule_pairhmm on the host cores."""
    from rovaca_b200 import synth

    pb = synth.config2(n_regions, seed=2)
    cells = pb.cells()
    with engine.resident(pb, want_flags=True) as res:
        res.run(warmup)
        st = res.run(steps)
        out, flags = res.results()
        f64 = res.check_fp64()
    pinned = pb.pinned()
    e2e_out = np.empty(pb.out_size)
    engine.compute(pinned, out=e2e_out)
    t = time.perf_counter()
    engine.compute(pinned, out=e2e_out)
    e2e_s = time.perf_counter() - t
    rep_ = {"regions": n_regions, "pairs": int(pb.out_size), "cells": int(cells),
            "gcups_device": round(cells * steps / st["device_ms"] / 1e6, 1),
            "gcups_e2e": round(cells / e2e_s / 1e9, 1),
            "e2e_equal_resident": bool(np.array_equal(e2e_out, out, equal_nan=True)),
            "fp64_rerun_fraction": round(float(flags.mean()), 4),
            "abs_err_log10_vs_fp64": error_report(out, flags, f64),
            "quality_preprocessing": "vector-API semantics: raw qualities, no cap, PCR NONE"}
    if cpu_threads:
        # the reference runs this shape at a few GCUPS on the host (most pairs in FP64): a seeded
        # tenth of the regions, every pair of them
        ref_regions = min(50, n_regions)
        end = pb.out_offsets()[ref_regions]
        rep_["vs_reference"] = reference_whole_batch(pb.subset(list(range(ref_regions))), out[:end], flags[:end],
                                                     cpu_threads)
        rep_["vs_reference"]["regions"] = f"regions 0-{ref_regions - 1} of {n_regions}"
    return rep_


def wgs_mixture(engine, fraction: float, cpu_threads: int | None, sample: int = 200) -> dict:
    """A seeded share of the WGS-like mixture (depth lognormal, median 60, sigma 0.5, clipped to
    [5, 2000]; 150 bp reads (90%) or 250 bp; haplotypes geometric, mean 6, max 128, of 200-1,200 bp;
    2% of regions from the underflow-stress regime): batched GCUPS end to end from pinned buffers,
    the plain one-region-per-call form on a seeded sample of regions, the reference's AVX-512 host
    path on the same sample (host threads), and genotype concordance on that sample -- calls from the
    engine's likelihoods against calls from the reference's likelihoods (its schedule_pairhmm), both
    normalised and filtered and genotyped by the reference's own genotyping code, for a biallelic
    event (haplotype 0 against the rest) and a multi-allelic one (haplotype h to allele h mod 4)."""
    from oracle import GenotypeRef, Ref, ref_available
    from oracle import genotype as G
    from rovaca_b200 import synth

    pb = synth.make(4, scale=fraction, seed=4)
    pinned = pb.pinned()
    out = np.empty(pb.out_size)
    engine.compute(pinned, out=out)
    t = time.perf_counter()
    _, _, st = engine.compute(pinned, out=out)
    el = time.perf_counter() - t
    rng = np.random.default_rng(44)
    pick = sorted(int(g) for g in rng.choice(pb.n_regions, min(sample, pb.n_regions), replace=False))
    plain_regions = [pb.subset([g]).pinned() for g in pick]
    plain_cells = sum(r.cells() for r in plain_regions)
    for r in plain_regions[:5]:
        engine.compute(r)
    t = time.perf_counter()
    for r in plain_regions:
        engine.compute(r)
    plain_s = time.perf_counter() - t
    res = {"regions": int(pb.n_regions), "cells": int(st["cells"]), "share_of_200k_regions": fraction,
           "gcups_e2e": round(st["cells"] / el / 1e9, 1), "gcups_device": round(st["cells"] / st["device_ms"] / 1e6, 1),
           "fp64_pairs": int(st["pairs_f64"]), "pairs": int(st["pairs"]),
           "plain_gcups_e2e": round(plain_cells / plain_s / 1e9, 2),
           "sample_regions": len(pick), "sample_cells": int(plain_cells)}
    if not (cpu_threads and ref_available()):
        return res
    sub = pb.subset(pick)
    ref = Ref()
    offs = sub.out_offsets()
    want = np.empty(sub.out_size)

    def work(g):
        want[offs[g]:offs[g + 1]] = ref.schedule_region(sub, g, 0.02, 0.02).reshape(-1)

    t = time.perf_counter()
    with ThreadPoolExecutor(max_workers=cpu_threads, initializer=ref.init_thread) as ex:
        list(ex.map(work, range(sub.n_regions)))
    ref_s = time.perf_counter() - t
    full_offs = pb.out_offsets()
    got = np.concatenate([out[full_offs[g]:full_offs[g + 1]] for g in pick])
    gref = GenotypeRef()
    events = same = 0
    max_gl = 0.0
    read0 = np.concatenate([[0], np.cumsum(sub.n_reads.astype(np.int64))])
    read_len = np.diff(sub.read_off.astype(np.int64))
    for k, g in enumerate(pick):
        M, N = int(sub.n_haps[k]), int(sub.n_reads[k])
        lens = read_len[read0[k]:read0[k] + N].tolist()
        mine, keep_m = G.normalize_filter(got[offs[k]:offs[k + 1]].reshape(M, N), lens)
        theirs, keep_t = G.normalize_filter(want[offs[k]:offs[k + 1]].reshape(M, N), lens)
        km, kt = int(keep_m.sum()), int(keep_t.sum())
        for A, ha in ((min(2, M), [0] + [1] * (M - 1)), (min(4, M), [h % 4 for h in range(M)])):
            _, gl_m = gref.genotype(mine[:, :km], np.array(ha, np.int8), A)
            _, gl_t = gref.genotype(theirs[:, :kt], np.array(ha, np.int8), A)
            events += 1
            same += int(G.best_genotype(gl_m) == G.best_genotype(gl_t))
            if km == kt:
                max_gl = max(max_gl, float(np.max(np.abs(gl_m - gl_t))))
    d = np.abs(got - want)
    fin = np.isfinite(d)
    res.update({"reference_host_gcups": round(sub.cells() / ref_s / 1e9, 2), "reference_threads": cpu_threads,
                "reference_seconds": round(ref_s, 2),
                "max_abs_diff_vs_reference_on_sample": float(d[fin].max()) if fin.any() else 0.0,
                "genotype_events_checked": events, "genotype_calls_identical": same,
                "max_abs_gl_diff": max_gl,
                "concordance": "calls from the engine's and from the reference's likelihoods, normalised and filtered, "
                               "genotyped by the reference's own code (oracle/_ref/libgenotype_ref.so)"})
    return res


def genotyping_run(engine, n_regions: int = 400, cpu_threads: int | None = None) -> dict:
    """Region API with genotyping events on the GPU (read preparation, likelihoods, normalise and
    filter, allele marginalisation, diploid genotype likelihoods, calls): throughput through the
    serving loop; then every event checked twice -- the GPU's allele and genotype likelihoods against
    the reference's own genotyping code (compiled from its sources) on the GPU's normalised matrix,
    and the GPU's call against the call the reference makes from its own likelihoods (its
    schedule_pairhmm on the prepared reads, normalised and filtered, then its genotyping code) -- and
    the calls from all-FP64 likelihoods beside them."""
    from oracle import GenotypeRef, Ref, ref_available
    from oracle import genotype as G
    import ctypes as C

    from rovaca_b200 import _lib, synth
    from rovaca_b200.pairhmm import PackedBatch, Region

    regions = synth.genotyping_regions(n_regions, seed=21)
    cells = sum(sum(len(h) for h in r["haplotypes"]) * sum(len(x) for x in r["reads"]) for r in regions)
    for r in regions[:8]:
        engine.submit_region(r["haplotypes"], r["reads"], r["quals"], r["mapq"], 18, 3, events=r["events"],
                             want_matrix=False).wait()
    t = time.perf_counter()
    tickets = [engine.submit_region(r["haplotypes"], r["reads"], r["quals"], r["mapq"], 18, 3, events=r["events"],
                                    want_matrix=False) for r in regions]
    for tk in tickets:
        tk.wait()
    el = time.perf_counter() - t
    out = {"regions": n_regions, "events": int(sum(len(r["events"]) for r in regions)),
           "regions_per_s": round(n_regions / el, 1), "gcups": round(cells / el / 1e9, 2),
           "form": "phmm_submit_region with events, genotype likelihoods only back to the host (PCR CONSERVATIVE, Q18)"}

    # the same regions again with the normalised matrix and allele likelihoods back
    full = [engine.submit_region(r["haplotypes"], r["reads"], r["quals"], r["mapq"], 18, 3, events=r["events"],
                                 want_allele_lk=True) for r in regions]
    lib = _lib.load()
    prepared = []
    for r in regions:
        qs, gops = [], []
        for rd, q, mq in zip(r["reads"], r["quals"], r["mapq"]):
            n = len(rd)
            qq = (C.c_uint8 * n)()
            lib.phmm_host_prepare_quals(q, n, int(mq), 18, qq)
            gop = (C.c_uint8 * n)(*([45] * n))
            lib.phmm_host_pcr_model(rd, n, gop, 3)
            qs.append(bytes(qq))
            gops.append(bytes(gop))
        prepared.append(Region(r["haplotypes"], r["reads"], qs, gops, gops, [bytes([10]) * len(x) for x in r["reads"]]))
    pb = PackedBatch.from_regions(prepared)
    offs = pb.out_offsets()
    with engine.resident(pb) as res:
        lk64_all = res.check_fp64()
    if not ref_available():
        out["reference"] = "unavailable (oracle/_ref not built)"
        return out
    gref = GenotypeRef()
    ref = Ref()
    lk_ref_all = np.empty(pb.out_size)

    def work(g):
        lk_ref_all[offs[g]:offs[g + 1]] = ref.schedule_region(pb, g, 0.02, 0.02).reshape(-1)

    with ThreadPoolExecutor(max_workers=cpu_threads or (os.cpu_count() or 1), initializer=ref.init_thread) as ex:
        list(ex.map(work, range(pb.n_regions)))
    total = gl_equal = alk_equal = calls_ref = calls_64 = truth_hits = keep_equal = 0
    max_gl_vs_ref_lk, max_tie = 0.0, 0.0
    for g, (r, tk) in enumerate(zip(regions, full)):
        mat, keep = tk.wait()
        got = tk.genotypes()
        M, N = len(r["haplotypes"]), len(r["reads"])
        K = int(keep.sum())
        lens = [len(x) for x in r["reads"]]
        norm_ref, keep_ref = G.normalize_filter(lk_ref_all[offs[g]:offs[g + 1]].reshape(M, N), lens)
        norm64, keep64 = G.normalize_filter(lk64_all[offs[g]:offs[g + 1]].reshape(M, N), lens)
        K64 = int(keep64.sum())
        keep_equal += int(np.array_equal(keep_ref, keep.astype(bool)))
        K_ref = int(keep_ref.sum())
        for (A, ha), (gl, best, alk), truth in zip(r["events"], got, r["truth"]):
            total += 1
            ralk, rgl = gref.genotype(mat[:, :K], ha, A)
            alk_equal += int(np.array_equal(alk[:, :K], ralk, equal_nan=True))
            gl_equal += int(np.array_equal(gl, rgl, equal_nan=True))
            _, gl_r = gref.genotype(norm_ref[:, :K_ref], ha, A)
            calls_ref += int(best == G.best_genotype(gl_r))
            max_gl_vs_ref_lk = max(max_gl_vs_ref_lk, float(np.max(np.abs(gl - gl_r))))
            _, gl64 = gref.genotype(norm64[:, :K64], ha, A)
            b64 = G.best_genotype(gl64)
            calls_64 += int(best == b64)
            if best != b64:
                max_tie = max(max_tie, abs(float(gl64[best] - gl64[b64])))
            truth_hits += int(best == truth)
    out.update({"checked_events": total,
                "gl_bit_equal_to_reference_genotyping_on_gpu_matrix": gl_equal,
                "allele_lk_bit_equal_to_reference_marginalisation": alk_equal,
                "regions_with_kept_reads_equal_to_reference_likelihoods": keep_equal,
                "calls_identical_to_reference_likelihoods_and_genotyping": calls_ref,
                "max_abs_gl_diff_vs_reference_likelihoods": max_gl_vs_ref_lk,
                "calls_identical_to_fp64_likelihoods": calls_64,
                "max_fp64_gl_gap_where_calls_differ": max_tie, "calls_equal_truth": truth_hits,
                "reference": "schedule_pairhmm (oracle/_ref/libphmm_ref.so) on the prepared reads, normalise/filter "
                             "restated (pinned to pairhmm_internal.cpp by the host tests), AlleleLikelihoods::marginalize "
                             "and GenotypeLikelihoodCalculator (oracle/_ref/libgenotype_ref.so)"})
    return out


def smith_waterman_run(engine, batch, steps: int, warmup: int, cpu: bool) -> dict:
    """Smith-Waterman realignment of every read of the batch against a haplotype of its own region
    (the aligner HaplotypeCaller runs per read after genotyping; genotyping parameters, the
    reference's int16/int32 choice): cell updates per second with the batch resident in HBM, end to
    end through phmm_sw_align from host buffers, results checked against the oracle on a sample, and
    the reference's own aligner on the host cores for a bounded sample."""
    from oracle import SwOracle, SwRef, build_ref_sw
    from rovaca_b200 import sw, synth

    b = synth.sw_realignment(batch)
    with engine.sw_resident(b) as rs:
        rs.run(warmup)
        ms = rs.run(steps)
        cls = rs.profile()
        res = rs.results()
    engine.sw_align(b)
    t = time.perf_counter()
    e2e_res = engine.sw_align(b)
    e2e_s = time.perf_counter() - t
    same = bool(np.array_equal(e2e_res.fields, res.fields) and np.array_equal(e2e_res.cigars, res.cigars))
    orc = SwOracle()
    rng = np.random.default_rng(7)
    sample = rng.choice(b.n, min(2000, b.n), replace=False)
    mism = sum(res.tuple(int(q)) != orc.align(*b.pair(int(q))) for q in sample)
    # bytes of 4-bit cell codes written per run (the per-warp scratch the trace-back reads)
    k_of = np.array(sw.CLASS_K[:-1])
    rl = b.items["read_len"].astype(np.int64)
    hl = b.items["hap_len"].astype(np.int64)
    kk = k_of[np.minimum(np.searchsorted(k_of, np.maximum((rl + 31) // 32, 1)), len(k_of) - 1)]
    stripes = np.maximum((rl + 32 * kk - 1) // (32 * kk), 1)
    code_bytes = int((stripes * hl * 128 * ((kk + 7) // 8)).sum())
    out = {"alignments": b.n, "cells": b.cells, "gcups_device": round(b.cells / ms / 1e6, 1),
           "ms_per_run": round(ms, 3), "gcups_e2e": round(b.cells / e2e_s / 1e9, 1),
           "e2e_ms": round(e2e_s * 1e3, 3), "e2e_equal_resident": same,
           "h2d_bytes": int(b.items.nbytes + b.hap_bases.size + b.read_bases.size + 12 * b.n),
           "d2h_bytes": int(24 * b.n + 4 * res.cigars.size),
           "class_ms": {str(k): round(float(v), 3) for k, v in zip(list(k_of) + ["wrap"], cls) if v > 0},
           "oracle_sample": int(len(sample)), "oracle_mismatches": int(mism),
           "cell_code_bytes_per_run": code_bytes,
           "cell_code_gbs": round(code_bytes / (ms / 1e3) / 1e9, 1),
           "workload": "every read of the 2,000-region batch against haplotype (read index mod haplotypes) of "
                       "its region; genotyping parameters (10, -15, -30, -5)"}
    if cpu and build_ref_sw() is not None:
        ref = SwRef()
        pairs = [b.pair(int(q)) for q in sample]
        cells = sum(len(h) * len(r) for h, r in pairs)
        th = os.cpu_count() or 1
        t = time.perf_counter()
        with ThreadPoolExecutor(th) as ex:
            outs = list(ex.map(lambda pr: ref.align(pr[0], pr[1]), pairs))
        dt = time.perf_counter() - t
        out["cpu_baseline"] = {"value": round(cells / dt / 1e9, 2), "unit": "GCUPS", "cores": th, "kind": "reference",
                               "sample": f"{len(pairs)} alignments of the batch ({dt:.2f} s), the reference's "
                                         "ro_sw aligner compiled from its sources, one alignment per task",
                               "mismatches_vs_gpu": int(sum(o != res.tuple(int(q)) for o, q in zip(outs, sample)))}
    return out


def run_resident_only(args) -> None:
    """Profiling mode: only the device-resident replay (the launches the ncu summaries cover)."""
    import torch

    from rovaca_b200 import Engine, synth

    torch.cuda.set_device(0)
    batch = synth.config1(n_regions=args.regions, seed=1)
    with Engine(device=0, use_cuda_graph=not args.no_graph, autotune=not args.no_autotune) as engine:
        with engine.resident(batch) as res:
            res.run(args.warmup)
            st = res.run(args.steps)
    print(json.dumps({"mode": "resident", "regions": args.regions, "graph": not args.no_graph, "steps": args.steps,
                      "ms_per_step": st["device_ms"] / args.steps, "fp32_pass_ms": st["fp32_ms"],
                      "fp64_pass_ms": st["fp64_ms"], "gcups": batch.cells() * args.steps / st["device_ms"] / 1e6,
                      "kernel_launches": st["kernel_launches"]}), flush=True)


def run_sw_only(args) -> None:
    """Profiling mode: the resident Smith-Waterman realignment of the reads of 500 regions of the
    benchmark's shape (about 125,000 alignments), warm-up and timed runs only."""
    import torch

    from rovaca_b200 import Engine, synth

    torch.cuda.set_device(0)
    b = synth.sw_realignment(synth.config1(n_regions=500, seed=1))
    with Engine(device=0, autotune=False) as engine:
        with engine.sw_resident(b) as rs:
            rs.run(args.warmup)
            ms = rs.run(args.steps)
    print(json.dumps({"mode": "sw", "alignments": b.n, "cells": b.cells, "steps": args.steps, "ms_per_run": ms,
                      "gcups": b.cells / ms / 1e6}), flush=True)


def run_ours(args, rank: int, world: int, dist) -> None:
    import torch

    from rovaca_b200 import Engine, synth

    device = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(device)
    batch = synth.config1(seed=shard_seed(rank))
    cells = batch.cells()
    engine = Engine(device=device, use_cuda_graph=not args.no_graph)
    dev = f"cuda:{device}"

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        return rank_reduce(dist, x, "max", dev)

    # device-resident batched throughput
    res = engine.resident(batch, want_flags=True)
    res.run(args.warmup)
    barrier()
    with ClockSampler(device) as clk:
        st = res.run(args.steps)
        barrier()
    value, ms_per_step = weak_scaling_value(dist, float(cells), args.steps, st["device_ms"], dev)
    total_cells = value * ms_per_step * args.steps * 1e6
    fp32_pass_ms = max_over_ranks(st["fp32_ms"])
    strong = None
    if world > 1:
        # strong scaling: one 2,000-region batch (the same seed on every rank) split across the ranks
        shared = batch if rank == 0 else synth.config1(seed=shard_seed(0))
        mine = shared.subset(strong_scaling_regions(shared, rank, world))
        with engine.resident(mine) as rs:
            rs.run(args.warmup)
            barrier()
            sst = rs.run(args.steps)
            barrier()
        s_ms = max_over_ranks(sst["device_ms"])
        strong = {"value": round(shared.cells() * args.steps / (s_ms / 1e3) / 1e9, 2), "unit": "GCUPS",
                  "ms_per_step": round(s_ms / args.steps, 3), "cells_per_step": int(shared.cells()),
                  "split": "regions of one 2,000-region batch by phmm_partition_regions (cells per rank balanced)"}
    out, flags = res.results()
    # every kernel class alone, after the timed region (CUDA events around each launch)
    prof = res.profile()
    # every pair again with the all-FP64 model, for the error of every likelihood
    f64_all = res.check_fp64()
    res.close()
    accuracy = error_report(out, flags, f64_all)
    f64_frac = float(flags.mean())
    launches = int(st["kernel_launches"])

    # end to end through the public API, pinned host buffers
    pinned = batch.pinned()
    out_e2e = np.empty(batch.out_size)
    for _ in range(args.warmup):
        engine.compute(pinned, out=out_e2e)
    barrier()
    with ClockSampler(device) as clk_e2e:
        t = time.perf_counter()
        for _ in range(args.steps):
            engine.compute(pinned, out=out_e2e)
        barrier()
        e2e_s = max_over_ranks(time.perf_counter() - t)
    e2e = total_cells / e2e_s / 1e9
    same = bool(np.array_equal(out_e2e, out))
    h2d = int(batch.read_bases.size * 5 + batch.hap_bases.size + batch.read_off.nbytes + batch.hap_off.nbytes +
              batch.n_haps.nbytes + batch.n_reads.nbytes)
    d2h = int(batch.out_size * 8)

    line = None
    if rank == 0:
        # plain: one region per call, on a sample of regions
        plain_regions = [pinned.subset([g]).pinned() for g in range(200)]
        plain_cells = sum(r.cells() for r in plain_regions)
        for r in plain_regions[:10]:
            engine.compute(r)
        torch.cuda.synchronize()
        t = time.perf_counter()
        plain_dev_ms = 0.0
        for r in plain_regions:
            _, _, s = engine.compute(r)
            plain_dev_ms += s["device_ms"]
        plain_s = time.perf_counter() - t
        plain = plain_cells / plain_s / 1e9
        plain_dev = plain_cells / (plain_dev_ms / 1e3) / 1e9

        # every pair against the reference's own schedule_pairhmm on the host cores (one GPU only:
        # the host is shared by all ranks otherwise)
        from oracle import Oracle, ref_available

        orc = Oracle()
        cores = os.cpu_count() or 1
        vs_ref = reference_whole_batch(batch, out, flags, cores) if world == 1 and ref_available() else None

        # serving loop latency (after a warm-up burst: slots sized, graphs captured, kernels loaded)
        cap = batch.n_regions / (e2e_s / args.steps)
        pool = RequestPool(batch, out)
        serving_latency(engine, pool, 2.0, cap, 1.0, seed=99)
        lat = [serving_latency(engine, pool, load, cap, args.serve_seconds, seed=100 + k)
               for k, load in enumerate((0.25, 0.5, 0.8, 0.95))]
        stress = underflow_stress(engine, args.steps, args.warmup, cores if world == 1 and ref_available() else None)
        wgs = wgs_mixture(engine, args.wgs_fraction, cores if world == 1 and ref_available() else None)
        geno = genotyping_run(engine, cpu_threads=cores)
        swr = smith_waterman_run(engine, batch, args.steps, args.warmup, world == 1)

        # roofline of the FP32 wavefront pass against the measured FP32 FMA peak
        peak_scalar, peak_packed = engine.fp32_fma_peak()
        peak = max(peak_scalar, peak_packed)
        n32 = 39
        cms, ccells = prof["class_ms"], prof["class_cells"].astype(np.float64)
        dom = int(np.argmax(cms[:n32]))
        achieved = ccells[dom] * FLOP_PER_CELL / (float(cms[dom]) / 1e3) / 1e12
        fp32_serial_ms = float(cms[:n32].sum())
        fp64_serial_ms = float(cms[n32:].sum())
        pass_achieved = float(ccells[:n32].sum()) * FLOP_PER_CELL / (fp32_serial_ms / 1e3) / 1e12
        mode_names = ["inter, constant gap qualities", "inter, per-row gap qualities", "intra"]
        shape = dom % 13
        kh, multi = (shape + 1, False) if shape < 8 else (shape - 4, True)
        dom_name = (f"fwd_f32 class {dom}: {mode_names[dom // 13]}, {kh} row pairs per lane"
                    f"{', multi-stripe' if multi else ''}")
        traffic = traffic_from_profiles(dom)

        # CPU baseline: the reference's own PairHMM on all host cores, bounded sample
        cpu = None
        if world == 1:
            if ref_available():
                sample_regions = list(range(64))
                reference_gcups(batch, sample_regions[:4], cores)
                g, dt = reference_gcups(batch, sample_regions, cores)
                g1, dt1 = reference_gcups(batch, sample_regions[:4], 1)
                cpu = {"value": round(g, 3), "unit": "GCUPS", "cores": cores, "kind": "reference",
                       "sample": f"regions 0-63 of the batch ({dt:.1f} s), one region per thread, reference "
                                 "schedule_pairhmm AVX path compiled from its sources",
                       "single_core": {"value": round(g1, 3), "sample": f"regions 0-3 on one thread ({dt1:.1f} s)"}}
            else:
                t = time.perf_counter()
                sub = batch.subset([0, 1, 2, 3])
                orc.batch(sub)
                dt = time.perf_counter() - t
                cpu = {"value": round(sub.cells() / dt / 1e9, 3), "unit": "GCUPS", "cores": 1, "kind": "port",
                       "sample": "regions 0-3 through the scalar oracle (reference build unavailable)"}

        clocks = clk.summary()
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "GCUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 recompute)",
            "data": "synthetic (seeded generator, one 2,000-region batch per rank)",
            "config": {"workload": WORKLOAD, "regions": batch.n_regions, "pairs": int(batch.out_size),
                       "cells_per_rank": int(cells), "l2": "inputs (~540 MB) larger than the 126 MB L2; no flush",
                       "quality_preprocessing": "vector-API semantics (schedule_pairhmm): raw qualities, no cap, "
                                                "PCR NONE; the genotyping leg uses the region API (Q18, PCR CONSERVATIVE)",
                       "parallelism": f"regions sharded per rank x{world}, no collective"},
            "e2e": {"value": round(e2e, 2), "unit": "GCUPS", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": round(1e3 * e2e_s / args.steps, 3), "results_identical_to_resident": same,
                    "batched_vs_plain": round(e2e / plain, 2), "plain_gcups": round(plain, 2),
                    "p50_p99_region_latency_ms_at_80pct_load": [next(x for x in lat if x["load"] == 0.8)["p50_ms"],
                                                                next(x for x in lat if x["load"] == 0.8)["p99_ms"]],
                    "max_abs_log10_err_vs_fp64_every_pair": accuracy["max"],
                    "pairs_checked_vs_fp64": accuracy["pairs"],
                    "max_abs_diff_vs_reference_every_pair": vs_ref["max_abs_diff"] if vs_ref else None,
                    "fp64_flag_disagreements_vs_reference": vs_ref["fp64_flag_disagreements"] if vs_ref else None},
            "gpu_launches": launches,
            "roofline": {"bound": "fp32", "achieved": round(achieved, 2), "peak": round(peak, 2), "unit": "TFLOP/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "kernel": dom_name + " (the longest-running kernel), 12 FLOP per cell of its work "
                                   "items, timed alone with CUDA events after the timed region",
                         "kernel_ms": round(float(cms[dom]), 3), "kernel_share_of_serial_fp32": round(
                             float(cms[dom]) / fp32_serial_ms, 3),
                         "fp32_pass_alone": {"ms": round(fp32_serial_ms, 3), "tflops": round(pass_achieved, 2),
                                             "frac": round(pass_achieved / peak, 4)},
                         "fp64_pass_alone_ms": round(fp64_serial_ms, 3),
                         "peak_source": "measured FP32 FMA throughput, max of scalar FFMA and packed FFMA2 "
                                        "(phmm_fp32_fma_peak, 2 FLOP per FMA)",
                         "peak_scalar_ffma": round(peak_scalar, 2), "peak_packed_ffma2": round(peak_packed, 2)},
            "cpu_baseline": cpu,
            "clocks": clocks,
            "clocks_e2e": clk_e2e.summary(),
            "plain": {"gcups_e2e": round(plain, 2), "gcups_device": round(plain_dev, 2), "regions": len(plain_regions),
                      "form": "one region per phmm_compute_regions call"},
            "batched_vs_plain": {"e2e": round(e2e / plain, 2), "device": round(value / world / plain_dev, 2)},
            "fp32_pass_ms": round(fp32_pass_ms, 3),
            "strong_scaling": strong,
            "fp64_rerun_fraction": round(f64_frac, 5),
            "accuracy_vs_fp64": accuracy,
            "vs_reference_every_pair": vs_ref,
            "latency": next(x for x in lat if x["load"] == 0.8),
            "latency_by_load": lat,
            "underflow_stress": stress,
            "wgs_mixture": wgs,
            "genotyping": geno,
            "smith_waterman": swr,
        }
    engine.close()
    if line is not None:
        print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--serve-seconds", type=float, default=6.0)
    ap.add_argument("--wgs-fraction", type=float, default=0.1,
                    help="share of the 200,000-region WGS-like mixture run in its leg (1.0: all of it)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="default tile shapes (profiling runs: no calibration launches before the batch)")
    ap.add_argument("--only", choices=["all", "resident", "sw"], default="all",
                    help="resident: only the device-resident replay (for profiling); sw: only the resident "
                         "Smith-Waterman realignment of a 500-region batch's reads (for profiling)")
    ap.add_argument("--no-graph", action="store_true", help="direct launches instead of CUDA-graph replay")
    ap.add_argument("--regions", type=int, default=2000,
                    help="--only resident: regions of the batch (a smaller batch of the same shape for profiling)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    try:
        if args.only == "resident":
            run_resident_only(args)
        elif args.only == "sw":
            run_sw_only(args)
        elif args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_ours(args, rank, world, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
