"""CPU-only checks of the engine library: it loads, exports every declared entry point, refuses to
run without a GPU, and its host-side logic (planning, read preparation, PCR model, post-processing)
matches the reference."""
from __future__ import annotations

import ctypes as C
import json
import multiprocessing as mp

import numpy as np
import pytest

from conftest import GOLDEN
from rovaca_b200 import _lib
from rovaca_b200.pairhmm import PackedBatch, Region, class32, class64, default_tiles, plan_summary


def _region(haps, reads, q=30, ins=45, gcp=10):
    return Region(haps, reads, [bytes([q]) * len(r) for r in reads], [bytes([ins]) * len(r) for r in reads],
                  [bytes([ins]) * len(r) for r in reads], [bytes([gcp]) * len(r) for r in reads])


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = _lib.declared_symbols()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n


def test_ctypes_mirrors_match_the_c_header_layout(tmp_path):
    """Every public struct of include/phmm_b200.h has the size and the field offsets (in declaration
    order) of its ctypes mirror in rovaca_b200/_lib.py: tests/native/abi_layout.c prints them as
    the C compiler lays them out."""
    import shutil
    import subprocess
    from pathlib import Path

    cc = shutil.which("gcc")
    if cc is None:
        pytest.skip("gcc not available")
    exe = tmp_path / "abi_layout"
    src = Path(__file__).resolve().parent / "native" / "abi_layout.c"
    subprocess.run([cc, "-std=c11", "-Wall", "-Wextra", "-Werror", str(src), "-o", str(exe)], check=True)
    sizes, fields = {}, {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        kind, name, value = line.split()
        if kind == "struct":
            sizes[name] = int(value)
        else:
            fields.setdefault(name.split(".")[0], []).append(int(value))
    mirrors = {"phmm_config": _lib.Config, "phmm_batch": _lib.Batch, "phmm_stats": _lib.Stats,
               "phmm_tile_table": _lib.TileTable, "phmm_tune_entry": _lib.TuneEntry,
               "phmm_tune_report": _lib.TuneReport, "phmm_region_input": _lib.RegionInput,
               "phmm_region_events": _lib.RegionEvents, "phmm_region_realign": _lib.RegionRealign,
               "phmm_server_stats": _lib.ServerStats, "phmm_sw_item": _lib.SwItem, "phmm_sw_result": _lib.SwResult}
    assert set(mirrors) == set(sizes)
    for name, cls in mirrors.items():
        assert C.sizeof(cls) == sizes[name], name
        assert [getattr(cls, f[0]).offset for f in cls._fields_] == fields[name], name


def test_status_strings_and_version():
    lib = _lib.load()
    for s in range(12):
        assert lib.phmm_status_string(s)
    assert b"sm_100a" in lib.phmm_version()


def _create_engine_without_gpu(q):
    try:
        from rovaca_b200 import Engine

        Engine()
        q.put("created")
    except _lib.PhmmError as e:
        q.put(e.name)


def test_engine_refuses_to_run_without_a_gpu():
    """No CUDA device: engine creation fails loudly (no CPU fallback exists)."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_create_engine_without_gpu, args=(q,))
    p.start()
    p.join(120)
    assert q.get(timeout=5) == "PHMM_ERR_NO_DEVICE"


# ---- planning -------------------------------------------------------------------------------

def cls(variant, kh, multi=False, uniform=True):
    """FP32 kernel class: mode (0 inter with constant gap qualities, 1 inter per-row, 2 intra) x 13
    shapes (single stripe KH 1..8, multi-stripe KH 4..8)."""
    mode = 2 if variant else (0 if uniform else 1)
    return class32(mode, kh, multi)


def cls64(variant, kh, multi=False, uniform=True):
    mode = 2 if variant else (0 if uniform else 1)
    return mode * 9 + (8 if multi else kh - 1)


def test_plan_rows_per_lane_follow_read_length():
    hap = b"ACGT" * 100
    reads = [hap[:n] for n in (1, 32, 33, 64, 100, 151, 200, 256)]
    s = plan_summary(PackedBatch.from_regions([_region([hap, hap[3:]], reads)]))
    # KH = ceil(R / 32) row pairs per lane; reads of equal KH share an item (two reads per warp)
    want = {1: 1, 2: 1, 4: 1, 5: 1, 7: 1, 8: 1}
    for k, n in want.items():
        assert s["class_items"][cls(0, k)] == n, (k, s["class_items"])
    assert s["class_items"].sum() == 6
    assert s["class_pairs"][cls64(0, 1)] == 4 and s["class_pairs"][cls64(0, 8)] == 2
    assert s["pairs"] == 16
    assert s["cells"] == sum(len(r) for r in reads) * (len(hap) + len(hap) - 3)


def test_plan_long_reads_use_multi_stripe_class():
    hap = b"ACGT" * 300
    s = plan_summary(PackedBatch.from_regions([_region([hap], [hap[:257], hap[:768], hap[:256]])]))
    assert s["class_items"][cls(0, 8, True)] == 2
    assert s["class_items"][cls(0, 8)] == 1


def test_plan_routes_n_pairs_to_the_intra_variant():
    h = b"ACGTACGGTCA" * 10
    hn = h[:20] + b"N" + h[21:]
    r = [h[5:60], h[10:40] + b"N" + h[41:70], h[:30]]
    s = plan_summary(PackedBatch.from_regions([_region([h, hn, h], r)]))
    # read with N: every pair intra; reads without N: the N haplotype alone is intra
    assert s["class_pairs"][18:].sum() == 3 + 2
    assert s["class_pairs"][:18].sum() == 2 * 2
    # each read without N streams [h] and [h] as two inter items split around the N haplotype
    assert s["class_items"][:26].sum() == 4
    assert s["class_items"][26:].sum() == 3


def test_plan_splits_long_haplotype_streams():
    haps = [b"A" * 1500] * 20  # 30,000 columns, more than one stream (8192 max)
    s = plan_summary(PackedBatch.from_regions([_region(haps, [b"A" * 100])]))
    assert s["class_items"][cls(0, 4)] == 4  # 5 haplotypes (7500 columns) per item
    assert s["pairs"] == 20


def test_plan_pairs_reads_and_gap_modes():
    hap = b"ACGT" * 60
    reads = [hap[k:k + 150] for k in range(5)]  # five reads of KH 5: items of 2 + 2 + 1
    reg = _region([hap], reads)
    s = plan_summary(PackedBatch.from_regions([reg]))
    assert s["class_items"][cls(0, 5)] == 3 and s["pairs"] == 5
    # varying gap-open qualities along a read select the per-row class
    reg.insertion_qualities[0] = bytes([45] * 149 + [40])
    s = plan_summary(PackedBatch.from_regions([reg]))
    assert s["class_items"][cls(0, 5, uniform=False)] == 1
    assert s["class_items"][cls(0, 5)] == 2
    # constant along the read but insertion != deletion: mode 0 shares M * mx between I and D
    # (mx == my), so such a read runs in the per-row class too; equal as quality & 127 is equal
    reg.insertion_qualities[0] = bytes([40] * 150)
    reg.insertion_qualities[1] = bytes([45 + 128] * 150)
    s = plan_summary(PackedBatch.from_regions([reg]))
    assert s["class_items"][cls(0, 5, uniform=False)] == 1
    assert s["class_items"][cls(0, 5)] == 2


def test_tile_table_shapes_route_reads():
    """A tile table moves a read-length bucket to a multi-stripe shape; FP64 classes follow the read
    length whatever the FP32 shape; invalid shapes are rejected."""
    hap = b"ACGT" * 100
    reads = [hap[:200], hap[:210], hap[:240], hap[:100]]  # buckets 7, 7, 8, 4
    pb = PackedBatch.from_regions([_region([hap, hap[5:]], reads)])
    d = plan_summary(pb)
    assert d["class_items"][cls(0, 7)] == 1 and d["class_items"][cls(0, 8)] == 1 and d["class_items"][cls(0, 4)] == 1
    kh, mu = default_tiles().as_arrays()
    assert list(kh[0, :10]) == [1, 2, 3, 4, 5, 6, 7, 8, 8, 8] and list(mu[0, :10]) == [0] * 8 + [1, 1]
    kh[0, 6], mu[0, 6] = 4, 1  # bucket 7 (193-224 rows): two 128-row stripes
    kh[0, 7], mu[0, 7] = 5, 1  # bucket 8 (225-256 rows): two 160-row stripes
    s = plan_summary(pb, _lib.TileTable.from_arrays(kh, mu))
    assert s["class_items"][cls(0, 4, True)] == 1 and s["class_items"][cls(0, 5, True)] == 1
    assert s["class_items"][cls(0, 4)] == 1 and s["class_items"].sum() == 3
    assert np.array_equal(s["class_pairs"], d["class_pairs"])
    assert s["class_pairs"][class64(0, 200)] == 4 and s["class_pairs"][class64(0, 240)] == 2
    assert s["cells"] == d["cells"] and s["pairs"] == d["pairs"]
    for b, k, m in ((6, 7, 1), (6, 6, 0), (3, 3, 1)):  # multi needs 4 <= KH < bucket, single KH >= bucket
        kh2, mu2 = default_tiles().as_arrays()
        kh2[0, b], mu2[0, b] = k, m
        with pytest.raises(_lib.PhmmError) as e:
            plan_summary(pb, _lib.TileTable.from_arrays(kh2, mu2))
        assert e.value.name == "PHMM_ERR_INVALID_ARGUMENT"


def test_plan_skips_empty_reads_and_haplotypes():
    s = plan_summary(PackedBatch.from_regions([_region([b"ACGT" * 10, b"", b"ACG"], [b"ACGT", b"", b"A" * 40])]))
    assert s["pairs"] == 4  # 2 non-empty haplotypes x 2 non-empty reads


def test_plan_rejects_regions_beyond_the_reference_limits():
    ok = b"ACGT"
    with pytest.raises(_lib.PhmmError) as e:
        plan_summary(PackedBatch.from_regions([_region([b"A" * 1537], [ok])]))
    assert e.value.name == "PHMM_ERR_LIMIT_EXCEEDED"
    with pytest.raises(_lib.PhmmError) as e:
        plan_summary(PackedBatch.from_regions([_region([ok], [b"A" * 769])]))
    assert e.value.name == "PHMM_ERR_LIMIT_EXCEEDED"
    with pytest.raises(_lib.PhmmError) as e:
        plan_summary(PackedBatch.from_regions([_region([ok] * 4097, [ok])]))
    assert e.value.name == "PHMM_ERR_LIMIT_EXCEEDED"
    plan_summary(PackedBatch.from_regions([_region([b"A" * 1536] * 2, [b"A" * 768])]))


def test_plan_rejects_bad_offsets():
    pb = PackedBatch.from_regions([_region([b"ACGT", b"ACG"], [b"AC"])])
    pb.hap_off = np.array([0, 4, 2], np.uint64)
    with pytest.raises(_lib.PhmmError) as e:
        plan_summary(pb)
    assert e.value.name == "PHMM_ERR_INVALID_ARGUMENT"


# ---- region-path host helpers ---------------------------------------------------------------

def test_pcr_model_and_repeats_match_reference_fixture():
    lib = _lib.load()
    data = json.loads((GOLDEN / "region_helpers.json").read_text())["reads"]
    assert len(data) >= 100
    for rec in data:
        s = rec["bases"].encode()
        n = len(s)
        got = [lib.phmm_host_tandem_repeat_length(s, n, o) for o in range(max(n - 1, 0))]
        assert got == rec["repeat"], rec["bases"]
        for model, name in ((1, "HOSTILE"), (2, "AGGRESSIVE"), (3, "CONSERVATIVE")):
            g = (C.c_uint8 * n)(*([45] * n))
            lib.phmm_host_pcr_model(s, n, g, model)
            assert list(bytes(g)) == rec[name], (name, rec["bases"])


def test_pcr_model_matches_reference_build_on_random_reads(ref):
    lib = _lib.load()
    ref.lib.ref_tandem_repeat.restype = C.c_int
    rng = np.random.default_rng(3)
    for t in range(300):
        n = int(rng.integers(2, 120))
        unit = rng.choice(list(b"ACGT"), int(rng.integers(1, 9)))
        s = bytes(np.asarray(np.resize(unit, n) if t % 2 else rng.choice(list(b"ACGT"), n), np.uint8))
        for o in range(n - 1):
            assert lib.phmm_host_tandem_repeat_length(s, n, o) == ref.lib.ref_tandem_repeat(s, n, o, 1)
        for model in (1, 2, 3):
            g1 = (C.c_uint8 * n)(*([45] * n))
            g2 = (C.c_uint8 * n)(*([45] * n))
            lib.phmm_host_pcr_model(s, n, g1, model)
            ref.lib.ref_pcr_model(s, n, g2, model, 1)
            assert bytes(g1) == bytes(g2)


def test_quality_preparation():
    lib = _lib.load()
    q = np.array([2, 5, 17, 18, 30, 45, 60], np.uint8)
    out = np.empty_like(q)
    lib.phmm_host_prepare_quals(q.ctypes.data_as(C.c_void_p), len(q), 40, 18, out.ctypes.data_as(C.c_void_p))
    assert out.tolist() == [6, 6, 6, 18, 30, 40, 40]


def _normalize_filter_expected(lk_hr, read_len):
    """normalize_likelihoods + collect_poorly_modelled_indices + transpose (pairhmm_internal.cpp:23-44,
    248-258,499-508), written out plainly."""
    n_haps, n_reads = lk_hr.shape
    out = np.full_like(lk_hr, np.nan)
    keep = []
    for r in range(n_reads):
        row = lk_hr[:, r].copy()
        best = row[0]
        for v in row[1:]:
            if best < v:
                best = v
        cmp = best - 4.5
        row = np.where(row < cmp, cmp, row)
        finite = row[~np.isnan(row)]
        b = finite.max() if finite.size else -np.inf
        if b < min(2.0, np.ceil(read_len[r] * 0.02)) * -4.0:
            keep.append(False)
        else:
            keep.append(True)
            out[:, sum(keep) - 1] = row
    return out, np.array(keep)


def test_normalize_and_filter_matches_restatement():
    lib = _lib.load()
    rng = np.random.default_rng(8)
    for t in range(200):
        nh, nr = int(rng.integers(1, 7)), int(rng.integers(1, 9))
        lk = -rng.random((nh, nr)) * 30
        if t % 5 == 0:
            lk[int(rng.integers(0, nh)), int(rng.integers(0, nr))] = np.nan
        rl = rng.integers(0, 300, nr).astype(np.uint64)
        out = np.empty_like(lk)
        keep = np.empty(nr, np.uint8)
        nk = C.c_uint32()
        lk_c = np.ascontiguousarray(lk)
        lib.phmm_host_normalize_filter(lk_c.ctypes.data_as(C.c_void_p), nh, nr, rl.ctypes.data_as(C.c_void_p),
                                       out.ctypes.data_as(C.c_void_p), keep.ctypes.data_as(C.c_void_p), C.byref(nk))
        want, wkeep = _normalize_filter_expected(lk, rl)
        assert np.array_equal(keep.astype(bool), wkeep)
        assert nk.value == wkeep.sum()
        assert np.array_equal(np.isnan(out), np.isnan(want))
        assert np.array_equal(out[~np.isnan(out)], want[~np.isnan(want)])


def test_normalize_matches_reference_build(ref):
    lib = _lib.load()
    rng = np.random.default_rng(9)
    for t in range(100):
        nh, nr = int(rng.integers(1, 7)), int(rng.integers(1, 9))
        lk_rh = -rng.random((nr, nh)) * 30
        want = lk_rh.copy()
        ref.lib.ref_normalize(want.ctypes.data_as(C.c_void_p), nr, nh)
        hr = np.ascontiguousarray(lk_rh.T)
        out = np.empty_like(hr)
        keep = np.empty(nr, np.uint8)
        nk = C.c_uint32()
        rl = np.full(nr, 10, np.uint64)  # threshold -4: every row's best is within 4.5 of itself
        lib.phmm_host_normalize_filter(hr.ctypes.data_as(C.c_void_p), nh, nr, rl.ctypes.data_as(C.c_void_p),
                                       out.ctypes.data_as(C.c_void_p), keep.ctypes.data_as(C.c_void_p), C.byref(nk))
        kept = keep.astype(bool)
        assert np.array_equal(out[:, : nk.value], want.T[:, kept])


# ---- several devices: the region partitioner ----------------------------------------------

def test_partition_balances_cells_and_places_every_region_once():
    """Longest-processing-time greedy by region cells: every region in exactly one part, the part
    cells add up, the largest part is within the ideal share plus one region (and within 4/3 of the
    optimum's lower bound), and the split does not depend on anything but the batch."""
    from rovaca_b200 import partition_regions, synth

    pb = synth.config1(300, seed=7)
    cells = np.array([pb.subset([g]).cells() for g in range(pb.n_regions)], np.uint64)
    for n in (1, 2, 3, 8, 13):
        part, load = partition_regions(pb, n)
        assert part.shape == (pb.n_regions,) and int(part.max()) < n
        for p in range(n):
            assert int(load[p]) == int(cells[part == p].sum())
        total, biggest = int(cells.sum()), int(cells.max())
        assert int(load.max()) <= total / n + biggest
        assert int(load.max()) <= 4 / 3 * max(total / n, biggest) + 1
        again, _ = partition_regions(pb, n)
        assert np.array_equal(part, again)


def test_partition_edge_cases():
    from rovaca_b200 import partition_regions

    reg = _region([b"ACGT" * 20], [b"ACGT" * 10])
    empty = _region([], [b"ACGT"])
    pb = PackedBatch.from_regions([reg, empty, reg])
    part, load = partition_regions(pb, 5)  # more parts than regions: some stay empty
    assert part[0] != part[2]  # the two equal regions go to different parts
    assert int(load.sum()) == 2 * 80 * 40 and (load == 0).sum() >= 3
    with pytest.raises(_lib.PhmmError):
        partition_regions(pb, 0)
    with pytest.raises(_lib.PhmmError) as e:
        partition_regions(PackedBatch.from_regions([_region([b"A" * 1537], [b"ACGT"])]), 2)
    assert e.value.name == "PHMM_ERR_LIMIT_EXCEEDED"
