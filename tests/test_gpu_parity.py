"""Parity of the CUDA engine with the oracle and the reference, through the C ABI.

Tolerances: the engine reproduces the reference's FP32/FP64 arithmetic exactly, so its log10 values
equal the oracle's up to the last bits of the final double log10 (|diff| <= 1e-12, far below the
6e-8 relative step between neighbouring FP32 sums, so equal values mean equal raw sums); against the
all-FP64 oracle the bound is the 1e-4 log10 of the specification; against the reference's own output
1e-5 (pairs the reference leaves to its intra kernel round the prior and the log once more)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import assert_same_values, case_tuple
from rovaca_b200 import synth
from rovaca_b200.pairhmm import PackedBatch, PhmmError, Region

pytestmark = pytest.mark.gpu

EXACT = 1e-12
SPEC = 1e-4


def _golden_batch(cases):
    regs = [Region([c["hap"]], [c["read"]], [bytes(c["q"])], [bytes(c["i"])], [bytes(c["d"])], [bytes(c["c"])])
            for c in cases]
    return PackedBatch.from_regions(regs)


def test_golden_vectors(engine, oracle, golden_cases):
    pb = _golden_batch(golden_cases)
    got, flags, _ = engine.compute(pb, want_flags=True)
    for k, c in enumerate(golden_cases):
        want, used = oracle.pair(*case_tuple(c))
        assert abs(got[k] - c["expected"]) < 1e-5, (c["line"], got[k], c["expected"])
        assert abs(got[k] - want) <= EXACT, (c["line"], got[k], want)
        assert bool(flags[k]) == used


@pytest.mark.parametrize("group", ["debug", "config0", "config1", "config2", "edge"])
def test_reference_regions(engine, oracle, ref_regions, group):
    pb, ref_out = ref_regions[group]
    got, flags, stats = engine.compute(pb, want_flags=True)
    want, used = oracle.batch(pb)
    assert_same_values(got, want, EXACT)
    assert np.array_equal(flags.astype(bool), used)
    assert stats["pairs_f64"] == int(used.sum())
    # the reference's own schedule_pairhmm output
    assert_same_values(got, ref_out, 1e-5, "reference output")
    # every FP32 -> FP64 decision equals the reference's, whichever of its kernels made it
    routes = np.concatenate([oracle.schedule_region(pb, g)[1].reshape(-1) for g in range(pb.n_regions)])
    ref_f64 = np.isin(routes, oracle.ROUTE_F64)
    assert np.array_equal(flags.astype(bool), ref_f64), int(np.sum(flags.astype(bool) != ref_f64))
    # the specification's bound against the all-FP64 oracle
    f64, _ = oracle.batch(pb, fp64_only=True)
    assert_same_values(got, f64, SPEC, "all-FP64 oracle")


def test_graph_and_direct_launch_agree(engine, engine_direct, ref_regions):
    for group in ("debug", "edge", "config1"):
        pb, _ = ref_regions[group]
        a, fa, _ = engine.compute(pb, want_flags=True)
        b, fb, _ = engine_direct.compute(pb, want_flags=True)
        assert np.array_equal(a, b, equal_nan=True)
        assert np.array_equal(fa, fb)


def test_region_result_independent_of_batch(engine):
    """Per-pair arithmetic does not depend on what else is in the batch."""
    pb = synth.config1(12, seed=5)
    full, _, _ = engine.compute(pb)
    offs = pb.out_offsets()
    for g in (0, 5, 11):
        alone, _, _ = engine.compute(pb.subset([g]))
        assert np.array_equal(alone, full[offs[g]:offs[g + 1]], equal_nan=True)
    rev = pb.subset(list(range(pb.n_regions))[::-1])
    back, _, _ = engine.compute(rev)
    roffs = rev.out_offsets()
    for g in range(pb.n_regions):
        r = pb.n_regions - 1 - g
        assert np.array_equal(back[roffs[r]:roffs[r + 1]], full[offs[g]:offs[g + 1]], equal_nan=True)


def test_bases_sent_early_then_arena_grows(oracle):
    """phmm_compute_regions copies bases and qualities while it plans when the arena already holds
    them; a batch with fewer bases but more pairs then grows the arena after those copies, which are
    made again: results equal the oracle's either way, also with a fresh engine at each size."""
    from rovaca_b200 import Engine, Region
    from rovaca_b200.pairhmm import PackedBatch

    rng = np.random.default_rng(8)
    bases = lambda n: bytes(rng.choice(np.frombuffer(b"ACGT", np.uint8), n))
    qual = lambda n: bytes(rng.integers(10, 41, n, dtype=np.uint8))
    haps = [bases(300) for _ in range(30)]

    def batch(n_reads, length):
        reads = [bases(length) for _ in range(n_reads)]
        gap = [bytes([45]) * length] * n_reads
        return PackedBatch.from_regions([Region(haps, reads, [qual(length) for _ in reads], gap, gap,
                                                [bytes([10]) * length] * n_reads)])

    many_bases = batch(40, 250)   # 10,000 read bases, 1,200 pairs
    many_pairs = batch(200, 30)   # 6,000 read bases (they fit), 6,000 pairs (the arena grows)
    with Engine(device=0, autotune=False) as eng:
        for pb in (many_bases, many_pairs, many_bases, many_pairs):
            got, _, _ = eng.compute(pb)
            want, _ = oracle.batch(pb)
            assert np.max(np.abs(got - want)) <= EXACT


def test_underflow_stress_region(engine, oracle):
    """Config-2 regime: most pairs fall below 1e-28 in FP32 and are recomputed in FP64."""
    pb = synth.config2(2, seed=21)
    got, flags, stats = engine.compute(pb, want_flags=True)
    want, used = oracle.batch(pb)
    assert used.mean() > 0.5
    assert np.array_equal(flags.astype(bool), used)
    assert np.max(np.abs(got - want)) <= EXACT
    f64, _ = oracle.batch(pb, fp64_only=True)
    assert np.max(np.abs(got - f64)) < SPEC


def test_empty_reads_and_haplotypes_give_nan(engine, oracle):
    reg = Region([b"ACGTACGTAA", b"", b"ACGGT"], [b"ACGT", b"", b"CGTAC"],
                 [b"\x1e" * 4, b"", b"\x1e" * 5], [b"\x2d" * 4, b"", b"\x2d" * 5], [b"\x2d" * 4, b"", b"\x2d" * 5],
                 [b"\x0a" * 4, b"", b"\x0a" * 5])
    pb = PackedBatch.from_regions([reg])
    got, _, stats = engine.compute(pb)
    m = got.reshape(3, 3)
    assert np.isnan(m[1]).all() and np.isnan(m[:, 1]).all()
    assert np.isfinite(m[[0, 2]][:, [0, 2]]).all()
    want, _ = oracle.batch(pb)
    assert_same_values(got, want, EXACT)
    assert stats["pairs"] == 4


def test_regions_without_reads_or_haplotypes(engine):
    regs = [Region([], [b"ACGT"], [b"\x1e" * 4], [b"-" * 4], [b"-" * 4], [b"\x0a" * 4]),
            Region([b"ACGT"], [], [], [], [], []),
            Region([b"ACGTT"], [b"ACGT"], [b"\x1e" * 4], [b"-" * 4], [b"-" * 4], [b"\x0a" * 4])]
    got, _, _ = engine.compute(PackedBatch.from_regions(regs))
    assert got.shape == (1,) and np.isfinite(got[0])


def test_limits_are_rejected(engine):
    reg = Region([b"A" * 1537], [b"ACGT"], [b"\x1e" * 4], [b"-" * 4], [b"-" * 4], [b"\x0a" * 4])
    with pytest.raises(PhmmError) as e:
        engine.compute(PackedBatch.from_regions([reg]))
    assert e.value.name == "PHMM_ERR_LIMIT_EXCEEDED"


def test_random_lengths_all_classes(engine, oracle):
    """Read lengths 1..768 (every rows-per-lane class and multi-stripe), haplotypes 1..1536, with N."""
    rng = np.random.default_rng(77)
    acgt = np.frombuffer(b"ACGTN", np.uint8)
    regs = []
    for g in range(6):
        H = [int(x) for x in rng.integers(1, 1537 if g == 0 else 400, int(rng.integers(1, 6)))]
        base = acgt[rng.integers(0, 4, max(H) + 800)]
        haps = [bytes(base[:h]) for h in H]
        if g % 2:
            hb = bytearray(haps[0])
            hb[len(hb) // 2] = ord("N")
            haps[0] = bytes(hb)
        lens = [int(x) for x in rng.integers(1, 769 if g < 2 else 300, int(rng.integers(1, 12)))]
        reads = []
        for L in lens:
            r = bytearray(base[int(rng.integers(0, 100)):][:L])
            if rng.random() < 0.2:
                r[int(rng.integers(0, len(r)))] = ord("N")
            reads.append(bytes(r))
        q = [rng.integers(2, 42, len(r)).astype(np.uint8).tobytes() for r in reads]
        i = [rng.integers(10, 46, len(r)).astype(np.uint8).tobytes() for r in reads]
        d = [rng.integers(10, 46, len(r)).astype(np.uint8).tobytes() for r in reads]
        c = [rng.integers(5, 15, len(r)).astype(np.uint8).tobytes() for r in reads]
        regs.append(Region(haps, reads, q, i, d, c))
    pb = PackedBatch.from_regions(regs)
    got, flags, _ = engine.compute(pb, want_flags=True)
    want, used = oracle.batch(pb)
    assert_same_values(got, want, EXACT)
    assert np.array_equal(flags.astype(bool), used)


def test_chunked_compute_equals_one_pipeline(oracle):
    """phmm_compute_regions run as a pipeline of region chunks on two device slots (chunk_cells
    forced down) gives the likelihoods, flags and counts of one pipeline, again when a second call
    reuses both slots; a smaller batch afterwards and an invalid region in a later chunk behave as
    without chunks (the whole batch is validated before anything is launched)."""
    from rovaca_b200 import Engine

    pb = synth.config1(40, seed=9)
    with Engine(device=0, autotune=False, chunk_cells=2**64 - 1) as one:
        want, wflags, ws = one.compute(pb, want_flags=True)
    offs = pb.out_offsets()
    with Engine(device=0, autotune=False, chunk_cells=1) as eng:
        for _ in range(2):
            got, flags, st = eng.compute(pb, want_flags=True)
            assert np.array_equal(got, want, equal_nan=True) and np.array_equal(flags, wflags)
            for k in ("regions", "pairs", "cells", "pairs_f64", "work_items", "h2d_bytes", "d2h_bytes"):
                assert st[k] == ws[k], k
            assert st["device_ms"] > 0 and st["kernel_launches"] > ws["kernel_launches"]
        got3, _, _ = eng.compute(pb.subset([3, 4, 5]))
        assert np.array_equal(got3, want[offs[3]:offs[6]], equal_nan=True)
        bad = Region([b"A" * 1537], [b"ACGT"], [b"\x1e" * 4], [b"-" * 4], [b"-" * 4], [b"\x0a" * 4])
        with pytest.raises(PhmmError) as e:
            eng.compute(PackedBatch.from_regions([pb.region(g) for g in range(6)] + [bad]))
        assert e.value.name == "PHMM_ERR_LIMIT_EXCEEDED"
        again, _, _ = eng.compute(pb)
        assert np.array_equal(again, want, equal_nan=True)
    sample = [0, 17, 39]
    ref, used = oracle.batch(pb.subset(sample))
    got_s = np.concatenate([want[offs[g]:offs[g + 1]] for g in sample])
    assert np.max(np.abs(got_s - ref)) <= EXACT


def test_bytes_outside_acgtn(engine, oracle):
    """Lower-case and IUPAC letters: pairs without 'N' compare raw bytes (so 'a' and 'E', or 'R' and
    'R', are told apart or matched exactly as bytes), pairs with 'N' use the reference's base classes."""
    rng = np.random.default_rng(91)
    alphabet = np.frombuffer(b"ACGTACGTACGTacgtRYKMSWEBDHV", np.uint8)
    regs = []
    for g in range(4):
        base = alphabet[rng.integers(0, len(alphabet), 700)]
        haps = [bytes(base[s:s + int(rng.integers(40, 300))]) for s in rng.integers(0, 300, 3)]
        reads = []
        for L in rng.integers(20, 260, 9):
            r = bytearray(base[int(rng.integers(0, 300)):][:int(L)])
            if g % 2 and rng.random() < 0.4:
                r[int(rng.integers(0, len(r)))] = ord("N")
            reads.append(bytes(r))
        q = [rng.integers(2, 42, len(r)).astype(np.uint8).tobytes() for r in reads]
        i = [rng.integers(10, 46, len(r)).astype(np.uint8).tobytes() for r in reads]
        d = [rng.integers(10, 46, len(r)).astype(np.uint8).tobytes() for r in reads]
        c = [rng.integers(5, 15, len(r)).astype(np.uint8).tobytes() for r in reads]
        regs.append(Region(haps, reads, q, i, d, c))
    pb = PackedBatch.from_regions(regs)
    got, flags, _ = engine.compute(pb, want_flags=True)
    want, used = oracle.batch(pb)
    assert_same_values(got, want, EXACT)
    assert np.array_equal(flags.astype(bool), used)


def test_full_size_batch_properties(engine, oracle):
    """The benchmark batch (2,000 regions, ~5.7e11 cells): deterministic, every pair finite, and a
    seeded sample of regions equal to the oracle."""
    pb = synth.config1()
    a, fa, sa = engine.compute(pb, want_flags=True)
    b, fb, sb = engine.compute(pb, want_flags=True)
    assert np.array_equal(a, b) and np.array_equal(fa, fb)
    assert np.isfinite(a).all()
    assert sa["pairs"] == pb.out_size and sa["pairs_f64"] == int(fa.sum())
    offs = pb.out_offsets()
    sample = [0, 777, 1999]
    want, used = oracle.batch(pb.subset(sample))
    got = np.concatenate([a[offs[g]:offs[g + 1]] for g in sample])
    gflags = np.concatenate([fa[offs[g]:offs[g + 1]] for g in sample])
    assert np.max(np.abs(got - want)) <= EXACT
    assert np.array_equal(gflags.astype(bool), used)


def _all_length_batch(seed):
    """Reads of every length bucket 1..24 (with and without N, constant and per-row gap
    qualities) against a few haplotypes."""
    rng = np.random.default_rng(seed)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    regs = []
    for g in range(3):
        base = acgt[rng.integers(0, 4, 2000)]
        haps = [bytes(base[s:s + int(rng.integers(100, 700))]) for s in rng.integers(0, 600, 4)]
        if g == 2:
            hb = bytearray(haps[1])
            hb[10] = ord("N")
            haps[1] = bytes(hb)
        reads, ins = [], []
        for bucket in range(1, 25):
            for k in range(2):
                L = int(rng.integers(32 * (bucket - 1) + 1, 32 * bucket + 1))
                r = bytearray(base[int(rng.integers(0, 1000)):][:L])
                if (bucket + k + g) % 5 == 0:
                    r[len(r) // 2] = ord("N")
                reads.append(bytes(r))
                ins.append(bytes([45] * L) if k == 0 else rng.integers(30, 46, L).astype(np.uint8).tobytes())
        q = [rng.integers(5, 42, len(r)).astype(np.uint8).tobytes() for r in reads]
        d = [bytes([45] * len(r)) for r in reads]
        c = [bytes([10] * len(r)) for r in reads]
        regs.append(Region(haps, reads, q, ins, d, c))
    return PackedBatch.from_regions(regs)


def _table(shape_of_bucket):
    from rovaca_b200 import _lib
    from rovaca_b200.pairhmm import default_tiles

    kh, mu = default_tiles().as_arrays()
    for m in range(3):
        for b in range(1, 25):
            s = shape_of_bucket(m, b)
            if s is not None:
                kh[m, b - 1], mu[m, b - 1] = s
    return _lib.TileTable.from_arrays(kh, mu)


def test_every_tile_shape_gives_identical_results(oracle):
    """Every FP32 kernel class (13 shapes x 3 modes) computes the same bits: the same batch under
    tables that move each bucket to each multi-stripe shape that can hold it."""
    from rovaca_b200 import Engine

    pb = _all_length_batch(7)
    want, used = oracle.batch(pb)
    with Engine(device=0, autotune=False, use_cuda_graph=False) as eng:
        base, fb, _ = eng.compute(pb, want_flags=True)
        assert_same_values(base, want, EXACT, "default tiles vs oracle")
        assert np.array_equal(fb.astype(bool), used)
        for kh in range(4, 9):
            eng.set_tiles(_table(lambda m, b, kh=kh: (kh, 1) if kh < b else None))
            got, fg, _ = eng.compute(pb, want_flags=True)
            assert np.array_equal(got, base, equal_nan=True), kh
            assert np.array_equal(fg, fb), kh
    # a captured graph is captured again for a new table (its FP64 dependencies follow the shapes)
    with Engine(device=0, autotune=False, use_cuda_graph=True) as eng:
        a, _, _ = eng.compute(pb)
        assert np.array_equal(a, base, equal_nan=True)
        eng.set_tiles(_table(lambda m, b: (4, 1) if b > 4 else None))
        got, fg, _ = eng.compute(pb, want_flags=True)
        assert np.array_equal(got, base, equal_nan=True) and np.array_equal(fg, fb)


def test_autotune_installs_a_valid_table(engine_direct):
    from rovaca_b200 import Engine

    with Engine(device=0, autotune=False) as eng:
        rep = eng.autotune()
        assert rep["seconds"] > 0 and rep["entries"]
        kh, mu = eng.tiles().as_arrays()
        chosen = [e for e in rep["entries"] if e["chosen"]]
        tuned = {(e["mode"], e["bucket"]) for e in rep["entries"]}
        assert {(e["mode"], e["bucket"]) for e in chosen} == tuned  # one winner per tuned bucket
        for e in chosen:
            assert kh[e["mode"], e["bucket"] - 1] == e["rows_per_lane"]
            assert bool(mu[e["mode"], e["bucket"] - 1]) == e["multi_stripe"]
        assert all(e["gcups"] > 0 for e in rep["entries"])
        pb = synth.config1(6, seed=3)
        a, _, _ = eng.compute(pb)
        b, _, _ = engine_direct.compute(pb)
        assert np.array_equal(a, b, equal_nan=True)


@pytest.mark.parametrize("group", ["debug", "config0", "config1", "config2", "edge"])
def test_fp64_check_equals_the_all_fp64_oracle(engine, oracle, ref_regions, group):
    """phmm_resident_check_fp64 recomputes every pair with the all-FP64 model on the device; it
    equals the CPU all-FP64 oracle pair for pair, and the resident gives its own results again after
    the next run."""
    pb, _ = ref_regions[group]
    want, _ = oracle.batch(pb, fp64_only=True)
    with engine.resident(pb, want_flags=True) as res:
        own, own_flags = res.results()
        got = res.check_fp64()
        assert_same_values(got, want, EXACT, group)
        res.run(1)
        again, again_flags = res.results()
    assert np.array_equal(again, own, equal_nan=True)
    assert np.array_equal(again_flags, own_flags)
