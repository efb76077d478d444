"""Serving loop (continuous batching) and the region API, through the C ABI."""
from __future__ import annotations

import threading

import numpy as np
import pytest

from conftest import assert_same_values
from rovaca_b200 import Engine, synth
from rovaca_b200._lib import PhmmError
from rovaca_b200.pairhmm import PackedBatch, call_pairhmm, schedule_pairhmm

pytestmark = pytest.mark.gpu


def test_each_result_same_alone_and_in_the_mix(engine):
    """Regions submitted concurrently from several threads, admitted while others run, give exactly
    the likelihoods the same region gets alone."""
    pb = synth.config1(40, seed=31)
    alone = [engine.compute(pb.subset([g]))[0] for g in range(pb.n_regions)]
    outs = [np.empty(a.size) for a in alone]
    tickets = [None] * pb.n_regions
    regions = [pb.subset([g]) for g in range(pb.n_regions)]

    def producer(k0):
        for g in range(k0, pb.n_regions, 4):
            tickets[g] = engine.submit(regions[g], outs[g])

    threads = [threading.Thread(target=producer, args=(k,)) for k in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    lat = [engine.wait(t) for t in tickets]
    for g in range(pb.n_regions):
        assert np.array_equal(outs[g], alone[g], equal_nan=True), g
    assert all(total >= queued >= 0 for queued, total in lat)
    st = engine.server_stats()
    assert st["requests_submitted"] >= pb.n_regions and st["requests_done"] >= pb.n_regions
    assert 1 <= st["batches"] <= st["requests_done"] and st["cells_done"] >= pb.cells()


def test_burst_from_many_threads_matches_the_batched_run():
    """A burst of 240 regions from 8 threads, which piles up while the slots are busy and is served
    in batches of many regions (large enough for the multi-threaded gather into pinned staging and
    copy back out): every request's likelihoods equal the same region's in one batched call."""
    pb = synth.config1(240, seed=43)
    with Engine(device=0, autotune=False) as eng:
        want, _, _ = eng.compute(pb)
        sizes = [int(pb.n_haps[g]) * int(pb.n_reads[g]) for g in range(pb.n_regions)]
        offs = np.concatenate([[0], np.cumsum(sizes)])
        regions = [pb.subset([g]) for g in range(pb.n_regions)]
        outs = [np.empty(n) for n in sizes]
        tickets = [None] * pb.n_regions

        def producer(k0):
            for g in range(k0, pb.n_regions, 8):
                tickets[g] = eng.submit(regions[g], outs[g])

        threads = [threading.Thread(target=producer, args=(k,)) for k in range(8)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        for t in tickets:
            eng.wait(t)
        st = eng.server_stats()
    for g in range(pb.n_regions):
        assert np.array_equal(outs[g], want[offs[g]:offs[g + 1]], equal_nan=True), g
    assert st["requests_done"] == pb.n_regions and st["max_batch_regions"] >= 2


def test_flags_and_poll(engine, oracle):
    pb = synth.config2(1, seed=41)
    out = np.empty(pb.out_size)
    fl = np.empty(pb.out_size, np.uint8)
    t = engine.submit(pb, out, fl)
    while not engine.poll(t):
        pass
    engine.wait(t)
    want, used = oracle.batch(pb)
    assert np.max(np.abs(out - want)) <= 1e-12
    assert np.array_equal(fl.astype(bool), used)


def test_cancel_and_timeout():
    """With a budget that fits one request at a time, later requests wait in the queue and can be
    cancelled; a zero timeout on an unfinished request reports TIMEOUT and keeps the ticket."""
    pb = synth.config2(1, seed=51)  # one region needs about 0.47 MB of device data
    one = PackedBatch.from_regions([pb.region(0)])
    with Engine(hbm_budget_bytes=700 << 10) as eng:
        outs = [np.empty(one.out_size) for _ in range(6)]
        ts = [eng.submit(one, o) for o in outs]
        cancelled = set()
        for t in ts[3:]:
            try:
                eng.cancel(t)
                cancelled.add(t)
            except PhmmError:
                pass  # already admitted
        assert cancelled
        released = set()
        try:
            eng.wait(ts[1], timeout_us=0)
            released.add(ts[1])
        except PhmmError as e:
            assert e.name == "PHMM_ERR_TIMEOUT"
        for t in ts:
            if t in released:
                continue
            if t in cancelled:
                with pytest.raises(PhmmError) as e:
                    eng.wait(t)
                assert e.value.name == "PHMM_ERR_CANCELLED"
            else:
                eng.wait(t)
                assert np.isfinite(outs[ts.index(t)]).all()


def test_oversized_request_is_rejected():
    pb = synth.config2(1, seed=52)
    with Engine(hbm_budget_bytes=100 << 10) as eng:
        with pytest.raises(PhmmError) as e:
            eng.submit(pb, np.empty(pb.out_size))
        assert e.value.name == "PHMM_ERR_LIMIT_EXCEEDED"


def test_schedule_pairhmm_vector_api(engine, oracle, ref_regions):
    pb, ref_out = ref_regions["debug"]
    offs = pb.out_offsets()
    for g in range(pb.n_regions):
        r = pb.region(g)
        ok, res = schedule_pairhmm(r.haplotypes, r.reads, r.quality, r.insertion_qualities, r.deletion_qualities,
                                   r.gap_contiguous_qualities, engine=engine)
        assert ok and res.shape == (r.n_reads, r.n_haps)
        want = ref_out[offs[g]:offs[g + 1]].reshape(r.n_haps, r.n_reads).T
        assert np.max(np.abs(res - want)) < 1e-5
    ok, _ = schedule_pairhmm([], [b"ACGT"], [b"\x1e" * 4], [b"-" * 4], [b"-" * 4], [b"\x0a" * 4], engine=engine)
    assert not ok


def _region_api_expected(oracle, haps, reads, quals, mapq, thr, pcr):
    """call_pairhmm restated on the oracle: read preparation (roDV_schedule.cpp:540-609), FP32/FP64
    likelihoods, normalise, drop poorly modelled reads, [hap][read] with kept reads first."""
    import ctypes as C

    from rovaca_b200 import _lib

    lib = _lib.load()
    lk = np.full((len(haps), len(reads)), np.nan)
    for r, (rd, q) in enumerate(zip(reads, quals)):
        n = len(rd)
        qq = np.array([min(x, mapq[r]) for x in q], np.uint8)
        qq = np.where(qq < thr, 6, qq).astype(np.uint8)
        gop = (C.c_uint8 * n)(*([45] * n))
        lib.phmm_host_pcr_model(rd, n, gop, pcr)  # pinned against the reference in test_host.py
        for h, hp in enumerate(haps):
            if n and len(hp):
                lk[h, r], _ = oracle.pair(hp, rd, qq.tobytes(), bytes(gop), bytes(gop), bytes([10]) * n)
    out = np.full_like(lk, np.nan)
    keep = []
    for r in range(len(reads)):
        row = lk[:, r].copy()
        best = row[0]
        for v in row[1:]:
            if best < v:
                best = v
        row = np.where(row < best - 4.5, best - 4.5, row)
        fin = row[~np.isnan(row)]
        b = fin.max() if fin.size else -np.inf
        ok = not (b < min(2.0, np.ceil(len(reads[r]) * 0.02)) * -4.0)
        keep.append(ok)
        if ok:
            out[:, sum(keep) - 1] = row
    return out, np.array(keep)


@pytest.mark.parametrize("pcr", ["NONE", "CONSERVATIVE", "HOSTILE"])
def test_call_pairhmm_region_api(engine, oracle, pcr):
    rng = np.random.default_rng({"NONE": 1, "CONSERVATIVE": 2, "HOSTILE": 3}[pcr])
    base = bytes(np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 420)])
    base = base[:100] + b"ACACACACACAC" + base[100:200] + b"TTTTTTTT" + base[200:]
    haps = [base[:400], base[:150] + b"G" + base[151:400], base[:300] + base[305:400]]
    reads, quals = [], []
    for k in range(24):
        L = int(rng.integers(60, 160))
        s = int(rng.integers(0, 400 - L))
        r = bytearray(base[s:s + L])
        if k % 7 == 3:
            r = bytearray(np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, L)])  # unrelated read
        reads.append(bytes(r))
        quals.append(rng.integers(2, 45, L).astype(np.uint8).tobytes())
    mapq = rng.integers(10, 61, len(reads)).astype(np.uint8)
    mat, kept = call_pairhmm(haps, reads, quals, mapq, 18, pcr, engine=engine)
    want, wkeep = _region_api_expected(oracle, haps, reads, quals, mapq, 18, {"NONE": 0, "CONSERVATIVE": 3,
                                                                              "HOSTILE": 1}[pcr])
    assert np.array_equal(kept, np.nonzero(wkeep)[0])
    assert_same_values(mat, want, 1e-12)
    assert len(kept) < len(reads)  # the unrelated reads are dropped


def test_call_pairhmm_over_limits_returns_nan_matrix(engine):
    haps = [b"A" * 1600]
    with pytest.raises(PhmmError) as e:
        call_pairhmm(haps, [b"ACGT"], [b"\x1e" * 4], [60], 18, "NONE", engine=engine)
    assert e.value.name == "PHMM_ERR_LIMIT_EXCEEDED"


def _host_region_path(engine, haps, reads, quals, mapq, thr, pcr):
    """The region API computed with the host-side preparation and post-processing (the exported
    phmm_host_* functions) around phmm_compute_regions: the device path must give the same bits."""
    import ctypes as C

    from rovaca_b200 import _lib
    from rovaca_b200.pairhmm import Region

    lib = _lib.load()
    qs, gops = [], []
    for rd, q, mq in zip(reads, quals, mapq):
        n = len(rd)
        qq = (C.c_uint8 * max(n, 1))()
        lib.phmm_host_prepare_quals(q, n, int(mq), thr, qq)
        gop = (C.c_uint8 * max(n, 1))(*([45] * max(n, 1)))
        lib.phmm_host_pcr_model(rd, n, gop, pcr)
        qs.append(bytes(qq)[:n])
        gops.append(bytes(gop)[:n])
    pb = PackedBatch.from_regions([Region(haps, reads, qs, gops, gops, [bytes([10]) * len(r) for r in reads])])
    lk, _, _ = engine.compute(pb)
    out = np.empty(len(haps) * len(reads))
    keep = np.empty(len(reads), np.uint8)
    nk = C.c_uint32()
    rlen = np.array([len(r) for r in reads], np.uint64)
    lib.phmm_host_normalize_filter(lk.ctypes.data, len(haps), len(reads), rlen.ctypes.data, out.ctypes.data,
                                   keep.ctypes.data, C.byref(nk))
    return out.reshape(len(haps), len(reads)), keep.astype(bool)


def _repeat_region(rng, n_reads, max_len):
    """Haplotypes and reads rich in tandem repeats of unit lengths 1-9."""
    acgt = np.frombuffer(b"ACGT", np.uint8)
    parts = []
    for _ in range(30):
        unit = bytes(acgt[rng.integers(0, 4, int(rng.integers(1, 10)))])
        parts.append(unit * int(rng.integers(1, 25)))
        parts.append(bytes(acgt[rng.integers(0, 4, int(rng.integers(0, 12)))]))
    base = b"".join(parts)[:1500]
    haps = [base[:1000], base[3:1003], base[:500] + base[507:1010]]
    reads, quals = [], []
    for _ in range(n_reads):
        L = int(rng.integers(1, max_len + 1))
        s = int(rng.integers(0, max(1, len(base) - L)))
        r = bytearray(base[s:s + L])
        if rng.random() < 0.1 and L:
            r[int(rng.integers(0, L))] = ord("N")
        reads.append(bytes(r))
        quals.append(rng.integers(0, 50, L).astype(np.uint8).tobytes())
    mapq = rng.integers(0, 70, n_reads).astype(np.uint8)
    return haps, reads, quals, mapq


@pytest.mark.parametrize("pcr", [0, 1, 2, 3])
def test_device_region_path_equals_host_preparation(engine, pcr):
    """Quality cap, gap qualities and the PCR tandem-repeat cap computed on the GPU, and the
    normalise/filter/compact step after it, give exactly the host functions' results."""
    rng = np.random.default_rng(100 + pcr)
    for thr, max_len in ((18, 768), (5, 200), (40, 300)):
        haps, reads, quals, mapq = _repeat_region(rng, 40, max_len)
        got, keep = engine.call_region(haps, reads, quals, mapq, thr, pcr)
        want, wkeep = _host_region_path(engine, haps, reads, quals, mapq, thr, pcr)
        assert np.array_equal(keep, wkeep)
        assert np.array_equal(got, want, equal_nan=True)
        assert 0 < keep.sum() < len(reads)


def test_region_and_plain_requests_mix(engine):
    """Region-API and plain requests submitted together from several threads: each gets the result
    it gets alone (the loop batches each kind separately)."""
    rng = np.random.default_rng(7)
    regions = [_repeat_region(rng, 20, 250) for _ in range(12)]
    alone = [engine.call_region(h, r, q, m, 18, 3) for h, r, q, m in regions]
    pb = synth.config1(12, seed=9)
    plain_alone = [engine.compute(pb.subset([g]))[0] for g in range(pb.n_regions)]
    outs = [np.empty(x.size) for x in plain_alone]
    tickets, rts = [None] * 12, [None] * 12

    def producer(k0):
        for g in range(k0, 12, 3):
            rts[g] = engine.submit_region(*regions[g], 18, 3)
            tickets[g] = engine.submit(pb.subset([g]), outs[g])

    threads = [threading.Thread(target=producer, args=(k,)) for k in range(3)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for g in range(12):
        mat, keep = rts[g].wait()
        engine.wait(tickets[g])
        assert np.array_equal(mat, alone[g][0], equal_nan=True)
        assert np.array_equal(keep, alone[g][1])
        assert np.array_equal(outs[g], plain_alone[g], equal_nan=True)


def _oracle_region_lk(oracle, haps, reads, quals, mapq, thr, pcr, fp64_only):
    """Region-API likelihoods [hap][read] from the oracle: host read preparation, then the oracle's
    FP32/FP64 switch (or all-FP64)."""
    import ctypes as C

    from rovaca_b200 import _lib
    from rovaca_b200.pairhmm import Region

    lib = _lib.load()
    qs, gops = [], []
    for rd, q, mq in zip(reads, quals, mapq):
        n = len(rd)
        qq = (C.c_uint8 * max(n, 1))()
        lib.phmm_host_prepare_quals(q, n, int(mq), thr, qq)
        gop = (C.c_uint8 * max(n, 1))(*([45] * max(n, 1)))
        lib.phmm_host_pcr_model(rd, n, gop, pcr)
        qs.append(bytes(qq)[:n])
        gops.append(bytes(gop)[:n])
    pb = PackedBatch.from_regions([Region(haps, reads, qs, gops, gops, [bytes([10]) * len(r) for r in reads])])
    lk, _ = oracle.batch(pb, fp64_only=fp64_only)
    return lk.reshape(len(haps), len(reads))


def test_genotyping_on_device_and_concordance(engine, oracle, genotype_ref):
    """Allele marginalisation and diploid genotype likelihoods on the GPU equal the reference's own
    genotyping code (compiled from its sources) and the checker's restatement on the same normalised
    matrix bit for bit; the calls are identical to the calls made
    from the reference's own likelihoods (its FP32 pass with the FP64 fallback, which the engine
    reproduces pair for pair); against calls from all-FP64 likelihoods a call may differ only where
    the two genotypes' FP64 likelihoods are a near-tie (within 1e-3 log10)."""
    from oracle import genotype as G

    regions = synth.genotyping_regions(16, seed=11)
    tickets = [engine.submit_region(r["haplotypes"], r["reads"], r["quals"], r["mapq"], 18, 3, events=r["events"],
                                    want_allele_lk=True) for r in regions]
    calls, truth_hits, diff64 = 0, 0, 0
    for r, t in zip(regions, tickets):
        mat, keep = t.wait()
        got = t.genotypes()
        K = int(keep.sum())
        for (A, ha), (gl, best, alk) in zip(r["events"], got):
            walk = G.marginalize(mat, K, list(ha), A)
            assert np.array_equal(alk[:, :K], walk)
            assert np.isnan(alk[:, K:]).all()
            wgl = G.genotype_likelihoods(walk)
            assert np.array_equal(gl, wgl)
            assert best == G.best_genotype(wgl)
            ralk, rgl = genotype_ref.genotype(mat[:, :K], ha, A)
            assert np.array_equal(alk[:, :K], ralk, equal_nan=True)
            assert np.array_equal(gl, rgl, equal_nan=True)
        lens = [len(x) for x in r["reads"]]
        lk_ref = _oracle_region_lk(oracle, r["haplotypes"], r["reads"], r["quals"], r["mapq"], 18, 3, False)
        res_ref, _, keep_ref = G.genotype_region(lk_ref, lens, r["events"])
        lk64 = _oracle_region_lk(oracle, r["haplotypes"], r["reads"], r["quals"], r["mapq"], 18, 3, True)
        res64, _, _ = G.genotype_region(lk64, lens, r["events"])
        assert np.array_equal(keep_ref, keep)
        for (gl, best, _), (glr, bestr, _), (gl64, best64, _), truth in zip(got, res_ref, res64, r["truth"]):
            assert best == bestr
            assert np.max(np.abs(gl - glr)) < 1e-9
            if best != best64:
                diff64 += 1
                assert abs(gl64[best] - gl64[best64]) < 1e-3
            calls += 1
            truth_hits += int(best == truth)
    assert diff64 <= calls // 10
    # sanity of the synthetic data only: sites near a window's ends have few reads, so some calls
    # miss the simulated truth whatever the likelihood engine
    assert truth_hits >= 0.6 * calls


def test_genotyping_only_results_come_back(engine):
    """With no matrix requested, only keep flags, genotype likelihoods and calls return."""
    r = synth.genotyping_regions(1, seed=12)[0]
    full = engine.submit_region(r["haplotypes"], r["reads"], r["quals"], r["mapq"], 18, 0, events=r["events"])
    lean = engine.submit_region(r["haplotypes"], r["reads"], r["quals"], r["mapq"], 18, 0, events=r["events"],
                                want_matrix=False)
    m1, k1 = full.wait()
    m2, k2 = lean.wait()
    assert m2 is None and np.array_equal(k1, k2)
    for (g1, b1, _), (g2, b2, _) in zip(full.genotypes(), lean.genotypes()):
        assert np.array_equal(g1, g2) and b1 == b2
    with pytest.raises(PhmmError) as e:
        engine.submit_region(r["haplotypes"], r["reads"], r["quals"], r["mapq"], 18, 0,
                             events=[(50, np.zeros(len(r["haplotypes"]), np.int8))])
    assert e.value.name == "PHMM_ERR_LIMIT_EXCEEDED"


def test_device_set_equals_one_engine():
    """A device set of two engines (both on device 0 here: one GPU per test box) splits a batch by
    region cells and returns exactly one engine's results, region blocks in place; serving requests
    go to the less loaded member and return the same bits."""
    from rovaca_b200 import DeviceSet, partition_regions

    pb = synth.config1(24, seed=33)
    with Engine(device=0, autotune=False) as eng:
        want, want_fl, _ = eng.compute(pb, want_flags=True)
    part, load = partition_regions(pb, 2)
    assert set(part.tolist()) == {0, 1}
    with DeviceSet([0, 0], autotune=False) as ds:
        got, fl, st = ds.compute(pb, want_flags=True)
        assert np.array_equal(got, want, equal_nan=True)
        assert np.array_equal(fl, want_fl)
        assert st["cells"] == pb.cells() and st["regions"] == pb.n_regions
        got2, _, _ = ds.compute(pb)  # staging buffers reused
        assert np.array_equal(got2, want, equal_nan=True)
        offs = pb.out_offsets()
        outs = [np.empty(offs[g + 1] - offs[g]) for g in range(pb.n_regions)]
        tickets = [ds.submit(pb.subset([g]), outs[g]) for g in range(pb.n_regions)]
        members = [ds.wait(t)[2] for t in tickets]
        assert set(members) == {0, 1}
        for g in range(pb.n_regions):
            assert np.array_equal(outs[g], want[offs[g]:offs[g + 1]], equal_nan=True), g
