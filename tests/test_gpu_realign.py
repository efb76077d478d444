"""Realignment of a region's kept reads to their best haplotypes inside the region pipeline on the GPU
(phmm_submit_region_realign): the best haplotype of every kept read equals the checker's
search_best_allele on the region's normalised matrix, and each read's alignment (score, end cell,
offset, CIGAR) equals the Smith-Waterman oracle's on (best haplotype, read without its clips)."""
from __future__ import annotations

import random

import numpy as np
import pytest

from oracle import genotype as G
from rovaca_b200 import PhmmError, synth

pytestmark = pytest.mark.gpu


def _realign_inputs(r, rng):
    M, N = len(r["haplotypes"]), len(r["reads"])
    prio = [float(rng.randint(-4, 1)) + (1.0 if h == 0 else 0.0) for h in range(M)]
    cl = [rng.choice([0, 0, 0, 1, 3, 7]) for _ in range(N)]
    cr = [rng.choice([0, 0, 0, 2, 5]) for _ in range(N)]
    return {"priority": prio, "clip_left": cl, "clip_right": cr}


def _check_region(r, ticket, rz, sw_oracle):
    mat, keep = ticket.wait()
    best, res = ticket.realignment()
    col = 0
    for q, read in enumerate(r["reads"]):
        if not keep[q]:
            assert best[q] == -1 and res.tuple(q) == (0, 0, 0, 0, [])
            continue
        want = G.search_best_allele(mat[:, col], rz["priority"])
        col += 1
        assert best[q] == want, (q, best[q], want)
        hap = bytes(r["haplotypes"][want])
        rd = bytes(read)[rz["clip_left"][q]:len(read) - rz["clip_right"][q]]
        assert res.tuple(q) == sw_oracle.align(hap, rd), (q, res.tuple(q)[:4])
    return int(keep.sum())


def test_realignment_in_the_region_pipeline(engine, sw_oracle):
    rng = random.Random(5)
    regions = synth.genotyping_regions(24, seed=31)
    inputs = [_realign_inputs(r, rng) for r in regions]
    # submitted together: they share batches, mixed with requests that do not realign
    tickets = []
    for i, (r, rz) in enumerate(zip(regions, inputs)):
        tickets.append(engine.submit_region(r["haplotypes"], r["reads"], r["quals"], r["mapq"], 18, 3,
                                            events=r["events"] if i % 3 == 0 else None,
                                            realign=rz if i % 4 != 3 else None))
    kept = 0
    for i, (r, rz, t) in enumerate(zip(regions, inputs, tickets)):
        if i % 4 == 3:
            t.wait()
            continue
        kept += _check_region(r, t, rz, sw_oracle)
    assert kept > 100


def test_realignment_alone_equals_in_a_mix(engine):
    regions = synth.genotyping_regions(6, seed=32)
    rng = random.Random(6)
    inputs = [_realign_inputs(r, rng) for r in regions]
    alone = []
    for r, rz in zip(regions, inputs):
        t = engine.submit_region(r["haplotypes"], r["reads"], r["quals"], r["mapq"], 18, 3, realign=rz)
        t.wait()
        alone.append(t.realignment())
    tickets = [engine.submit_region(r["haplotypes"], r["reads"], r["quals"], r["mapq"], 18, 3, realign=rz)
               for r, rz in zip(regions, inputs)]
    for (b0, s0), t in zip(alone, tickets):
        t.wait()
        b1, s1 = t.realignment()
        assert np.array_equal(b0, b1) and np.array_equal(s0.fields, s1.fields) and np.array_equal(s0.cigars, s1.cigars)


def test_realignment_cigar_buffer_too_small(engine):
    r = synth.genotyping_regions(1, seed=33)[0]
    rz = _realign_inputs(r, random.Random(7))
    full = engine.submit_region(r["haplotypes"], r["reads"], r["quals"], r["mapq"], 18, 3, realign=rz)
    full.wait()
    need = full.cigar_total.value
    assert need > 0
    small = engine.submit_region(r["haplotypes"], r["reads"], r["quals"], r["mapq"], 18, 3,
                                 realign=dict(rz, cigar_capacity=need - 1))
    with pytest.raises(PhmmError):
        small.wait()
    assert small.cigar_total.value == need
    assert np.array_equal(small.best_hap, full.best_hap)


def test_realignment_input_checks(engine):
    r = synth.genotyping_regions(1, seed=34)[0]
    with pytest.raises(ValueError):
        engine.submit_region(r["haplotypes"], r["reads"], r["quals"], r["mapq"], 18, 3, realign={"priority": [0.0]})
    n = len(r["reads"])
    too_much = {"priority": [0.0] * len(r["haplotypes"]), "clip_left": [1000] * n, "clip_right": [0] * n}
    with pytest.raises(PhmmError):
        engine.submit_region(r["haplotypes"], r["reads"], r["quals"], r["mapq"], 18, 3, realign=too_much)
