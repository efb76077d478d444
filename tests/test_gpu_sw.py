"""Smith-Waterman realignment on the GPU against the oracle and the reference's golden outputs: score,
alignment offset, end cell and CIGAR identical for every pair (integer work, so bit for bit)."""
from __future__ import annotations

import random

import numpy as np
import pytest

from oracle import cigar_string
from rovaca_b200 import PhmmError, sw

pytestmark = pytest.mark.gpu


def _mutate(rng: random.Random, s: bytes, rate: float) -> bytes:
    out = bytearray()
    for c in s:
        r = rng.random()
        if r < rate / 3:
            continue
        if r < 2 * rate / 3:
            out += bytes([rng.choice(b"ACGT"), c])
        elif r < rate:
            out.append(rng.choice(b"ACGT"))
        else:
            out.append(c)
    return bytes(out)


def _realign_pairs(rng: random.Random, n: int, hap_len=(150, 600), read_len=(100, 250)) -> list[tuple[bytes, bytes]]:
    """Reads cut from haplotypes with substitutions and short indels, as HaplotypeCaller realigns
    them (each read against its best haplotype)."""
    pairs = []
    hap = b""
    for q in range(n):
        if q % 20 == 0:
            hap = bytes(rng.choice(b"ACGT") for _ in range(rng.randint(*hap_len)))
        ln = min(rng.randint(*read_len), len(hap))
        st = rng.randint(0, len(hap) - ln)
        pairs.append((hap, _mutate(rng, hap[st:st + ln], rng.choice([0.0, 0.01, 0.03, 0.1]))))
    return pairs


def _check(engine, sw_oracle, pairs, params, variant=0, every=1):
    batch = sw.SwBatch.from_pairs(pairs)
    res = engine.sw_align(batch, params, variant)
    for q in range(0, len(pairs), every):
        h, r = pairs[q]
        want = sw_oracle.align(h, r, params, variant)
        got = res.tuple(q)
        assert got == want, (q, len(h), len(r), params, variant, got[:4], want[:4], cigar_string(got[4]),
                             cigar_string(want[4]))
    return res


def test_golden_outputs_of_the_reference(engine, sw_golden):
    """Every golden case (the reference unit test's sequences and seeded synthetic pairs, with the
    reference's kernel choice and with its int16 / int32 kernels forced) in batches per parameter set."""
    groups: dict = {}
    for c in sw_golden:
        groups.setdefault((tuple(c["params"]), c["variant"]), []).append(c)
    for (params, variant), cases in groups.items():
        batch = sw.SwBatch.from_pairs([(c["hap"].encode(), c["read"].encode()) for c in cases])
        res = engine.sw_align(batch, params, variant)
        for q, c in enumerate(cases):
            want = (c["score"], c["offset"], c["max_i"], c["max_j"], c["ops"])
            assert res.tuple(q) == want, (c["name"], res.tuple(q)[:4], want[:4], res.cigar(q), c["cigar"])


@pytest.mark.parametrize("params", [sw.GENOTYPING, sw.ASSEMBLY], ids=["genotyping", "assembly"])
def test_realignment_batch_matches_oracle(engine, sw_oracle, params):
    rng = random.Random(11 if params == sw.GENOTYPING else 12)
    _check(engine, sw_oracle, _realign_pairs(rng, 3000), params)


@pytest.mark.parametrize("variant", [1, 2])
def test_forced_kernels_match_oracle(engine, sw_oracle, variant):
    """The int32 and int16 kernels forced for every pair, read lengths 1..300 (every stripe width)."""
    rng = random.Random(20 + variant)
    pairs = _realign_pairs(rng, 1200, hap_len=(20, 400), read_len=(1, 300))
    _check(engine, sw_oracle, pairs, sw.GENOTYPING, variant)


def test_every_stripe_width_and_random_reads(engine, sw_oracle):
    """Read lengths on both sides of each stripe-width boundary (32 x K), unrelated random reads,
    reads with N."""
    rng = random.Random(31)
    pairs = []
    for k in (1, 2, 3, 4, 5, 6, 8, 10, 12, 16, 20, 24):
        for ln in (32 * k - 1, 32 * k, 32 * k + 1):
            hap = bytes(rng.choice(b"ACGT") for _ in range(rng.randint(ln // 2 + 1, ln + 200)))
            pairs.append((hap, _mutate(rng, (hap * 4)[:ln], 0.05)[:ln]))
            pairs.append((hap, bytes(rng.choice(b"ACGTN") for _ in range(ln))))
    _check(engine, sw_oracle, pairs, sw.GENOTYPING)
    _check(engine, sw_oracle, pairs, sw.ASSEMBLY)


def test_long_inputs_several_stripes_and_refusal(engine, sw_oracle):
    """Reads longer than one 768-column stripe, haplotypes up to 2047 bases, and inputs of 2048 bases
    or more, which the reference refuses (alignment offset 1, no CIGAR)."""
    rng = random.Random(41)
    hap = bytes(rng.choice(b"ACGT") for _ in range(2047))
    pairs = [(hap, _mutate(rng, hap[100:100 + ln], 0.02)) for ln in (700, 769, 1000, 1536, 1900)]
    pairs += [(hap[:1200], _mutate(rng, hap[:1200], 0.01)), (hap, _mutate(rng, hap, 0.005)[:2047])]
    pairs += [(hap + b"A", hap[:150]), (hap[:300], (hap + b"C")[:2048]), (hap + b"AC", hap + b"G")]
    res = _check(engine, sw_oracle, pairs, sw.GENOTYPING)
    for q in (-3, -2, -1):
        assert res.tuple(q) == (0, 1, 0, 0, [])


def test_sixteen_bit_wrap_around(engine, sw_oracle):
    """Parameters for which the int16 kernel's adds wrap (positive gap scores) run in the wrap-around
    class and still equal the reference's int16 results."""
    rng = random.Random(51)
    pairs = _realign_pairs(rng, 200, hap_len=(100, 400), read_len=(16, 200))
    for params in ((100, 50, 20, 10), (300, -200, -400, -300), (30, -20, -15000, -9000)):
        _check(engine, sw_oracle, pairs, params, 2)
        _check(engine, sw_oracle, pairs, params, 0)


def test_empty_and_tiny_inputs(engine, sw_oracle):
    pairs = [(b"", b""), (b"ACGT", b""), (b"", b"ACGT"), (b"A", b"A"), (b"A", b"C"), (b"", b"A" * 40),
             (b"ACGTACGT", b"T"), (b"T", b"ACGTACGTACGTACGTACGT")]
    _check(engine, sw_oracle, pairs, sw.GENOTYPING)
    _check(engine, sw_oracle, pairs, sw.ASSEMBLY)


def _core(fields):
    return fields[["score", "alignment_offset", "max_i", "max_j", "cigar_count"]]


def test_cigar_capacity_and_counts(engine, sw_oracle):
    """With a smaller per-alignment capacity the first ops are stored and cigar_count stays the full
    count; the compact buffer holds the alignments in item order."""
    rng = random.Random(61)
    pairs = _realign_pairs(rng, 300)
    batch = sw.SwBatch.from_pairs(pairs)
    full = engine.sw_align(batch)
    capped = engine.sw_align(batch, cigar_cap=2)
    assert np.array_equal(_core(full.fields), _core(capped.fields))
    for q in range(len(pairs)):
        assert capped.ops(q) == full.ops(q)[:2]
    offs = full.fields["cigar_offset"].astype(np.int64)
    assert offs[0] == 0 and np.array_equal(np.diff(offs), full.fields["cigar_count"][:-1].astype(np.int64))
    assert full.cigars.size == int(full.fields["cigar_count"].sum())
    none = engine.sw_align(batch, cigar_cap=0)
    assert np.array_equal(_core(full.fields), _core(none.fields)) and none.cigars.size == 0


def test_small_cigar_buffer_is_reported_and_retried(engine):
    """A CIGAR buffer smaller than the batch needs: PHMM_ERR_LIMIT_EXCEEDED with the needed size and
    the results filled (C ABI); the Python call retries once with that size."""
    import ctypes as C

    from rovaca_b200 import _lib

    rng = random.Random(62)
    batch = sw.SwBatch.from_pairs(_realign_pairs(rng, 200, read_len=(100, 250)))
    want = engine.sw_align(batch)
    again = engine.sw_align(batch, ops_per_alignment=1)
    assert np.array_equal(again.fields, want.fields) and np.array_equal(again.cigars, want.cigars)
    lib = _lib.load()
    fields = np.zeros(batch.n, sw.SW_RESULT_DTYPE)
    small = np.zeros(4, np.uint32)
    total = C.c_uint64()
    st = lib.phmm_sw_align(engine._h, None, 0, batch.n, batch.items.ctypes.data, batch.hap_bases.ctypes.data,
                           batch.hap_bases.size, batch.read_bases.ctypes.data, batch.read_bases.size, 2047,
                           fields.ctypes.data, small.ctypes.data, small.size, C.byref(total))
    assert st == _lib.PHMM_ERR_LIMIT_EXCEEDED and total.value == want.cigars.size
    assert np.array_equal(fields, want.fields) and not small.any()


def test_cigar_consumes_the_read_and_the_haplotype_span(engine):
    """Size-independent properties on a large batch: M/I/S ops cover the read; M/D ops cover the
    haplotype from the alignment offset to the end cell; soft clips only at the ends."""
    rng = random.Random(71)
    pairs = _realign_pairs(rng, 20000)
    batch = sw.SwBatch.from_pairs(pairs)
    res = engine.sw_align(batch)
    for q in range(len(pairs)):
        h, r = pairs[q]
        ops = res.ops(q)
        f = res.fields[q]
        read_span = sum(c >> 4 for c in ops if (c & 15) in (0, 1, 4))
        hap_span = sum(c >> 4 for c in ops if (c & 15) in (0, 2))
        assert read_span == len(r)
        assert hap_span == int(f["max_i"]) - int(f["alignment_offset"])
        assert all((c & 15) != 4 for c in ops[1:-1])


def test_resident_runs_equal_host_call(engine):
    rng = random.Random(81)
    batch = sw.SwBatch.from_pairs(_realign_pairs(rng, 2000))
    want = engine.sw_align(batch)
    with engine.sw_resident(batch) as rs:
        ms = rs.run(3)
        assert ms > 0
        got = rs.results()
        assert np.array_equal(got.fields, want.fields) and np.array_equal(got.cigars, want.cigars)
        cls = rs.profile()
        assert cls.shape == (len(sw.CLASS_K),) and cls.sum() > 0
        again = rs.results()
        assert np.array_equal(again.cigars, want.cigars)


def test_items_outside_the_buffers_are_rejected(engine):
    batch = sw.SwBatch.from_pairs([(b"ACGT", b"ACG")])
    batch.items[0]["read_len"] = 10
    with pytest.raises(PhmmError):
        engine.sw_align(batch)
    with pytest.raises(ValueError):
        engine.sw_align(sw.SwBatch.from_pairs([(b"A", b"A")]), variant=3)
    empty = engine.sw_align(sw.SwBatch.from_pairs([]))
    assert len(empty) == 0
