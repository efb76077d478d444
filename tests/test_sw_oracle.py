"""The Smith-Waterman oracle is pinned before it is trusted: against the outputs of the reference's own
aligner stored in tests/golden/sw_golden.json (its unit-test sequences and seeded synthetic pairs), and,
where the reference build exists, against that build on fresh random pairs."""
from __future__ import annotations

import random

import pytest

from oracle import SwRef, build_ref_sw, cigar_string


def test_oracle_reproduces_reference_golden_outputs(sw_oracle, sw_golden):
    """Score, alignment offset, best cell and CIGAR equal the reference's for every golden case, under
    the reference's kernel choice and with the int16 / int32 kernels forced."""
    assert len(sw_golden) > 150
    for c in sw_golden:
        got = sw_oracle.align(c["hap"].encode(), c["read"].encode(), tuple(c["params"]), c["variant"])
        want = (c["score"], c["offset"], c["max_i"], c["max_j"], c["ops"])
        assert got == want, (c["name"], got[:4], want[:4], cigar_string(got[4]), c["cigar"])


def test_kernel_choice_follows_reference_rule(sw_oracle, sw_golden):
    """int32 below 16 read bases, for match <= 0, or when min(length) x match exceeds INT16_MAX
    (ro_sw.c:26-40)."""
    for c in sw_golden:
        assert sw_oracle.uses_int32(len(c["hap"]), len(c["read"]), c["params"][0]) == c["int32"], c["name"]
    assert sw_oracle.uses_int32(400, 15, 10) and not sw_oracle.uses_int32(400, 16, 10)
    assert not sw_oracle.uses_int32(300, 163, 200) and sw_oracle.uses_int32(300, 164, 200)
    assert sw_oracle.uses_int32(300, 100, 0)


def test_reference_unit_test_alignment(sw_golden):
    """The reference unit test's indel case aligns as 28M6D214M (alignment_utils_unit_test.cpp:373-414)."""
    c = next(c for c in sw_golden if c["name"] == "alignment_utils_unit_test[4]")
    assert c["cigar"] == "28M6D214M"


def test_oracle_matches_reference_build_on_random_pairs(sw_oracle):
    if build_ref_sw() is None:
        pytest.skip("reference Smith-Waterman build (oracle/_ref) not available here")
    ref = SwRef()
    rng = random.Random(99)
    n = 0
    for _ in range(400):
        h = bytes(rng.choice(b"ACGT") for _ in range(rng.randint(1, 600)))
        st = rng.randint(0, len(h) - 1)
        r = bytearray(h[st:st + rng.randint(1, 250)])
        for _ in range(len(r) // 15):
            r[rng.randrange(len(r))] = rng.choice(b"ACGTN")
        if rng.random() < 0.3:
            k = rng.randrange(len(r))
            r[k:k] = bytes(rng.choice(b"ACGT") for _ in range(rng.randint(1, 8)))
        prm = rng.choice([SwRef.GENOTYPING, SwRef.ASSEMBLY])
        for v in (0, 1, 2):
            assert sw_oracle.align(h, bytes(r), prm, v) == ref.align(h, bytes(r), prm, v), (len(h), len(r), prm, v)
            n += 1
    assert n == 1200
