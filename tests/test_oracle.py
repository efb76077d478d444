"""The oracle is pinned before it is trusted: against the reference's golden vectors, against the
reference's own kernels (raw sums bit for bit), and against the reference's scheduler output."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import case_tuple, f32_of_hex, f64_of_hex
from oracle import FUSED, INTER, INTRA, UNFUSED


def test_golden_vectors_expected_values(oracle, golden_cases):
    """104 golden cases (pairhmm-testdata.txt) and the two hand cases, within the 1e-5 the
    reference's own tests allow (pairhmm_unittest.cpp:117-141,431-464)."""
    for c in golden_cases:
        v, _ = oracle.pair(*case_tuple(c))
        assert abs(v - c["expected"]) < 1e-5, (c["line"], v, c["expected"])


def test_golden_vectors_bit_exact_with_reference_kernels(oracle, golden_cases):
    """Raw scaled sums equal the reference's intra and inter kernels bit for bit, FP32 and FP64."""
    for c in golden_cases:
        t = case_tuple(c)
        assert oracle.raw_f32(*t, kernel=INTRA, fused=FUSED) == f32_of_hex(c["ref_intra_raw_f32"]), c["line"]
        assert oracle.raw_f64(*t, kernel=INTRA, fused=FUSED) == f64_of_hex(c["ref_intra_raw_f64"]), c["line"]
        assert oracle.raw_f32(*t, kernel=INTER, fused=FUSED) == f32_of_hex(c["ref_inter_raw_f32"]), c["line"]
        assert oracle.raw_f64(*t, kernel=INTER, fused=FUSED) == f64_of_hex(c["ref_inter_raw_f64"]), c["line"]


def test_all_fp64_oracle_agrees_with_reference_fp64(oracle, golden_cases):
    for c in golden_cases:
        assert abs(oracle.log10_f64(*case_tuple(c)) - c["ref_intra_log10_f64"]) < 1e-9, c["line"]


def test_restated_scheduler_reproduces_reference_output(oracle, ref_regions):
    """schedule_pairhmm restated (routing, FP32/FP64 switch, result conversions) equals the
    reference's output bit for bit on every fixture pair: the 8 debug regions, seeded synthetic
    regions and the edge cases (N, short/long reads, many haplotypes, extreme qualities, IUPAC)."""
    n = 0
    for group, (pb, want) in ref_regions.items():
        got = np.concatenate([oracle.schedule_region(pb, g)[0].reshape(-1) for g in range(pb.n_regions)])
        assert np.array_equal(got, want), (group, float(np.nanmax(np.abs(got - want))))
        n += got.size
    assert n > 20000


def test_tables_match_reference_formulas(oracle):
    """ph2pr and the match-to-match table: spot values and monotonicity (context.h:50-60,98,138)."""
    assert oracle.lib.oracle_ph2pr_f64(10) == pytest.approx(0.1, rel=1e-15)
    assert oracle.lib.oracle_ph2pr_f32(20) == pytest.approx(0.01, rel=1e-7)
    assert oracle.lib.oracle_mm_f64(45, 45) == pytest.approx(1 - 2 * 10 ** -4.5, rel=1e-6)
    vals = [oracle.lib.oracle_mm_f32(q, q) for q in range(10, 60)]
    assert all(a <= b for a, b in zip(vals, vals[1:]))


def test_unfused_differs_from_fused_only_in_rounding(oracle, golden_cases):
    """The AVX2 build (no FMA) and the AVX-512 build differ by rounding only."""
    for c in golden_cases[:30]:
        t = case_tuple(c)
        a = oracle.raw_f32(*t, kernel=INTER, fused=FUSED)
        b = oracle.raw_f32(*t, kernel=INTER, fused=UNFUSED)
        assert abs(a - b) <= 1e-4 * abs(a)


def test_random_pairs_bit_exact_against_reference_build(oracle, ref):
    """Seeded random pairs against the compiled reference (only where the reference sources exist)."""
    rng = np.random.default_rng(99)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    pairs = []
    for _ in range(48):
        H, R = int(rng.integers(5, 400)), int(rng.integers(3, 260))
        hap = acgt[rng.integers(0, 4, H)].tobytes()
        read = bytearray(hap[: min(R, H)] + acgt[rng.integers(0, 4, max(0, R - H))].tobytes())
        for k in range(len(read)):
            if rng.random() < 0.03:
                read[k] = int(acgt[rng.integers(0, 4)])
        if rng.random() < 0.2:
            read[int(rng.integers(0, len(read)))] = ord("N")
        q, i, d, c = (rng.integers(lo, hi, R).astype(np.uint8).tobytes() for lo, hi in ((2, 42), (10, 46), (10, 46), (5, 15)))
        pairs.append((hap, bytes(read), q, i, d, c))
    for p in pairs:
        assert oracle.raw_f32(*p, kernel=INTRA) == ref.intra_raw_f32(*p)
        assert oracle.raw_f64(*p, kernel=INTRA) == ref.intra_raw_f64(*p)
    w = ref.width_f32
    clean = [p for p in pairs if b"N" not in p[1]][: (len(pairs) // w) * w]
    for g in range(0, len(clean) - w + 1, w):
        got = ref.inter(clean[g:g + w], raw=True)
        want = [oracle.raw_f32(*p, kernel=INTER) for p in clean[g:g + w]]
        assert np.array_equal(np.float32(got), np.float32(want))


def test_table_probabilities_bound_used_by_flush_free_fp64_steps(oracle):
    """The FP64 pass skips its flushes in steps whose inputs are all 0 or at least
    2^(-1022 + 44 (K + 1)); that bound rests on every nonzero probability the cell update multiplies
    by being at least 2^-44 (and none negative).  Checked over the whole tables."""
    import ctypes as C

    lib = oracle.lib
    lib.oracle_ph2pr_f64.restype = C.c_double
    lib.oracle_ph2pr_f64.argtypes = [C.c_int]
    lib.oracle_mm_f64.restype = C.c_double
    lib.oracle_mm_f64.argtypes = [C.c_int, C.c_int]
    vals = []
    for q in range(128):
        d = lib.oracle_ph2pr_f64(q)
        vals += [d, d / 3.0, 1.0 - d]                  # gap and base-quality terms, mismatch, match, gapm
    vals += [lib.oracle_mm_f64(i, j) for i in range(128) for j in range(128)]
    assert min(vals) >= 0.0
    assert min(v for v in vals if v > 0.0) >= 2.0 ** -44
