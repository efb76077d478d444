"""The genotyping restatement of the checker (oracle/genotype.py) against the reference's own
compiled genotyping code (oracle/_ref/libgenotype_ref.so: AlleleLikelihoods::marginalize and
GenotypeLikelihoodCalculator, built from the reference sources by oracle/build_ref_genotype.sh), bit
for bit, and against the definition of the reference's unit test
(genotype/test/genotype_likelihood_calculator_unit_test.cpp:86-130: GL = sum_r [log10sum_c(lk(r, a_c) +
log10(count_c)) - log10(2)], accepted within 1e-4) and its genotype order.  No GPU."""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import genotype as G


def _unit_test_gl(alk: np.ndarray, a: int, b: int) -> float:
    comps = [(a, 2)] if a == b else [(a, 1), (b, 1)]
    total = 0.0
    for r in range(alk.shape[1]):
        vals = [alk[x, r] + math.log10(c) for x, c in comps]
        m = max(vals)
        s = m + math.log10(sum(10.0 ** (v - m) for v in vals)) if m != -math.inf else -math.inf
        total += s - math.log10(2)
    return total


@pytest.mark.parametrize("alleles", [1, 2, 5, 6])
@pytest.mark.parametrize("reads", [0, 1, 10, 100])
def test_genotype_likelihoods_match_reference_definition(alleles, reads):
    rng = np.random.default_rng(alleles * 1000 + reads)
    alk = -rng.exponential(3.0, (alleles, reads))
    gl = G.genotype_likelihoods(alk)
    assert len(gl) == alleles * (alleles + 1) // 2
    for b in range(alleles):
        for a in range(b + 1):
            assert abs(gl[b * (b + 1) // 2 + a] - _unit_test_gl(alk, a, b)) < 1e-4


def test_genotype_order_is_vcf_order():
    # (0,0) (0,1) (1,1) (0,2) (1,2) (2,2): an allele with all the support wins at its hom index
    alk = np.array([[-9.0] * 20, [-9.0] * 20, [-0.1] * 20])
    gl = G.genotype_likelihoods(alk)
    assert G.best_genotype(gl) == 5
    alk[1, :10], alk[2, :10] = -0.1, -9.0  # half the reads for allele 1, half for allele 2
    assert G.best_genotype(G.genotype_likelihoods(alk)) == 4  # het (1,2)


def test_approximate_log10sum_accuracy_and_edges():
    rng = np.random.default_rng(3)
    for _ in range(2000):
        a, b = -rng.exponential(5.0, 2)
        exact = math.log10(10 ** a + 10 ** b)
        assert abs(G.approx_log10sum(a, b) - exact) < 1e-4
    assert G.approx_log10sum(-math.inf, -2.0) == -2.0
    assert G.approx_log10sum(-1.0, -20.0) == -1.0  # difference beyond 8: the larger value


def test_marginalisation_takes_the_best_haplotype_and_skips_nan():
    norm = np.array([[-1.0, -3.0, np.nan], [-2.0, np.nan, np.nan], [-0.5, -4.0, np.nan]])
    alk = G.marginalize(norm, 2, [0, 0, 1], 3)
    assert alk[0].tolist() == [-1.0, -3.0] and alk[1].tolist() == [-0.5, -4.0]
    assert alk[2].tolist() == [-math.inf, -math.inf]


def test_best_haplotype_follows_reference_unit_test_rule():
    """With the reference-allele priority (1 for the reference, 0 otherwise) the best allele is the
    most likely one unless the reference is within 0.2 of it, then the reference
    (allele_likelihoods_unit_test.cpp:106-163, testBestAlleles)."""
    import random

    from oracle.genotype import search_best_allele

    rng = random.Random(3)
    for _ in range(3000):
        M = rng.randint(1, 8)
        vals = [round(-rng.random() * 3, rng.choice([1, 2, 6])) for _ in range(M)]
        ref = rng.randrange(M)
        prio = [1.0 if a == ref else 0.0 for a in range(M)]
        best_idx, best_lk = -1, float("-inf")
        for a, v in enumerate(vals):
            if v > best_lk:
                best_idx, best_lk = a, v
        override = ref != best_idx and best_lk - vals[ref] < 0.2
        assert search_best_allele(vals, prio) == (ref if override else best_idx), (vals, ref)


def test_best_haplotype_priorities_break_ties():
    from oracle.genotype import search_best_allele

    assert search_best_allele([-1.0, -1.1, -5.0], [0, 2, 9]) == 1      # -5 is outside the threshold
    assert search_best_allele([-1.0, -1.5], [0, 9]) == 0               # not within 0.2: likelihood wins
    assert search_best_allele([-1.0, -1.0, -1.0], [3, 1, 3]) == 0      # equal priorities keep the first
    assert search_best_allele([-2.0], [0]) == 0


def test_restatement_equals_the_reference_build_bit_for_bit(genotype_ref):
    """1,000 random events: 1-6 alleles, 0-500 reads, 1-16 haplotypes (some mapped to no allele),
    NaN likelihoods and whole NaN columns; allele likelihoods and genotype likelihoods identical."""
    rng = np.random.default_rng(2024)
    for k in range(1000):
        H = int(rng.integers(1, 17))
        N = int(rng.integers(0, 501)) if k % 10 == 0 else int(rng.integers(0, 80))
        A = int(rng.integers(1, 7))
        lk = -rng.exponential(rng.choice([0.5, 3.0, 20.0]), (H, N))
        if N and k % 3 == 0:
            lk[rng.integers(0, H, 3), rng.integers(0, N, 3)] = np.nan
        if N and k % 7 == 0:
            lk[:, rng.integers(0, N)] = np.nan
        ha = rng.integers(-1, A, H).astype(np.int8)
        alk_ref, gl_ref = genotype_ref.genotype(lk, ha, A)
        alk = G.marginalize(lk, N, list(ha), A)
        gl = G.genotype_likelihoods(alk)
        assert np.array_equal(alk, alk_ref, equal_nan=True), k
        assert np.array_equal(gl, gl_ref, equal_nan=True), k
        assert G.best_genotype(gl) == G.best_genotype(gl_ref)
