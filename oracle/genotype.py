"""Genotyping restatement for the checker (test infrastructure only; the engine never imports it).

Restates, for one sample and ploidy 2, what HaplotypeCaller does after call_pairhmm:
  * normalise / drop poorly modelled reads / kept reads first
      src/haplotypecaller/pairhmm/pairhmm_internal.cpp:23-44,248-258,489-508
  * haplotype -> allele marginalisation: per read the maximum over the allele's haplotypes,
    -inf when none, NaN never wins            src/haplotypecaller/genotype/allele_likelihoods.hpp:702-730
  * diploid genotype likelihoods: genotype (a <= b) at index b(b+1)/2 + a,
      per read  lk(a) + log10(2)                   if a == b
                approximate_log10sum(lk(a), lk(b)) otherwise
      GL = (sum over reads, from 0 in read order) - reads * log10(2)
                                              src/haplotypecaller/genotype/genotype_likelihood_calculator.cpp:59-100,
                                              genotype_likelihood_calculator.h:90-142
  * approximate_log10sum(a, b) = max + table[round((max - min) * 1e4)] below a difference of 8, the
    Jacobian table log10(1 + 10^(-k/1e4))   src/haplotypecaller/common/utils/math_utils.cpp:280-290,
                                              math_utils.h:209-242
  * best haplotype of a read for the realignment: search_best_allele with can_be_reference and
    priorities -- the running maximum and runner-up over the haplotypes (strict >), then, when the
    runner-up is within 0.2 (log10) of the best, the haplotypes within 0.2 of it ranked by priority
    (strict >)                                src/haplotypecaller/genotype/allele_likelihoods.hpp:589-658
    HaplotypeCaller's priority: (is_reference ? 1 : 0) + 1 - cigar elements
                                              src/haplotypecaller/genotype/utils/assembly_based_caller_utils.cpp:150-155
The reference's own unit test (genotype/test/genotype_likelihood_calculator_unit_test.cpp:86-130)
defines GL as sum_r [log10sum_c(lk(r, a_c) + log10(count_c)) - log10(2)] and accepts 1e-4; the
tests here hold this restatement to that definition.
"""
from __future__ import annotations

import math

import numpy as np

_JAC = None
_INV_STEP = 1.0 / 0.0001
LOG10_TWO = math.log10(2.0)


def jacobian() -> np.ndarray:
    global _JAC
    if _JAC is None:
        k = np.arange(80001, dtype=np.float64)
        _JAC = np.array([math.log10(1.0 + math.pow(10.0, -0.0001 * float(i))) for i in k], np.float64)
    return _JAC


def _round_half_away(x: float) -> int:
    """std::round for the non-negative differences used here (x - floor(x) is exact)."""
    f = math.floor(x)
    return int(f) + (1 if x - f >= 0.5 else 0)


def approx_log10sum(a: float, b: float) -> float:
    if a > b:
        a, b = b, a
    if a == -math.inf:
        return b
    diff = b - a
    return b + (float(jacobian()[_round_half_away(diff * _INV_STEP)]) if diff < 8.0 else 0.0)


def normalize_filter(lk_hr: np.ndarray, read_len) -> tuple[np.ndarray, np.ndarray]:
    """[hap][read] -> (matrix with kept reads first and NaN after, keep mask)."""
    M, N = lk_hr.shape
    out = np.full((M, N), np.nan)
    keep = np.zeros(N, bool)
    k = 0
    for r in range(N):
        row = lk_hr[:, r].copy()
        if M:
            best = row[0]
            for x in row[1:]:
                if best < x:
                    best = x
            cmp = best - 4.5
            row = np.array([cmp if x < cmp else x for x in row])
        fin = [x for x in row if not math.isnan(x)]
        b = max(fin) if fin else -math.inf
        min_lk = min(2.0, math.ceil(read_len[r] * 0.02)) * -4.0
        if not (b < min_lk):
            keep[r] = True
            out[:, k] = row
            k += 1
    return out, keep


def marginalize(norm_hr: np.ndarray, n_kept: int, hap_allele, n_alleles: int) -> np.ndarray:
    """[allele][kept read] maximum over each allele's haplotypes (-inf if none)."""
    alk = np.full((n_alleles, n_kept), -math.inf)
    for h, a in enumerate(hap_allele):
        if a < 0:
            continue
        for r in range(n_kept):
            x = norm_hr[h, r]
            if x > alk[a, r]:
                alk[a, r] = x
    return alk


def genotype_likelihoods(alk: np.ndarray) -> np.ndarray:
    A, K = alk.shape
    gl = np.empty(A * (A + 1) // 2)
    for b in range(A):
        for a in range(b + 1):
            s = 0.0
            for r in range(K):
                s += (alk[a, r] + LOG10_TWO) if a == b else approx_log10sum(alk[a, r], alk[b, r])
            gl[b * (b + 1) // 2 + a] = s - float(K) * LOG10_TWO
    return gl


def best_genotype(gl: np.ndarray) -> int:
    arg = 0
    for g in range(1, len(gl)):
        if gl[g] > gl[arg]:
            arg = g
    return arg


def genotype_region(lk_hr: np.ndarray, read_len, events):
    """events: [(n_alleles, hap_allele)] -> [(gl, best, allele_lk)] after normalise/filter."""
    norm, keep = normalize_filter(lk_hr, read_len)
    K = int(keep.sum())
    res = []
    for A, ha in events:
        alk = marginalize(norm, K, list(ha), int(A))
        gl = genotype_likelihoods(alk)
        res.append((gl, best_genotype(gl), alk))
    return res, norm, keep


INFORMATIVE_LOG10 = 0.2  # s_log_10_informative_threshold, allele_likelihoods.hpp:27


def search_best_allele(values, priorities) -> int:
    """Index of the best allele (haplotype) for one read's likelihoods, ties within the informative
    threshold broken by priority."""
    M = len(values)
    best, second = 0, 0
    bl, sl = float(values[0]), -math.inf
    for a in range(1, M):
        c = float(values[a])
        if c > bl:
            second, best, sl, bl = best, a, bl, c
        elif c > sl:
            second, sl = a, c
    if bl - sl < INFORMATIVE_LOG10:
        bp, sp = float(priorities[best]), float(priorities[second])
        for a in range(M):
            c = float(values[a])
            if a == best or bl - c > INFORMATIVE_LOG10:
                continue
            cp = float(priorities[a])
            if cp > bp:
                second, best, sp, bp = best, a, bp, cp
            elif cp > sp:
                second, sp = a, cp
    return best

