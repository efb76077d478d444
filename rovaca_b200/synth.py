"""Seeded synthetic active regions with the shapes of the benchmark configurations.

No real data travels with this repository; these generators stand in for it.  Every region is
built the same way, as HaplotypeCaller's active regions are: a uniform-ACGT reference window of
the region's haplotype length, every haplotype that same window edited with its own SNPs and short
indels (so haplotypes of one region span the same locus), reads sampled from random haplotypes at
uniform offsets with substitution errors (a read longer than its haplotype continues into the
reference flank), and per-base qualities drawn uniformly.  numpy's PCG64 generator, seeded per
configuration.

  config 0  one region: 8 haplotypes of 300-320 bp (0-3 SNPs, 0-2 indels of 1-10 bp), 64 reads of
            151 bp, 1% errors, base quality U[10,40], ins/del 45, GCP 10
  config 1  2,000 regions: reads U[10,500] of length U[100,250], base quality U[2,41], ins/del 45,
            GCP 10, 1% errors; haplotypes U[2,32] of length 150-600
  config 2  underflow stress: 500 regions x 200 reads of 250 bp, base quality U[2,15], 5% errors,
            16 haplotypes of 800-1,000 bp carrying 5-10 indels each
  config 4  WGS-like mixture: depth lognormal (median 60, sigma 0.5, clipped to [5, 2000]), reads of
            150 bp (90%) or 250 bp (10%), haplotypes geometric (mean 6, max 128) of 200-1,200 bp,
            2% of regions drawn from config 2's regime
"""
from __future__ import annotations

import numpy as np

from .pairhmm import PackedBatch

ACGT = np.frombuffer(b"ACGT", dtype=np.uint8)


def _edit(rng, seq: np.ndarray, n_snp: int, n_indel: int, indel_len: tuple[int, int]) -> np.ndarray:
    s = seq.copy()
    if n_snp and len(s):
        pos = rng.integers(0, len(s), n_snp)
        s[pos] = (s[pos] + rng.integers(1, 4, n_snp)) % 4
    for _ in range(n_indel):
        if len(s) < 2:
            break
        p = int(rng.integers(0, len(s)))
        ln = int(rng.integers(indel_len[0], indel_len[1] + 1))
        if rng.random() < 0.5:
            s = np.concatenate([s[:p], rng.integers(0, 4, ln).astype(np.uint8), s[p:]])
        else:
            s = np.concatenate([s[:p], s[p + ln:]])
    return s


def _region(rng, n_haps: int, hap_len: tuple[int, int], n_reads: int, read_lens: np.ndarray,
            qual: tuple[int, int], err: float, snps: tuple[int, int], indels: tuple[int, int],
            indel_len: tuple[int, int] = (1, 10)) -> dict:
    lo, hi = hap_len
    L = int(rng.integers(lo, hi + 1))                       # the region's window
    flank = int(read_lens.max()) if n_reads else 0
    ref = rng.integers(0, 4, L + flank).astype(np.uint8)     # window + right flank
    haps = []
    for _ in range(n_haps):
        h = _edit(rng, ref[:L], int(rng.integers(snps[0], snps[1] + 1)),
                  int(rng.integers(indels[0], indels[1] + 1)), indel_len)
        if len(h) > hi:
            h = h[:hi]
        if len(h) < lo:
            h = np.concatenate([h, ref[L:L + lo - len(h)]])
        haps.append(h)
    hlen = np.array([len(h) for h in haps], np.int64)
    # each haplotype continued by the reference flank, for reads that run past its end
    ext = [np.concatenate([h, ref[L:]]) for h in haps]
    elen = np.array([len(e) for e in ext], np.int64)
    eoff = np.concatenate([[0], np.cumsum(elen)])
    ecat = np.concatenate(ext)
    R = read_lens.astype(np.int64)
    src = rng.integers(0, n_haps, n_reads)
    off = (rng.random(n_reads) * np.maximum(hlen[src] - R + 1, 1)).astype(np.int64)
    roff = np.concatenate([[0], np.cumsum(R)])
    tot = int(roff[-1])
    idx_in_read = np.arange(tot) - np.repeat(roff[:-1], R)
    pos = np.minimum(np.repeat(off, R) + idx_in_read, np.repeat(elen[src] - 1, R))
    bases = ecat[np.repeat(eoff[src], R) + pos]
    flip = rng.random(tot) < err
    bases = np.where(flip, (bases + rng.integers(1, 4, tot)) % 4, bases).astype(np.uint8)
    return {
        "hap_bases": ACGT[np.concatenate(haps)], "hap_len": hlen, "read_bases": ACGT[bases], "read_len": R,
        "qual": rng.integers(qual[0], qual[1] + 1, tot).astype(np.uint8),
    }


def _pack(regions: list[dict], ins: int = 45, gcp: int = 10) -> PackedBatch:
    nh = np.array([len(r["hap_len"]) for r in regions], np.uint32)
    nr = np.array([len(r["read_len"]) for r in regions], np.uint32)
    hap_bases = np.concatenate([r["hap_bases"] for r in regions])
    read_bases = np.concatenate([r["read_bases"] for r in regions])
    hap_off = np.concatenate([[0], np.cumsum(np.concatenate([r["hap_len"] for r in regions]))]).astype(np.uint64)
    read_off = np.concatenate([[0], np.cumsum(np.concatenate([r["read_len"] for r in regions]))]).astype(np.uint64)
    qual = np.concatenate([r["qual"] for r in regions])
    n = read_bases.size
    return PackedBatch(nh, nr, hap_bases, hap_off, read_bases, qual, np.full(n, ins, np.uint8),
                       np.full(n, ins, np.uint8), np.full(n, gcp, np.uint8), read_off)


def config0(seed: int = 0) -> PackedBatch:
    rng = np.random.default_rng([seed, 0])
    return _pack([_region(rng, 8, (300, 320), 64, np.full(64, 151), (10, 40), 0.01, (0, 3), (0, 2))])


def config1(n_regions: int = 2000, seed: int = 1) -> PackedBatch:
    rng = np.random.default_rng([seed, 1])
    regs = []
    for _ in range(n_regions):
        n_reads = int(rng.integers(10, 501))
        regs.append(_region(rng, int(rng.integers(2, 33)), (150, 600), n_reads, rng.integers(100, 251, n_reads),
                            (2, 41), 0.01, (0, 3), (0, 2)))
    return _pack(regs)


def _config2_region(rng, n_reads: int = 200) -> dict:
    return _region(rng, 16, (800, 1000), n_reads, np.full(n_reads, 250), (2, 15), 0.05, (0, 3), (5, 10))


def config2(n_regions: int = 500, seed: int = 2, n_reads: int = 200) -> PackedBatch:
    rng = np.random.default_rng([seed, 2])
    return _pack([_config2_region(rng, n_reads) for _ in range(n_regions)])


def config4(n_regions: int = 200_000, seed: int = 4, sigma: float = 0.5) -> PackedBatch:
    rng = np.random.default_rng([seed, 4])
    regs = []
    for _ in range(n_regions):
        if rng.random() < 0.02:
            regs.append(_config2_region(rng))
            continue
        depth = int(np.clip(round(60 * np.exp(sigma * rng.standard_normal())), 5, 2000))
        n_haps = int(min(rng.geometric(1 / 6), 128))
        R = np.where(rng.random(depth) < 0.9, 150, 250)
        regs.append(_region(rng, n_haps, (200, 1200), depth, R, (2, 41), 0.01, (0, 3), (0, 2)))
    return _pack(regs)


def make(config: int, scale: float = 1.0, seed: int | None = None) -> PackedBatch:
    """Config by number; scale < 1 draws proportionally fewer regions (same per-region shapes)."""
    kw = {} if seed is None else {"seed": seed}
    if config == 0:
        return config0(**kw)
    if config == 1:
        return config1(max(1, int(round(2000 * scale))), **kw)
    if config == 2:
        return config2(max(1, int(round(500 * scale))), **kw)
    if config == 4:
        return config4(max(1, int(round(200_000 * scale))), **kw)
    raise ValueError(f"no generator for config {config}")


def genotyping_regions(n_regions: int, seed: int = 5, depth: int = 40, read_len: int = 150,
                       window: tuple[int, int] = (300, 400), sites: tuple[int, int] = (1, 3)):
    """Regions with known variant sites for the genotyping path, one diploid sample each.

    Each region: a reference window with 1-3 variant sites (a SNP, or an insertion or deletion of
    1-6 bases) at distinct positions and a true genotype per site (0/0, 0/1 or 1/1, the two true
    haplotypes phased at random); candidate haplotypes are the reference and every combination of
    alternate alleles; reads of `read_len` come from the two true haplotypes at uniform offsets with
    1% substitution errors and base qualities U[10,40].  Each site is one event with alleles
    {ref, alt}; a haplotype maps to the alt allele when it carries the site's alternate.
    Returns dicts with haplotypes, reads, quals, mapq, events [(2, allele of each haplotype)] and
    truth (genotype index per site: 0 hom-ref, 1 het, 2 hom-alt)."""
    rng = np.random.default_rng([seed, 5])
    out = []
    for _ in range(n_regions):
        L = int(rng.integers(window[0], window[1] + 1))
        ref = rng.integers(0, 4, L + read_len).astype(np.uint8)
        n_sites = int(rng.integers(sites[0], sites[1] + 1))
        pos = np.sort(rng.choice(np.arange(20, L - 20, 25), n_sites, replace=False))
        kinds = []
        for p in pos:
            k = rng.integers(0, 3)
            if k == 0:
                kinds.append(("snp", int(p), int((ref[p] + rng.integers(1, 4)) % 4)))
            elif k == 1:
                kinds.append(("ins", int(p), rng.integers(0, 4, int(rng.integers(1, 7))).astype(np.uint8)))
            else:
                kinds.append(("del", int(p), int(rng.integers(1, 7))))

        def build(carry):
            s, last = [], 0
            for (kind, p, x), c in zip(kinds, carry):
                if not c:
                    continue
                s.append(ref[last:p])
                if kind == "snp":
                    s.append(np.array([x], np.uint8))
                    last = p + 1
                elif kind == "ins":
                    s.append(ref[p:p + 1])
                    s.append(x)
                    last = p + 1
                else:
                    s.append(ref[p:p + 1])
                    last = p + 1 + x
            s.append(ref[last:L])
            return np.concatenate(s)

        combos = [tuple((m >> i) & 1 for i in range(n_sites)) for m in range(1 << n_sites)]
        haps = [build(c) for c in combos]
        truth = [int(g) for g in rng.integers(0, 3, n_sites)]
        phase = [(0, 0) if g == 0 else ((1, 1) if g == 2 else ((0, 1) if rng.random() < 0.5 else (1, 0))) for g in truth]
        true_haps = [combos.index(tuple(ph[k] for ph in phase)) for k in range(2)]
        reads, quals = [], []
        for _ in range(depth):
            h = haps[true_haps[int(rng.integers(0, 2))]]
            ext = np.concatenate([h, ref[L:]])
            o = int(rng.integers(0, max(1, len(h) - read_len + 1)))
            r = ext[o:o + read_len].copy()
            flip = rng.random(len(r)) < 0.01
            r[flip] = (r[flip] + rng.integers(1, 4, int(flip.sum()))) % 4
            reads.append(ACGT[r].tobytes())
            quals.append(rng.integers(10, 41, len(r)).astype(np.uint8).tobytes())
        events = [(2, np.array([c[i] for c in combos], np.int8)) for i in range(n_sites)]
        out.append({"haplotypes": [ACGT[h].tobytes() for h in haps], "reads": reads, "quals": quals,
                    "mapq": np.full(depth, 60, np.uint8), "events": events, "truth": truth})
    return out


def sw_realignment(pb: PackedBatch, best_hap: np.ndarray | None = None):
    """Every read of every region against one haplotype of its own region, as HaplotypeCaller
    realigns reads to their best haplotype: best_hap[q] (index within the read's region) when given,
    else haplotype q mod n_haps of the region.  Returns an ``sw.SwBatch`` over the batch's base buffers."""
    from .sw import SW_ITEM_DTYPE, SwBatch

    nh = pb.n_haps.astype(np.int64)
    nr = pb.n_reads.astype(np.int64)
    g = np.repeat(np.arange(len(nr)), nr)
    first_read = np.concatenate([[0], np.cumsum(nr)[:-1]])
    first_hap = np.concatenate([[0], np.cumsum(nh)[:-1]])
    local = np.arange(int(nr.sum())) - first_read[g]
    pick = local % nh[g] if best_hap is None else np.asarray(best_hap, np.int64)
    h = first_hap[g] + pick
    hap_off = pb.hap_off.astype(np.uint64)
    read_off = pb.read_off.astype(np.uint64)
    items = np.zeros(len(g), SW_ITEM_DTYPE)
    items["hap_offset"] = hap_off[h]
    items["hap_len"] = (hap_off[h + 1] - hap_off[h]).astype(np.uint32)
    items["read_offset"] = read_off[:-1]
    items["read_len"] = np.diff(read_off).astype(np.uint32)
    return SwBatch(pb.hap_bases, pb.read_bases, items)

