"""Regenerates tests/golden/sw_golden.json from the reference's Smith-Waterman aligner (run where the
reference project exists).

The expected outputs come from the reference's own aligner compiled from its sources by
oracle/build_ref_sw.sh (oracle/_ref/libsw_ref.so: ro_sw_avx512_run and its int16 / int32 kernels),
called the way AlignmentUtils::create_read_aligned_to_ref calls it (seq1 = haplotype, seq2 = read).
Inputs:
  * the haplotype and read sequences of the reference's own test
    src/haplotypecaller/genotype/test/alignment_utils_unit_test.cpp (make_test_data, read from
    that file here), with the genotyping parameters;
  * seeded synthetic pairs: reads cut from a random haplotype with substitutions and indels, random
    reads, the int16/int32 switch boundaries (read length 15/16/17, min length x match around
    32767), empty sequences, lengths 2047 and 2048 (refused), parameters that wrap in 16 bits;
    each under the genotyping and assembly parameters (lib/sw_avx/sw_avx.c:14-15) and the
    variants 0 (the reference's choice), 1 (int32 kernel) and 2 (int16 kernel).

Usage: python tests/golden/make_sw_golden.py [REFERENCE_ROOT]
"""
from __future__ import annotations

import json
import random
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle import SwRef, build_ref_sw, cigar_string  # noqa: E402
from oracle.oracle import reference_root as oracle_reference_root  # noqa: E402

GENOTYPING = SwRef.GENOTYPING
ASSEMBLY = SwRef.ASSEMBLY


def test_file_pairs(ref_root: Path) -> list[tuple[bytes, bytes]]:
    """(haplotype, read) pairs of make_test_data in alignment_utils_unit_test.cpp."""
    src = (ref_root / "src/haplotypecaller/genotype/test/alignment_utils_unit_test.cpp").read_text()
    body = src[src.index("::make_test_data("):]
    lits = {}
    for m in re.finditer(r'const char\*\s+(\w+)\s*=\s*((?:"[^"]*"\s*)+);', body):
        lits.setdefault(m.group(1), "".join(re.findall(r'"([^"]*)"', m.group(2))).encode())
    hap = lits["hap"]
    pairs = [(hap, hap)]
    for name in ("bases", "front_padded_bases", "back_padded_bases"):
        pairs.append((hap, lits[name]))
    pairs.append((lits["hap_bases"], lits["bad_sw_read_bases"]))
    return pairs


def mutate(rng: random.Random, s: bytes, rate: float) -> bytes:
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


def synthetic_pairs(rng: random.Random) -> list[tuple[bytes, bytes, tuple, int]]:
    def rnd(n):
        return bytes(rng.choice(b"ACGT") for _ in range(n))

    out = []
    for _ in range(120):
        h = rnd(rng.randint(20, 500))
        st = rng.randint(0, len(h) // 2)
        ln = rng.randint(1, min(251, len(h) - st))
        r = mutate(rng, h[st:st + ln], rng.choice([0.0, 0.01, 0.05, 0.2]))
        out.append((h, r, rng.choice([GENOTYPING, ASSEMBLY]), 0))
    for _ in range(20):
        out.append((rnd(rng.randint(1, 300)), bytes(rng.choice(b"ACGTN") for _ in range(rng.randint(1, 160))),
                    rng.choice([GENOTYPING, ASSEMBLY]), 0))
    # the int16 / int32 switch: read length 15/16/17; min length x match around INT16_MAX
    h = rnd(400)
    for ln in (15, 16, 17):
        for v in (0, 1, 2):
            out.append((h, mutate(rng, h[100:100 + ln], 0.05), GENOTYPING, v))
    for ln in (163, 164):
        for v in (0, 1, 2):
            out.append((h, mutate(rng, h[50:50 + ln], 0.03), ASSEMBLY, v))
    # empty sequences
    for hap, read in ((b"", b""), (b"ACGT", b""), (b"", b"ACGT"), (b"A", b"A"), (b"A", b"C"), (b"", b"A" * 20)):
        out.append((hap, read, GENOTYPING, 0))
    # long sequences: 2047 accepted, 2048 refused
    h = rnd(2047)
    out.append((h, mutate(rng, h[300:450], 0.02), GENOTYPING, 0))
    out.append((h, mutate(rng, h[:1000], 0.02), ASSEMBLY, 0))
    out.append((h, mutate(rng, h, 0.01)[:2047], GENOTYPING, 0))
    out.append((h[:1500], rnd(700), GENOTYPING, 0))
    out.append((h + b"A", h[:150], GENOTYPING, 0))
    out.append((h[:150], (h + b"C")[:2048], GENOTYPING, 0))
    # parameters that wrap in 16 bits, and small unit scores
    for prm in ((100, 50, 20, 10), (300, -200, -400, -300), (1, -1, -2, -1), (5, -4, -10, -10)):
        hh = rnd(300)
        for v in (0, 1, 2):
            out.append((hh, mutate(rng, hh[40:200], 0.05), prm, v))
    return out


def main(ref_root: str | None = None) -> None:
    ref_root = ref_root or oracle_reference_root()
    if ref_root is None:
        raise SystemExit("pass the reference's source root or set REFERENCE_ROOT")
    build_ref_sw(ref_root)
    ref = SwRef()
    rng = random.Random(20240611)
    cases = []
    for k, (h, r) in enumerate(test_file_pairs(Path(ref_root))):
        cases.append((f"alignment_utils_unit_test[{k}]", h, r, GENOTYPING, 0))
    for k, (h, r, p, v) in enumerate(synthetic_pairs(rng)):
        cases.append((f"synthetic[{k}]", h, r, p, v))
    rows = []
    for name, h, r, p, v in cases:
        sc, off, mi, mj, cig = ref.align(h, r, p, v)
        rows.append({"name": name, "hap": h.decode(), "read": r.decode(), "params": list(p), "variant": v,
                     "int32": ref.uses_int32(len(h), len(r), p[0]), "score": sc, "offset": off, "max_i": mi,
                     "max_j": mj, "cigar": cigar_string(cig), "ops": cig})
    (HERE / "sw_golden.json").write_text(json.dumps({"cases": rows}, separators=(",", ":")) + "\n")
    print(f"sw_golden.json: {len(rows)} cases")


if __name__ == "__main__":
    main(*sys.argv[1:])
