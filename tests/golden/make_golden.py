"""Regenerates the golden fixtures in this folder from the reference project (run where it exists).

Inputs read from the reference (paths inside the reference project):
  src/haplotypecaller/pairhmm/resource/pairhmm-testdata.txt  104 golden cases
      (hap read qual ins del gcp expected, qualities Phred+33; format of
       test/pairhmm_unittest.cpp:39-92)
  src/haplotypecaller/pairhmm/resource/pairhmm_debug.txt     8 real regions (format of
       test/assemble_log_parser.cpp:14-120), no stored expectations
  test/pairhmm_unittest.cpp:108-141                           two hand cases (ACGT, ACGTA at Q43)
Outputs of the reference's own kernels, compiled from its sources by oracle/build_ref.sh
(oracle/_ref/libphmm_ref.so, AVX-512 path), are stored beside the inputs:
  golden_cases.json     per case: the file's expected value, the intra kernel's FP32->FP64 result,
                        its FP64-only result, and the raw FP32/FP64 sums of the intra and inter
                        kernels (inter in groups of 16 / 8 with wrap-around for the last group)
  ref_regions.npz       packed regions (the 8 debug regions, seeded synthetic regions, edge cases)
                        and schedule_pairhmm's log10 output for each, [hap][read]

Usage: python tests/golden/make_golden.py [REFERENCE_ROOT]
"""
from __future__ import annotations

import json
import re
import struct
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle import Ref, build_ref  # noqa: E402
from oracle.oracle import reference_root as oracle_reference_root  # noqa: E402
from rovaca_b200 import synth  # noqa: E402
from rovaca_b200.pairhmm import PackedBatch, Region  # noqa: E402


def f32_hex(x: float) -> str:
    return struct.pack(">f", x).hex()


def f64_hex(x: float) -> str:
    return struct.pack(">d", x).hex()


def parse_testdata(path: Path) -> list[dict]:
    cases = []
    for ln, line in enumerate(path.read_text().splitlines()):
        if ln == 0 or not line.strip():
            continue
        f = line.split()
        if len(f) < 7:
            continue
        q = lambda s: [ord(ch) - 33 for ch in s]
        cases.append({"line": ln + 1, "hap": f[0], "read": f[1], "q": q(f[2]), "i": q(f[3]), "d": q(f[4]),
                      "c": q(f[5]), "expected": float(f[6])})
    return cases


def parse_debug_regions(path: Path) -> list[Region]:
    lines = path.read_text().splitlines()
    regions, k = [], 0
    while k < len(lines):
        if not lines[k].startswith("=== Region:"):
            k += 1
            continue
        nh = int(re.search(r"Haplotypes: (\d+)", lines[k + 1]).group(1))
        nr = int(re.search(r"Reads: (\d+)", lines[k + 2]).group(1))
        k += 3
        haps, reads, quals = [], [], {"read-qual": [], "read-ins-qual": [], "read-del-qual": [], "gcp": []}
        while len(haps) < nh:
            if re.match(r"^H\d+:", lines[k]):
                haps.append(lines[k].split(":", 1)[1].strip())
            k += 1
        while len(reads) < nr:
            if re.match(r"^R\d+:", lines[k]):
                reads.append(lines[k].split(":", 1)[1].strip())
                for _ in range(4):
                    k += 1
                    key, vals = lines[k].strip().split(":", 1)
                    quals[key].append([int(v) for v in vals.split()])
            k += 1
        regions.append(Region(haps, reads, quals["read-qual"], quals["read-ins-qual"], quals["read-del-qual"],
                              quals["gcp"]))
    return regions


def edge_regions(rng) -> list[Region]:
    """Cases the reference handles that the benchmark shapes do not reach."""
    acgt = np.frombuffer(b"ACGT", np.uint8)

    def seq(n):
        return acgt[rng.integers(0, 4, n)].tobytes()

    def quals(n, lo=2, hi=41):
        return rng.integers(lo, hi + 1, n).astype(np.uint8).tobytes()

    def reg(haps, reads, qlo=2, qhi=41, ins=45, gcp=10):
        return Region(haps, reads, [quals(len(r), qlo, qhi) for r in reads], [bytes([ins]) * len(r) for r in reads],
                      [bytes([ins]) * len(r) for r in reads], [bytes([gcp]) * len(r) for r in reads])

    out = []
    # reads with N, haplotypes with N (intra kernel: N matches everything)
    h = [seq(200), seq(180)]
    h_n = h[0][:50] + b"N" + h[0][51:120] + b"NN" + h[0][122:]
    r = [h[0][10:160], h[1][5:105], h[0][30:130][:40] + b"N" + h[0][71:130], seq(90)]
    out.append(reg([h[0], h_n, h[1]], r))
    # short reads (1..40 bases, one row per lane) and short haplotypes
    hs = [seq(n) for n in (1, 2, 7, 33, 64)]
    out.append(reg(hs, [hs[4][:n] if n <= 64 else seq(n) for n in (1, 2, 3, 16, 31, 32, 33, 40)]))
    # long reads: several 256-row stripes (257..768) against long haplotypes (up to 1536)
    base = seq(1536)
    out.append(reg([base, base[100:1300], base[:700] + seq(3) + base[700:1400]],
                   [base[20:20 + n] for n in (257, 300, 512, 513, 700, 768)]))
    # many haplotypes: the column stream of one read crosses many haplotype boundaries
    b2 = seq(400)
    out.append(reg([b2[k:k + 250 + k] for k in range(0, 120, 4)], [b2[30:180], b2[50:260], b2[0:120]]))
    # extreme qualities (0 and >= 128, masked with & 127) and high gap-continuation
    out.append(reg([b2[:300], b2[5:290]], [b2[40:190], b2[60:200]], qlo=0, qhi=200, ins=127, gcp=60))
    # non-ACGT letters (IUPAC codes compare as raw bytes in pairs without N)
    hm = bytearray(b2[:260])
    hm[100] = ord("R")
    hm[150] = ord("Y")
    rm = bytearray(b2[90:210])
    rm[10] = ord("R")
    out.append(reg([bytes(hm), b2[:260]], [bytes(rm), b2[50:200]]))
    return out


def main(reference_root: str | None = None) -> None:
    reference_root = reference_root or oracle_reference_root()
    if reference_root is None:
        raise SystemExit("pass the reference's source root or set REFERENCE_ROOT")
    res = Path(reference_root) / "src/haplotypecaller/pairhmm/resource"
    lib = build_ref(reference_root)
    if lib is None:
        raise SystemExit("reference sources not found; golden fixtures cannot be regenerated here")
    ref = Ref(lib)
    if ref.isa != 512:
        raise SystemExit("the fixtures record the reference's AVX-512 path; this host has no AVX-512")

    # ---- golden cases ----------------------------------------------------------------------
    cases = parse_testdata(res / "pairhmm-testdata.txt")
    hand = [{"line": 0, "hap": "ACGT", "read": "ACGT", "q": [43] * 4, "i": [43] * 4, "d": [43] * 4, "c": [43] * 4,
             "expected": -6.022797e-01},
            {"line": 0, "hap": "ACGTA", "read": "ACGTA", "q": [43] * 5, "i": [43] * 5, "d": [43] * 5, "c": [43] * 5,
             "expected": -0.69925308227539062}]
    allc = cases + hand
    tup = lambda c: (c["hap"].encode(), c["read"].encode(), bytes(c["q"]), bytes(c["i"]), bytes(c["d"]), bytes(c["c"]))
    for c in allc:
        t = tup(c)
        c["ref_intra_log10"] = ref.intra_log10(*t, use_double=False)
        c["ref_intra_log10_f64"] = ref.intra_log10(*t, use_double=True)
        c["ref_intra_raw_f32"] = f32_hex(ref.intra_raw_f32(*t))
        c["ref_intra_raw_f64"] = f64_hex(ref.intra_raw_f64(*t))
    n = len(allc)
    for key, w, dbl in (("ref_inter_raw_f32", ref.width_f32, False), ("ref_inter_raw_f64", ref.width_f64, True)):
        for g in range(0, n, w):
            idx = [(g + k) % n for k in range(w)]
            vals = ref.inter([tup(allc[j]) for j in idx], dbl=dbl, raw=True)
            for j, v in zip(idx[: n - g] if g + w > n else idx, vals):
                allc[j][key] = f64_hex(float(v)) if dbl else f32_hex(float(np.float32(v)))
    (HERE / "golden_cases.json").write_text(json.dumps({"source": "pairhmm-testdata.txt + pairhmm_unittest.cpp "
                                                        "hand cases; reference outputs from oracle/_ref (AVX-512)",
                                                        "cases": allc}, indent=0))

    # ---- regions through the reference's scheduler -----------------------------------------
    rng = np.random.default_rng(20260)
    groups = {
        "debug": parse_debug_regions(res / "pairhmm_debug.txt"),
        "config0": [synth.config0().region(0)],
        "config1": [synth.config1(3, seed=11).region(g) for g in range(3)],
        "config2": [synth.config2(1, seed=12).region(0)],
        "edge": edge_regions(rng),
    }
    arrays = {}
    for name, regs in groups.items():
        pb = PackedBatch.from_regions(regs)
        outs = [ref.schedule_region(pb, g, 0.02, 0.02).reshape(-1) for g in range(pb.n_regions)]
        for f in ("n_haps", "n_reads", "hap_bases", "hap_off", "read_bases", "read_qual", "read_ins", "read_del",
                  "read_gcp", "read_off"):
            arrays[f"{name}.{f}"] = getattr(pb, f)
        arrays[f"{name}.ref_log10"] = np.concatenate(outs)
    np.savez_compressed(HERE / "ref_regions.npz", **arrays)

    # ---- region-path helpers: PCR model and tandem repeats (pairhmm_internal.cpp) ----------
    import ctypes as C

    lib = ref.lib
    lib.ref_tandem_repeat.restype = C.c_int
    prng = np.random.default_rng(4242)
    reads = []
    for k in range(120):
        n = int(prng.integers(1, 160))
        unit = prng.choice(list(b"ACGT"), int(prng.integers(1, 9)))
        if k % 3 == 0:
            s = prng.choice(list(b"ACGT"), n)
        elif k % 3 == 1:
            s = np.resize(unit, n)
        else:
            s = np.concatenate([prng.choice(list(b"ACGT"), 12), np.resize(unit, n), prng.choice(list(b"AC"), 9)])[:n]
        reads.append(bytes(np.asarray(s, np.uint8)))
    helpers = []
    for s in reads:
        n = len(s)
        rec = {"bases": s.decode(), "repeat": [lib.ref_tandem_repeat(s, n, o, 1) for o in range(max(n - 1, 0))]}
        for model, name in ((1, "HOSTILE"), (2, "AGGRESSIVE"), (3, "CONSERVATIVE")):
            g = (C.c_uint8 * n)(*([45] * n))
            lib.ref_pcr_model(s, n, g, model, 1)
            rec[name] = list(bytes(g))
        helpers.append(rec)
    (HERE / "region_helpers.json").write_text(json.dumps({"source": "apply_pcr_error_model_rolling and "
                                                          "find_tandem_repeat_units_rolling from oracle/_ref",
                                                          "reads": helpers}))
    print(f"wrote {HERE / 'golden_cases.json'} ({len(allc)} cases) and {HERE / 'ref_regions.npz'} "
          f"({', '.join(f'{k}: {len(v)}' for k, v in groups.items())} regions)")


if __name__ == "__main__":
    main(*sys.argv[1:])
