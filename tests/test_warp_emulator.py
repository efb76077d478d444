"""The engine's wavefront kernels run on the CPU: tests/native/warp_emu.cpp compiles their device
code (rovaca_b200/csrc/phmm_warp32.cuh, phmm_warp64.cuh and what they include) with g++ and runs each
class on one emulated warp, 32 host threads standing for the lanes (tests/native/warp_emu_shim.h),
over a batch the engine's own planner cuts.  Results must equal the oracle's pair for pair, as the GPU
tests require: equal raw sums (|log10 diff| <= 1e-12) and the same FP32 -> FP64 decisions.

The emulator's cost grows with the haplotype columns a warp streams, not with read length, so the
batches pair long reads (every rows-per-lane shape, multi-stripe reads up to 768) with short
haplotypes.  One region per kernel mode: equal constant gap qualities (mode 0), per-row and unequal
constant gap qualities (mode 1), N in reads and haplotypes (intra), and bytes outside A/C/G/T/N
(the inter kernel's checked path)."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import assert_same_values
from rovaca_b200.pairhmm import PackedBatch, Region

ROOT = Path(__file__).resolve().parent.parent
NATIVE = ROOT / "tests" / "native"
BIN = NATIVE / "_build" / "warp_emu"
CSRC = ROOT / "rovaca_b200" / "csrc"
EXACT = 1e-12
LENS = (17, 40, 70, 100, 150, 180, 200, 240, 256, 300, 500, 768)
LOG10_C_F64 = 307.050595577260822  # log10 of the FP64 initial scale 2^1020


@pytest.fixture(scope="module")
def emulator():
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    srcs = [NATIVE / "warp_emu.cpp", NATIVE / "warp_emu_shim.h", CSRC / "phmm_plan.cpp", CSRC / "phmm_tables.cpp",
            *CSRC.glob("*.cuh"), *CSRC.glob("*.h"), ROOT / "include" / "phmm_b200.h"]
    if not BIN.exists() or any(s.stat().st_mtime > BIN.stat().st_mtime for s in srcs):
        BIN.parent.mkdir(exist_ok=True)
        subprocess.run([gxx, "-std=c++20", "-O2", "-mfma", "-ffp-contract=off", "-pthread", "-w",
                        str(NATIVE / "warp_emu.cpp"), str(CSRC / "phmm_plan.cpp"), str(CSRC / "phmm_tables.cpp"),
                        "-o", str(BIN)], check=True)
    return BIN


def _write(pb: PackedBatch, path: Path) -> None:
    with open(path, "wb") as f:
        f.write(b"PHMMEMU1")
        f.write(np.array([pb.n_regions], np.uint32).tobytes())
        f.write(np.array([pb.n_haps.sum(), pb.n_reads.sum(), pb.hap_bases.size, pb.read_bases.size], np.uint64).tobytes())
        for a, t in ((pb.n_haps, np.uint32), (pb.n_reads, np.uint32), (pb.hap_off, np.uint64),
                     (pb.read_off, np.uint64)):
            f.write(np.ascontiguousarray(a, t).tobytes())
        for a in (pb.hap_bases, pb.read_bases, pb.read_qual, pb.read_ins, pb.read_del, pb.read_gcp):
            f.write(np.ascontiguousarray(a, np.uint8).tobytes())


def _run(binary, pb: PackedBatch, tmp_path: Path, mode: str = "engine", tiles: str = "default"):
    src, dst = tmp_path / "batch.bin", tmp_path / "out.bin"
    _write(pb, src)
    subprocess.run([str(binary), str(src), str(dst), mode, tiles], check=True, timeout=900)
    raw = dst.read_bytes()
    n = pb.out_size
    return (np.frombuffer(raw[:8 * n], np.float64), np.frombuffer(raw[8 * n:9 * n], np.uint8),
            int(np.frombuffer(raw[9 * n:], np.uint32)[0]))


def _batch(seed: int) -> PackedBatch:
    rng = np.random.default_rng(seed)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    regs = []
    for kind in ("equal", "per-row", "unequal", "N", "exotic"):
        haps = [bytearray(acgt[rng.integers(0, 4, int(rng.integers(8, 40)))]) for _ in range(int(rng.integers(2, 4)))]
        reads, q, ins, dels = [], [], [], []
        for L in LENS:
            r = bytearray(acgt[rng.integers(0, 4, L)])
            if kind == "N" and rng.random() < 0.5:
                r[L // 2] = ord("N")
            if kind == "exotic" and rng.random() < 0.5:
                r[L // 3] = ord("R")
            reads.append(bytes(r))
            q.append(rng.integers(2, 41, L).astype(np.uint8).tobytes())
            if kind == "per-row":
                ins.append(rng.integers(20, 46, L).astype(np.uint8).tobytes())
                dels.append(rng.integers(20, 46, L).astype(np.uint8).tobytes())
            else:
                ins.append(bytes([45] * L))
                dels.append(bytes([40 if kind == "unequal" else 45] * L))
        if kind == "N":
            haps[0][len(haps[0]) // 2] = ord("N")
        if kind == "exotic":
            haps[-1][1] = ord("R")
        regs.append(Region([bytes(h) for h in haps], reads, q, ins, dels, [bytes([10] * len(r)) for r in reads]))
    return PackedBatch.from_regions(regs)


@pytest.mark.parametrize("tiles", ["default", "multi4"])
def test_emulated_kernels_equal_the_oracle(emulator, oracle, tmp_path, tiles):
    pb = _batch(11)
    got, flags, status = _run(emulator, pb, tmp_path, tiles=tiles)
    want, used = oracle.batch(pb)
    assert status == 0
    assert_same_values(got, want, EXACT, tiles)
    assert np.array_equal(flags.astype(bool), used)
    assert used.any() and not used.all()  # both passes ran


def test_emulated_all_fp64_check_equals_the_oracle(emulator, oracle, tmp_path):
    pb = _batch(12)
    got, _, status = _run(emulator, pb, tmp_path, mode="check64")
    want, _ = oracle.batch(pb, fp64_only=True)
    assert status == 0
    assert_same_values(got, want, EXACT)


def test_emulated_fp64_recompute_of_mode0_equals_the_oracle(emulator, oracle, tmp_path):
    """Every pair of the constant-gap, insertion = deletion region through the FP64 recompute classes
    of mode 0 (the two-value lane state with the reference's flush-to-zero and the warp's vote), not
    only the pairs that underflow in FP32: each equals the reference's FP64 kernel on that pair."""
    pb = _batch(13)
    got, _, status = _run(emulator, pb, tmp_path, mode="eq64")
    assert status == 0
    n_h, n_r = int(pb.n_haps[0]), int(pb.n_reads[0])
    got0 = got[:n_h * n_r].reshape(n_h, n_r)
    want = np.empty((n_h, n_r))
    for h in range(n_h):
        hap = bytes(pb.hap_bases[pb.hap_off[h]:pb.hap_off[h + 1]])
        for r in range(n_r):
            s = slice(int(pb.read_off[r]), int(pb.read_off[r + 1]))
            raw = oracle.raw_f64(hap, bytes(pb.read_bases[s]), bytes(pb.read_qual[s]), bytes(pb.read_ins[s]),
                                 bytes(pb.read_del[s]), bytes(pb.read_gcp[s]))
            with np.errstate(divide="ignore"):
                want[h, r] = np.log10(raw) - LOG10_C_F64
    assert_same_values(got0, want, EXACT, "mode-0 FP64")
    # reads up to 500 bases end far below the FP32 range (-500 log10) but within FP64's; the 768-base
    # read underflows FP64 as well (-inf on both sides), through the flushes
    assert np.isfinite(want[:, :-1]).all() and (want[:, :-1] < -300).any() and np.isinf(want[:, -1]).all()


def test_emulated_fp64_recompute_of_per_row_modes_equals_the_oracle(emulator, oracle, tmp_path):
    """Every pair of the FP32 classes of modes 1 (per-row or unequal gap qualities) and 2 (intra)
    through the FP64 recompute classes of those modes (the two-value lane state with per-row gap
    parameters), not only the underflowed ones: each equals the reference's FP64 kernel of its
    variant on that pair."""
    pb = _batch(14)
    got, _, status = _run(emulator, pb, tmp_path, mode="row64")
    assert status == 0
    sizes = pb.n_haps.astype(np.int64) * pb.n_reads.astype(np.int64)
    offs = np.concatenate([[0], np.cumsum(sizes)])
    h0 = np.concatenate([[0], np.cumsum(pb.n_haps)])
    r0 = np.concatenate([[0], np.cumsum(pb.n_reads)])
    checked = 0
    for g in (1, 2, 3):  # per-row, unequal, N (its intra pairs)
        n_h, n_r = int(pb.n_haps[g]), int(pb.n_reads[g])
        blk = got[offs[g]:offs[g + 1]].reshape(n_h, n_r)
        for h in range(n_h):
            hh = int(h0[g]) + h
            hap = bytes(pb.hap_bases[pb.hap_off[hh]:pb.hap_off[hh + 1]])
            for r in range(n_r):
                rr = int(r0[g]) + r
                s = slice(int(pb.read_off[rr]), int(pb.read_off[rr + 1]))
                read = bytes(pb.read_bases[s])
                intra = b"N" in hap or b"N" in read
                if g == 3 and not intra:
                    continue  # constant equal gaps: mode 0, not run here
                raw = oracle.raw_f64(hap, read, bytes(pb.read_qual[s]), bytes(pb.read_ins[s]), bytes(pb.read_del[s]),
                                     bytes(pb.read_gcp[s]), kernel=1 if intra else 0)
                with np.errstate(divide="ignore"):
                    want = np.log10(raw) - LOG10_C_F64
                assert_same_values(np.array([blk[h, r]]), np.array([want]), EXACT, f"region {g} hap {h} read {r}")
                checked += 1
    assert checked > 60
