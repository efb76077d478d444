"""The Rovaca-side binding (integration/pairhmm_engine_b200.cpp), compiled against the reference's own
headers by integration/build_check.sh with the driver tests/native/integration_check.cpp (fake
libhts-backed records).  CPU: the failure paths return what call_roDV_pairhmm_scheduled returns
(pairhmm_internal.cpp:576-623) -- an all-NaN [hap][read] matrix with every read kept -- for a pool
that is not a RovacaMemoryPool and for a missing engine.  GPU: the bound rovaca::call_pairhmm and the
pipelined form (region k+1 submitted before region k is collected) give the library's region-API
results bit for bit, erasing the same reads."""
from __future__ import annotations

import math
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
BIN = ROOT / "integration" / "_build" / "integration_check"


def _binary():
    from oracle.oracle import reference_root

    src = [ROOT / "integration" / "pairhmm_engine_b200.cpp", ROOT / "integration" / "pairhmm_engine_b200.h",
           ROOT / "tests" / "native" / "integration_check.cpp", ROOT / "integration" / "build_check.sh"]
    fresh = BIN.exists() and all(BIN.stat().st_mtime >= s.stat().st_mtime for s in src)
    if not fresh and Path(reference_root(), "src/haplotypecaller/pairhmm").is_dir():
        subprocess.run(["bash", str(ROOT / "integration" / "build_check.sh"), reference_root()], check=True,
                       capture_output=True)
        fresh = True
    if not fresh:
        pytest.skip("integration driver not built (needs the reference's headers)")
    return BIN


def _regions(n: int, seed: int):
    from rovaca_b200 import synth

    return synth.genotyping_regions(n, seed=seed, depth=24)


def _input(regions) -> str:
    lines = []
    for k, r in enumerate(regions):
        if k:
            lines.append("E")
        lines += [f"H {h.decode()}" for h in r["haplotypes"]]
        for rd, q, mq in zip(r["reads"], r["quals"], r["mapq"]):
            lines.append(f"R {rd.decode()} {int(mq)} {','.join(str(x) for x in q)}")
    return "\n".join(lines) + "\n"


def _run(mode: str, regions, thr: int, pcr: int):
    p = subprocess.run([str(_binary()), mode, str(thr), str(pcr)], input=_input(regions), capture_output=True,
                       text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    out, cur = [], None
    for line in p.stdout.splitlines():
        f = line.split()
        if f[0] == "region":
            cur = {"reads": int(f[3]), "kept": [int(x) for x in f[5:]], "rows": []}
            out.append(cur)
        elif f[0] == "row":
            cur["rows"].append([float(x) for x in f[2:]])
    return out, p.stdout + p.stderr  # the reference's logger (spdlog) writes to stdout


@pytest.mark.parametrize("mode", ["foreign-pool", "no-engine"])
def test_failure_paths_return_nan_and_keep_every_read(mode):
    regions = _regions(3, seed=5)
    res, err = _run(mode, regions, 18, 3)
    assert len(res) == 3
    for r, g in zip(regions, res):
        assert g["reads"] == len(r["reads"]) and g["kept"] == list(range(len(r["reads"])))
        assert len(g["rows"]) == len(r["haplotypes"])
        assert all(math.isnan(v) for row in g["rows"] for v in row)
    assert ("pool is not RovacaMemoryPool" if mode == "foreign-pool" else "engine not initialised") in err


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["sync", "pipeline"])
def test_bound_call_pairhmm_equals_the_region_api(mode):
    from rovaca_b200 import Engine, call_pairhmm

    regions = _regions(6, seed=9)
    res, _ = _run(mode, regions, 18, 3)
    with Engine(device=0, autotune=False) as eng:
        for r, g in zip(regions, res):
            mat, kept = call_pairhmm(r["haplotypes"], r["reads"], r["quals"], r["mapq"], 18, "CONSERVATIVE",
                                     engine=eng)
            assert g["kept"] == [int(k) for k in kept]
            assert g["reads"] == len(kept)
            got = np.array(g["rows"])
            assert got.shape == mat.shape
            assert np.array_equal(got, mat, equal_nan=True)
