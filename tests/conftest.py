"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device (B200); the rest run on CPU."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(ROOT))

PACK_FIELDS = ("n_haps", "n_reads", "hap_bases", "hap_off", "read_bases", "read_qual", "read_ins", "read_del",
               "read_gcp", "read_off")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on a B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def ref():
    from oracle import Ref, build_ref

    if build_ref() is None:
        pytest.skip("reference build (oracle/_ref) not available here")
    return Ref()


@pytest.fixture(scope="session")
def genotype_ref():
    from oracle import GenotypeRef, build_ref_genotype

    if build_ref_genotype() is None:
        pytest.skip("reference genotyping build (oracle/_ref) not available here")
    return GenotypeRef()


@pytest.fixture(scope="session")
def golden_cases():
    return json.loads((GOLDEN / "golden_cases.json").read_text())["cases"]


@pytest.fixture(scope="session")
def sw_golden():
    return json.loads((GOLDEN / "sw_golden.json").read_text())["cases"]


@pytest.fixture(scope="session")
def sw_oracle():
    from oracle import SwOracle

    return SwOracle()


@pytest.fixture(scope="session")
def ref_regions():
    """{group: (PackedBatch, reference schedule_pairhmm log10 [hap][read] flat)} from the fixtures."""
    from rovaca_b200.pairhmm import PackedBatch

    z = np.load(GOLDEN / "ref_regions.npz")
    groups = sorted({k.split(".")[0] for k in z.files})
    return {g: (PackedBatch(*(z[f"{g}.{f}"] for f in PACK_FIELDS)), z[f"{g}.ref_log10"]) for g in groups}


@pytest.fixture(scope="session")
def engine():
    from rovaca_b200 import Engine

    eng = Engine(device=0)
    yield eng
    eng.close()


@pytest.fixture(scope="session")
def engine_direct():
    """Same engine without CUDA-graph replay (only non-empty kernel classes launched)."""
    from rovaca_b200 import Engine

    eng = Engine(device=0, use_cuda_graph=False)
    yield eng
    eng.close()


def assert_same_values(got, want, tol: float, what: str = "") -> None:
    """got and want agree pair for pair: NaN at the same pairs, the same infinities at the same
    pairs, and every finite pair within tol (absolute).  A plain nanmax of the difference would
    skip NaN-vs-value pairs and -inf - -inf pairs alike."""
    got = np.asarray(got, dtype=np.float64)
    want = np.asarray(want, dtype=np.float64)
    assert got.shape == want.shape, (what, got.shape, want.shape)
    nan_g, nan_w = np.isnan(got), np.isnan(want)
    assert np.array_equal(nan_g, nan_w), (what, "NaN masks differ", int(np.sum(nan_g != nan_w)))
    inf_g, inf_w = np.isinf(got), np.isinf(want)
    assert np.array_equal(inf_g, inf_w), (what, "infinity masks differ", int(np.sum(inf_g != inf_w)))
    assert np.array_equal(got[inf_g], want[inf_w]), (what, "infinities of different sign")
    fin = ~(nan_g | inf_g)
    if fin.any():
        err = float(np.max(np.abs(got[fin] - want[fin])))
        assert err <= tol, (what, err, tol)


def case_tuple(c):
    return (c["hap"].encode(), c["read"].encode(), bytes(c["q"]), bytes(c["i"]), bytes(c["d"]), bytes(c["c"]))


def f32_of_hex(h: str) -> float:
    return float(np.frombuffer(bytes.fromhex(h), ">f4")[0])


def f64_of_hex(h: str) -> float:
    return float(np.frombuffer(bytes.fromhex(h), ">f8")[0])
