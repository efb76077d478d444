"""phmm_compute_regions_noalloc, the entry point for callers that cannot allocate device memory
(their GPU memory belongs to another allocator, or allocation is forbidden on their threads).

It must give what phmm_compute_regions gives, on consecutive calls that share its fixed device
array, and it must not allocate device memory.  This file is collected last so that a run stopping
at the first failure has run every other test; it passes alone in a fresh process and after the
rest."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import assert_same_values
from rovaca_b200 import Engine, synth
from rovaca_b200._lib import PhmmError
from rovaca_b200.pairhmm import PackedBatch, compute_noalloc

pytestmark = pytest.mark.gpu

EXACT = 1e-12  # same kernels and arithmetic as the allocating entry point


def _mixed_batch(ref_regions):
    """Regions of every kernel path: the single-region benchmark shape, uneven regions, an
    underflow-stress region (FP64 recompute) and the edge regions (N, short, multi-stripe reads)."""
    regs = [synth.config0().region(0)] + [synth.config1(3, seed=61).region(g) for g in range(3)]
    regs.append(synth.config2(1, seed=62).region(0))
    edge, _ = ref_regions["edge"]
    regs += [edge.region(g) for g in range(edge.n_regions)]
    return PackedBatch.from_regions(regs)


def test_noalloc_matches_allocating_entry_point_on_consecutive_calls(ref_regions, oracle):
    batch = _mixed_batch(ref_regions)
    with Engine(device=0) as eng:
        want, want_flags, _ = eng.compute(batch, want_flags=True)
    assert want_flags.any()  # the FP64 recompute path runs
    for call in range(2):
        got, flags = compute_noalloc(batch, device=0, want_flags=True)
        assert_same_values(got, want, EXACT, f"call {call}")
        assert np.array_equal(flags, want_flags), call
    # and directly against the oracle, pair for pair, with its FP32 -> FP64 decisions
    ref, used = oracle.batch(batch)
    assert_same_values(got, ref, EXACT, "oracle")
    assert np.array_equal(flags.astype(bool), used)


def test_noalloc_second_batch_does_not_see_the_first():
    a = synth.config1(2, seed=71)
    b = synth.config0()
    got_a, _ = compute_noalloc(a)
    got_b, _ = compute_noalloc(b)
    with Engine(device=0) as eng:
        want_a, _, _ = eng.compute(a)
        want_b, _, _ = eng.compute(b)
    assert_same_values(got_a, want_a, EXACT, "first batch")
    assert_same_values(got_b, want_b, EXACT, "second batch")
    assert np.isfinite(got_b).all()  # every pair of the smaller second batch was computed
    assert got_a.size != got_b.size


def test_noalloc_allocates_no_device_memory():
    """Free device memory is the same before and after a call (after one warm-up call of the same
    batch, which loads the kernels it launches and sets the device up)."""
    import torch

    batch = synth.config1(20, seed=91)
    compute_noalloc(batch)
    torch.cuda.synchronize(0)
    free_before, _ = torch.cuda.mem_get_info(0)
    got, _ = compute_noalloc(batch)
    torch.cuda.synchronize(0)
    free_after, _ = torch.cuda.mem_get_info(0)
    assert free_after == free_before, (free_before, free_after)
    assert np.isfinite(got).all()


def test_noalloc_rejects_batches_beyond_its_array():
    big = synth.config1(400, seed=81)
    with pytest.raises(PhmmError) as e:
        compute_noalloc(big)
    assert e.value.name == "PHMM_ERR_LIMIT_EXCEEDED"
    assert "scratch" in str(e.value)
