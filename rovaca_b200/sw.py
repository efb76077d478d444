"""Smith-Waterman realignment of reads to haplotypes on the GPU (phmm_sw_align in include/phmm_b200.h).

The reference aligns one read at a time through a ``lib_sw_avx`` context (seq1 = haplotype, seq2 =
read, ``sw->avx_function(sw)``; genotype/utils/alignment_utils.cpp:571-579) and reads back score,
alignment offset and CIGAR.  Here a batch of (haplotype, read) pairs goes to the device in one call and
every pair's fields come back, equal to the reference's.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _lib

GENOTYPING = (10, -15, -30, -5)   # sw_parameters_genotype, lib/sw_avx/sw_avx.c:15
ASSEMBLY = (200, -150, -260, -11)  # sw_parameters_assemble, lib/sw_avx/sw_avx.c:14
MAX_CIGAR = 2047                   # the reference emits at most cigar_max_len - 1 ops (sw_cigar.c:164)
CIGAR_OPS = "MIDNSHP=XB"
# read columns per lane of the kernel classes (phmm_sw.h kSwK); the last class is the 16-bit
# wrap-around class for parameters whose int16 adds can wrap
CLASS_K = (1, 2, 3, 4, 5, 6, 7, 8, 10, 12, 16, 20, 24, 24)

SW_ITEM_DTYPE = np.dtype([("hap_offset", "<u8"), ("read_offset", "<u8"), ("hap_len", "<u4"), ("read_len", "<u4")])
SW_RESULT_DTYPE = np.dtype([("score", "<i4"), ("alignment_offset", "<i4"), ("max_i", "<i4"), ("max_j", "<i4"),
                            ("cigar_count", "<u4"), ("cigar_offset", "<u4")])


def cigar_string(ops) -> str:
    return "".join(f"{int(c) >> 4}{CIGAR_OPS[int(c) & 15]}" for c in ops)


def _bytes(x) -> bytes:
    if isinstance(x, str):
        return x.encode()
    return bytes(x)


@dataclass
class SwBatch:
    """Packed alignments: haplotype and read bases concatenated, one item per pair."""

    hap_bases: np.ndarray   # uint8
    read_bases: np.ndarray  # uint8
    items: np.ndarray       # SW_ITEM_DTYPE

    @property
    def n(self) -> int:
        return int(self.items.shape[0])

    @property
    def cells(self) -> int:
        return int((self.items["hap_len"].astype(np.uint64) * self.items["read_len"].astype(np.uint64)).sum())

    @classmethod
    def from_pairs(cls, pairs: Sequence[tuple[bytes, bytes]]) -> "SwBatch":
        """One item per (haplotype, read) pair; equal haplotypes given as the same object are stored once."""
        haps, hap_at = [], {}
        reads = []
        items = np.zeros(len(pairs), SW_ITEM_DTYPE)
        hoff = roff = 0
        for q, (h, r) in enumerate(pairs):
            key = id(h)
            if key not in hap_at:
                hb = _bytes(h)
                hap_at[key] = (hoff, len(hb))
                haps.append(hb)
                hoff += len(hb)
            items[q]["hap_offset"], items[q]["hap_len"] = hap_at[key]
            rb = _bytes(r)
            items[q]["read_offset"], items[q]["read_len"] = roff, len(rb)
            reads.append(rb)
            roff += len(rb)
        return cls(np.frombuffer(b"".join(haps), np.uint8).copy(), np.frombuffer(b"".join(reads), np.uint8).copy(),
                   items)

    def pair(self, q: int) -> tuple[bytes, bytes]:
        it = self.items[q]
        h = self.hap_bases[int(it["hap_offset"]):int(it["hap_offset"]) + int(it["hap_len"])].tobytes()
        r = self.read_bases[int(it["read_offset"]):int(it["read_offset"]) + int(it["read_len"])].tobytes()
        return h, r


def _params(params) -> C.Array:
    p = tuple(int(x) for x in (params if params is not None else GENOTYPING))
    if len(p) != 4:
        raise ValueError("params = (match, mismatch, gap_open, gap_extend)")
    return (C.c_int32 * 4)(*p)


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data) if a.size else None


def _check_variant(variant: int) -> None:
    if variant not in (0, 1, 2):
        raise ValueError("variant must be 0 (the reference's choice), 1 (int32) or 2 (int16)")


@dataclass
class SwResults:
    """Per alignment: score, alignment_offset, max_i, max_j, cigar_count, cigar_offset
    (SW_RESULT_DTYPE) and the compact CIGAR ops (BAM encoding, read order): alignment q's first
    min(cigar_count, cigar_cap) ops at cigars[cigar_offset:]."""

    fields: np.ndarray
    cigars: np.ndarray
    cigar_cap: int

    def __len__(self) -> int:
        return int(self.fields.shape[0])

    def ops(self, q: int) -> list[int]:
        f = self.fields[q]
        o, n = int(f["cigar_offset"]), min(int(f["cigar_count"]), self.cigar_cap)
        return [int(x) for x in self.cigars[o:o + n]]

    def cigar(self, q: int) -> str:
        return cigar_string(self.ops(q))

    def tuple(self, q: int):
        """(score, alignment_offset, max_i, max_j, ops): the oracle's result layout."""
        f = self.fields[q]
        return int(f["score"]), int(f["alignment_offset"]), int(f["max_i"]), int(f["max_j"]), self.ops(q)


def _capacity(batch: SwBatch, cigar_cap: int) -> int:
    """Ops the compact CIGAR buffer needs at most: min(cap, haplotype + read length) per alignment."""
    ln = batch.items["hap_len"].astype(np.int64) + batch.items["read_len"].astype(np.int64)
    return int(np.minimum(ln, min(cigar_cap, MAX_CIGAR)).sum())


def align(engine, batch: SwBatch, params=GENOTYPING, variant: int = 0, cigar_cap: int = MAX_CIGAR,
          ops_per_alignment: int = 32) -> SwResults:
    """Aligns every pair of the batch on the engine's device (host buffers in and out).  The CIGAR
    buffer starts at ops_per_alignment ops per pair (or the most the batch can need, if smaller);
    a batch that needs more is aligned again with the size the first call reported."""
    _check_variant(variant)
    lib = _lib.load()
    n = batch.n
    fields = np.zeros(n, SW_RESULT_DTYPE)
    size = min(_capacity(batch, cigar_cap), n * ops_per_alignment)
    total = C.c_uint64()
    for _ in range(2):
        cigars = np.empty(max(size, 1), np.uint32)
        if not n:
            break
        st = lib.phmm_sw_align(engine._h, _params(params), variant, n, _ptr(batch.items), _ptr(batch.hap_bases),
                               batch.hap_bases.size, _ptr(batch.read_bases), batch.read_bases.size, cigar_cap,
                               _ptr(fields), _ptr(cigars), cigars.size, C.byref(total))
        if st == _lib.PHMM_ERR_LIMIT_EXCEEDED and total.value > size:
            size = total.value
            continue
        _lib.check(st)
        break
    return SwResults(fields, cigars[:total.value], cigar_cap)


class SwResident:
    """A batch kept on the device: run it many times (device time per run), read results on demand."""

    def __init__(self, engine, batch: SwBatch, params=GENOTYPING, variant: int = 0, cigar_cap: int = MAX_CIGAR):
        _check_variant(variant)
        self._lib = _lib.load()
        self.engine = engine
        self.n = batch.n
        self.cells = batch.cells
        self.cigar_cap = cigar_cap
        h = C.c_void_p()
        _lib.check(self._lib.phmm_sw_resident_create(engine._h, _params(params), variant, self.n, _ptr(batch.items),
                                                     _ptr(batch.hap_bases), batch.hap_bases.size,
                                                     _ptr(batch.read_bases), batch.read_bases.size, cigar_cap,
                                                     C.byref(h)))
        self._h = h

    def run(self, iterations: int = 1) -> float:
        """Runs the batch `iterations` times back to back; returns device ms per run."""
        ms = C.c_float()
        _lib.check(self._lib.phmm_sw_resident_run(self._h, iterations, C.byref(ms), None))
        return float(ms.value)

    def profile(self) -> np.ndarray:
        """Device ms of each kernel class in one run (CLASS_K: read columns per lane of the 14 classes;
        the last is the 16-bit wrap-around class)."""
        cls = (C.c_float * len(CLASS_K))()
        _lib.check(self._lib.phmm_sw_resident_run(self._h, 0, None, C.cast(cls, C.c_void_p)))
        return np.array(cls[:], np.float32)

    def results(self) -> SwResults:
        fields = np.zeros(self.n, SW_RESULT_DTYPE)
        total = C.c_uint64()
        _lib.check(self._lib.phmm_sw_resident_results(self._h, _ptr(fields), None, 0, C.byref(total)))
        cigars = np.empty(max(total.value, 1), np.uint32)
        _lib.check(self._lib.phmm_sw_resident_results(self._h, _ptr(fields), _ptr(cigars), cigars.size,
                                                      C.byref(total)))
        return SwResults(fields, cigars[:total.value], self.cigar_cap)

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.phmm_sw_resident_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
