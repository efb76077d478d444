"""Python host interface of the B200 PairHMM engine, mirroring the reference's PairHMM entry points.

Reference interfaces mirrored (paths inside the reference project):
  * ``schedule_pairhmm`` -- the vector API the reference's tests and perf harness drive:
    ``bool schedule_pairhmm(haplotypes, reads, result, quality, insertion_qualities,
    deletion_qualities, gap_contiguous_qualities, ...)``, result ``[read][hap]`` log10
    (src/haplotypecaller/pairhmm/roDV_schedule.h:16-27, roDV_schedule.cpp:154-361).
  * ``call_pairhmm`` -- the HaplotypeCaller entry point ``DoubleVector2D call_pairhmm(hs, rs,
    min_quality_threshold, pcr_option, pool)``, result ``[hap][read]`` with poorly modelled reads
    removed from ``rs`` (src/haplotypecaller/pairhmm/pairhmm_engine.h:14,
    pairhmm_internal.cpp:576-623).
  * ``Engine.compute`` -- batched form: many regions in one persistent launch.
  * ``Engine.submit/poll/wait/cancel`` -- the serving loop (continuous batching).

All computation happens in libphmm_b200.so on the GPU; nothing here computes likelihoods.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Iterable, Sequence

import numpy as np

from . import _lib
from ._lib import PCR_MODELS, PhmmError, check

Seq = "bytes | np.ndarray | Sequence[int]"


def _u8(x) -> np.ndarray:
    if isinstance(x, (bytes, bytearray, memoryview)):
        return np.frombuffer(bytes(x), dtype=np.uint8)
    if isinstance(x, str):
        return np.frombuffer(x.encode(), dtype=np.uint8)
    return np.ascontiguousarray(np.asarray(x, dtype=np.uint8))


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


@dataclass
class Region:
    """One active region: candidate haplotypes and reads with their per-base qualities."""

    haplotypes: list
    reads: list
    quality: list
    insertion_qualities: list
    deletion_qualities: list
    gap_contiguous_qualities: list

    @property
    def n_haps(self) -> int:
        return len(self.haplotypes)

    @property
    def n_reads(self) -> int:
        return len(self.reads)


@dataclass
class PackedBatch:
    """Regions in the flat, concatenated layout of ``phmm_batch`` (include/phmm_b200.h)."""

    n_haps: np.ndarray      # u32 [n_regions]
    n_reads: np.ndarray     # u32 [n_regions]
    hap_bases: np.ndarray   # u8
    hap_off: np.ndarray     # u64 [sum(n_haps)+1]
    read_bases: np.ndarray  # u8
    read_qual: np.ndarray
    read_ins: np.ndarray
    read_del: np.ndarray
    read_gcp: np.ndarray
    read_off: np.ndarray    # u64 [sum(n_reads)+1]
    _keep: list = field(default_factory=list, repr=False)

    @property
    def n_regions(self) -> int:
        return int(self.n_haps.shape[0])

    @property
    def out_size(self) -> int:
        return int(np.sum(self.n_haps.astype(np.uint64) * self.n_reads.astype(np.uint64)))

    def out_offsets(self) -> np.ndarray:
        """Start of each region's [hap][read] block in the flat output (n_regions+1 entries)."""
        sizes = self.n_haps.astype(np.uint64) * self.n_reads.astype(np.uint64)
        return np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)

    def cells(self) -> int:
        """Sum over all pairs of read length x haplotype length."""
        hl = np.diff(self.hap_off).astype(np.int64)
        rl = np.diff(self.read_off).astype(np.int64)
        total, h0, r0 = 0, 0, 0
        for m, n in zip(self.n_haps.tolist(), self.n_reads.tolist()):
            total += int(hl[h0:h0 + m].sum()) * int(rl[r0:r0 + n].sum())
            h0 += m
            r0 += n
        return total

    def region(self, g: int) -> Region:
        """Region g back as sequences (for checks)."""
        h0 = int(self.n_haps[:g].sum())
        r0 = int(self.n_reads[:g].sum())
        m, n = int(self.n_haps[g]), int(self.n_reads[g])
        hs = [bytes(self.hap_bases[self.hap_off[h]:self.hap_off[h + 1]]) for h in range(h0, h0 + m)]
        sl = [(int(self.read_off[r]), int(self.read_off[r + 1])) for r in range(r0, r0 + n)]
        return Region(hs, [bytes(self.read_bases[a:b]) for a, b in sl], [bytes(self.read_qual[a:b]) for a, b in sl],
                      [bytes(self.read_ins[a:b]) for a, b in sl], [bytes(self.read_del[a:b]) for a, b in sl],
                      [bytes(self.read_gcp[a:b]) for a, b in sl])

    @classmethod
    def from_regions(cls, regions: Iterable[Region]) -> "PackedBatch":
        regions = list(regions)
        haps = [_u8(h) for r in regions for h in r.haplotypes]
        reads = [_u8(x) for r in regions for x in r.reads]
        cat = lambda parts: np.concatenate(parts) if parts else np.zeros(0, np.uint8)
        qual = [_u8(x) for r in regions for x in r.quality]
        ins = [_u8(x) for r in regions for x in r.insertion_qualities]
        dele = [_u8(x) for r in regions for x in r.deletion_qualities]
        gcp = [_u8(x) for r in regions for x in r.gap_contiguous_qualities]
        for arr in (qual, ins, dele, gcp):
            if [len(a) for a in arr] != [len(a) for a in reads]:
                raise ValueError("every quality array must have its read's length")
        off = lambda parts: np.concatenate([[0], np.cumsum([len(p) for p in parts])]).astype(np.uint64)
        return cls(np.array([r.n_haps for r in regions], np.uint32), np.array([r.n_reads for r in regions], np.uint32),
                   cat(haps), off(haps), cat(reads), cat(qual), cat(ins), cat(dele), cat(gcp), off(reads))

    def pinned(self) -> "PackedBatch":
        """A copy whose arrays live in page-locked host memory (fast DMA); uses torch for the pinning."""
        import torch

        def pin(a: np.ndarray) -> np.ndarray:
            t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
            v = t.numpy().view(a.dtype)[: a.size]
            v[...] = a
            keep.append(t)
            return v

        keep: list = []
        pb = PackedBatch(*(pin(getattr(self, f)) for f in ("n_haps", "n_reads", "hap_bases", "hap_off", "read_bases",
                                                           "read_qual", "read_ins", "read_del", "read_gcp", "read_off")))
        pb._keep = keep
        return pb

    def subset(self, regions: Sequence[int]) -> "PackedBatch":
        return PackedBatch.from_regions([self.region(g) for g in regions])

    def as_c(self) -> _lib.Batch:
        b = _lib.Batch()
        b.n_regions = self.n_regions
        b.n_haps = _ptr(self.n_haps)
        b.n_reads = _ptr(self.n_reads)
        b.hap_bases = _ptr(self.hap_bases)
        b.hap_off = _ptr(self.hap_off)
        b.read_bases = _ptr(self.read_bases)
        b.read_qual = _ptr(self.read_qual)
        b.read_ins = _ptr(self.read_ins)
        b.read_del = _ptr(self.read_del)
        b.read_gcp = _ptr(self.read_gcp)
        b.read_off = _ptr(self.read_off)
        return b


def compute_noalloc(batch: PackedBatch, device: int = 0, want_flags: bool = False):
    """phmm_compute_regions_noalloc: the batch computation without any device allocation (for
    callers that cannot call cudaMalloc); all device data lives in the library's fixed 64 MiB array.
    Returns (likelihoods, flags or None) in the layout of Engine.compute."""
    lib = _lib.load()
    out = np.empty(batch.out_size, np.float64)
    fl = np.empty(batch.out_size, np.uint8) if want_flags else None
    b = batch.as_c()
    check(lib.phmm_compute_regions_noalloc(C.byref(b), _ptr(out), _ptr(fl), device))
    return out, fl


def plan_summary(batch: PackedBatch, tiles: "_lib.TileTable | None" = None) -> dict:
    """How the engine cuts a batch into work (host only): items per FP32 class and pairs per FP64
    class, under a tile table (default shapes when None)."""
    lib = _lib.load()
    items = np.zeros(_lib.FP32_CLASSES, np.uint32)
    pairs = np.zeros(_lib.FP64_CLASSES, np.uint64)
    tp, tc = C.c_uint64(), C.c_uint64()
    b = batch.as_c()
    check(lib.phmm_host_plan_summary(C.byref(b), C.byref(tiles) if tiles is not None else None, _ptr(items),
                                     _ptr(pairs), C.byref(tp), C.byref(tc)))
    return {"class_items": items, "class_pairs": pairs, "pairs": tp.value, "cells": tc.value}


def default_tiles() -> "_lib.TileTable":
    """phmm_tile_table_default: smallest single stripe up to 256 rows, 256-row stripes beyond."""
    t = _lib.TileTable()
    _lib.load().phmm_tile_table_default(C.byref(t))
    return t


def class32(mode: int, kh: int, multi: bool = False) -> int:
    """FP32 kernel class of a mode (0 inter with constant gaps and insertion = deletion quality, 1 other
    inter, 2 intra) and shape."""
    return mode * 13 + (4 + kh if multi else kh - 1)


def class64(mode: int, read_len: int) -> int:
    """FP64 recompute class of a pair from its mode (that of the FP32 class that ran it: 0 inter
    constant gaps, 1 inter per-row, 2 intra) and its read length."""
    return mode * 9 + (8 if read_len > 256 else (read_len + 31) // 32 - 1)


class Engine:
    """One engine per CUDA device (phmm_engine_create)."""

    def __init__(self, device: int = 0, use_cuda_graph: bool = True, autotune: bool = True,
                 hbm_budget_bytes: int = 0, chunk_cells: int = 0):
        """chunk_cells: compute() runs batches of at least this many cells as a pipeline of region
        chunks (0: the library default, 2**64 - 1: never)."""
        self._lib = _lib.load()
        cfg = _lib.Config(device, int(use_cuda_graph), int(autotune), 0, hbm_budget_bytes, chunk_cells)
        h = C.c_void_p()
        check(self._lib.phmm_engine_create(C.byref(cfg), C.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            check(self._lib.phmm_engine_destroy(self._h))
            self._h = None

    def __enter__(self) -> "Engine":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def version() -> str:
        return _lib.load().phmm_version().decode()

    def sw_align(self, batch, params=None, variant: int = 0, cigar_cap: int | None = None, **kw):
        """Smith-Waterman realignment of a batch of (haplotype, read) pairs (rovaca_b200.sw)."""
        from . import sw

        return sw.align(self, batch, sw.GENOTYPING if params is None else params, variant,
                        sw.MAX_CIGAR if cigar_cap is None else cigar_cap, **kw)

    def sw_resident(self, batch, params=None, variant: int = 0, cigar_cap: int | None = None):
        from . import sw

        return sw.SwResident(self, batch, sw.GENOTYPING if params is None else params, variant,
                             sw.MAX_CIGAR if cigar_cap is None else cigar_cap)

    # ---- batched -----------------------------------------------------------------------
    def compute(self, batch: PackedBatch, want_flags: bool = False, out: np.ndarray | None = None,
                flags: np.ndarray | None = None):
        """Every pair of every region; returns (likelihoods, flags or None, stats dict).

        likelihoods is flat: region blocks in order, [hap][read] inside (see PackedBatch.out_offsets)."""
        n = batch.out_size
        if out is None:
            out = np.empty(n, np.float64)
        if want_flags and flags is None:
            flags = np.empty(n, np.uint8)
        st = _lib.Stats()
        b = batch.as_c()
        check(self._lib.phmm_compute_regions(self._h, C.byref(b), _ptr(out), _ptr(flags) if want_flags else None,
                                             C.byref(st)))
        return out, (flags if want_flags else None), st.as_dict()

    def compute_regions(self, regions: Sequence[Region], want_flags: bool = False):
        """List of [n_haps][n_reads] arrays, one per region."""
        pb = PackedBatch.from_regions(regions)
        out, fl, _ = self.compute(pb, want_flags)
        offs = pb.out_offsets()
        res = []
        for g in range(pb.n_regions):
            blk = out[offs[g]:offs[g + 1]].reshape(int(pb.n_haps[g]), int(pb.n_reads[g]))
            res.append(blk if fl is None else (blk, fl[offs[g]:offs[g + 1]].reshape(blk.shape)))
        return res

    # ---- device-resident batches -------------------------------------------------------
    def resident(self, batch: PackedBatch, want_flags: bool = False) -> "ResidentBatch":
        return ResidentBatch(self, batch, want_flags)

    def fp32_fma_peak(self) -> tuple[float, float]:
        """Measured FP32 FMA throughput of the device, TFLOP/s (an FMA counts 2 FLOPs): with scalar
        FFMA and with packed FFMA2 instructions."""
        a, b = C.c_double(), C.c_double()
        check(self._lib.phmm_fp32_fma_peak(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    # ---- serving loop ------------------------------------------------------------------
    def submit(self, region: PackedBatch, out: np.ndarray, flags: np.ndarray | None = None) -> int:
        """Queues one region (region.n_regions == 1); out (and flags) must stay alive until wait()."""
        t = C.c_uint64()
        b = region.as_c()
        check(self._lib.phmm_submit(self._h, C.byref(b), _ptr(out), _ptr(flags), C.byref(t)))
        return t.value

    def poll(self, ticket: int) -> bool:
        d = C.c_int32()
        check(self._lib.phmm_poll(self._h, ticket, C.byref(d)))
        return bool(d.value)

    def wait(self, ticket: int, timeout_us: int = -1):
        """Blocks until done; returns (queued_us, total_us) and releases the ticket."""
        q, t = C.c_double(), C.c_double()
        check(self._lib.phmm_wait(self._h, ticket, timeout_us, C.byref(q), C.byref(t)))
        return q.value, t.value

    def cancel(self, ticket: int) -> None:
        check(self._lib.phmm_cancel(self._h, ticket))

    def tiles(self) -> "_lib.TileTable":
        t = _lib.TileTable()
        check(self._lib.phmm_engine_get_tiles(self._h, C.byref(t)))
        return t

    def set_tiles(self, table: "_lib.TileTable") -> None:
        check(self._lib.phmm_engine_set_tiles(self._h, C.byref(table)))

    def autotune(self) -> dict:
        """Runs the tile-shape autotuner now; returns its measurements (the table is installed)."""
        rep = _lib.TuneReport()
        check(self._lib.phmm_engine_autotune(self._h, C.byref(rep)))
        entries = [{"mode": e.mode, "bucket": e.bucket, "rows_per_lane": e.rows_per_lane,
                    "multi_stripe": bool(e.multi_stripe), "chosen": bool(e.chosen), "gcups": round(e.gcups, 1)}
                   for e in rep.entries[:rep.n_entries]]
        return {"seconds": rep.seconds, "entries": entries}

    def server_stats(self) -> dict:
        """Counters of the serving loop (phmm_server_stats_get)."""
        st = _lib.ServerStats()
        check(self._lib.phmm_server_stats_get(self._h, C.byref(st)))
        return st.as_dict()

    # ---- region API ----------------------------------------------------------------------
    def submit_region(self, haplotypes, reads, base_quals, mapq, min_quality_threshold: int = 18,
                      pcr_option: str | int = "CONSERVATIVE", events=None, want_matrix: bool = True,
                      want_allele_lk: bool = False, realign=None) -> "RegionTicket":
        """phmm_submit_region: queues one region with call_pairhmm semantics (read preparation and
        post-processing on the GPU).  events: optional list of (n_alleles, allele of each haplotype,
        -1 for none) to genotype on the GPU.  realign: optional dict with "priority" (one per
        haplotype) and optional "clip_left" / "clip_right" (one per read) to realign the kept reads
        to their best haplotypes on the GPU (phmm_submit_region_realign).  RegionTicket.wait() returns
        (matrix or None, keep mask), RegionTicket.genotypes() the per-event results and
        RegionTicket.realignment() the best haplotypes and alignments."""
        return RegionTicket(self, haplotypes, reads, base_quals, mapq, min_quality_threshold, pcr_option, events,
                            want_matrix, want_allele_lk, realign)

    def call_region(self, haplotypes, reads, base_quals, mapq, min_quality_threshold: int = 18,
                    pcr_option: str | int = "CONSERVATIVE"):
        """call_pairhmm semantics; returns (matrix [n_haps][n_reads] with kept reads first, keep mask)."""
        pcr = PCR_MODELS[pcr_option] if isinstance(pcr_option, str) else int(pcr_option)
        hs = [_u8(h) for h in haplotypes]
        rs = [_u8(r) for r in reads]
        qs = [_u8(q) for q in base_quals]
        cat = lambda parts: np.concatenate(parts) if parts else np.zeros(1, np.uint8)
        off = lambda parts: np.concatenate([[0], np.cumsum([len(p) for p in parts])]).astype(np.uint64)
        hb, hoff, rb, roff, qb = cat(hs), off(hs), cat(rs), off(rs), cat(qs)
        mq = np.ascontiguousarray(np.asarray(mapq, np.uint8).reshape(-1))
        if mq.size == 1 and len(rs) > 1:
            mq = np.full(len(rs), mq[0], np.uint8)
        out = np.empty(len(hs) * len(rs), np.float64)
        keep = np.empty(len(rs), np.uint8)
        nk = C.c_uint32()
        st = self._lib.phmm_call_region(self._h, len(hs), _ptr(hb), _ptr(hoff), len(rs), _ptr(rb), _ptr(qb), _ptr(roff),
                                        _ptr(mq), int(min_quality_threshold), pcr, _ptr(out), _ptr(keep), C.byref(nk))
        check(st)
        return out.reshape(len(hs), len(rs)), keep.astype(bool)


class RegionTicket:
    """A region submitted with phmm_submit_region; keeps its buffers alive until wait()."""

    def __init__(self, engine: Engine, haplotypes, reads, base_quals, mapq, min_quality_threshold, pcr_option,
                 events=None, want_matrix: bool = True, want_allele_lk: bool = False, realign=None):
        pcr = PCR_MODELS[pcr_option] if isinstance(pcr_option, str) else int(pcr_option)
        hs = [_u8(h) for h in haplotypes]
        rs = [_u8(r) for r in reads]
        qs = [_u8(q) for q in base_quals]
        cat = lambda parts: np.concatenate(parts) if parts else np.zeros(1, np.uint8)
        off = lambda parts: np.concatenate([[0], np.cumsum([len(p) for p in parts])]).astype(np.uint64)
        self._keepalive = [cat(hs), off(hs), cat(rs), off(rs), cat(qs)]
        hb, hoff, rb, roff, qb = self._keepalive
        mq = np.ascontiguousarray(np.asarray(mapq, np.uint8).reshape(-1))
        if mq.size == 1 and len(rs) > 1:
            mq = np.full(len(rs), mq[0], np.uint8)
        self._keepalive.append(mq)
        self.n_haps, self.n_reads = len(hs), len(rs)
        self.out = np.empty(self.n_haps * self.n_reads, np.float64) if want_matrix else None
        self.keep = np.empty(max(self.n_reads, 1), np.uint8)
        self.n_kept = C.c_uint32()
        inp = _lib.RegionInput(self.n_haps, hb.ctypes.data, hoff.ctypes.data, self.n_reads, rb.ctypes.data,
                               qb.ctypes.data, roff.ctypes.data, mq.ctypes.data, int(min_quality_threshold), pcr)
        self.events = None
        ev_ptr = None
        if events:
            na = np.array([int(a) for a, _ in events], np.uint8)
            ha = np.ascontiguousarray(np.array([np.asarray(m, np.int8).reshape(-1) for _, m in events], np.int8))
            n_gl = int(sum(int(a) * (int(a) + 1) // 2 for a in na))
            self.gl = np.empty(max(n_gl, 1), np.float64)
            self.best = np.empty(len(na), np.int32)
            self.allele_lk = np.empty(max(int(na.astype(np.int64).sum()) * self.n_reads, 1)) if want_allele_lk else None
            self._keepalive += [na, ha]
            self.events = _lib.RegionEvents(len(na), na.ctypes.data, ha.ctypes.data, self.gl.ctypes.data,
                                            self.best.ctypes.data,
                                            self.allele_lk.ctypes.data if want_allele_lk else None)
            self._n_alleles = na
            ev_ptr = C.byref(self.events)
        self._engine = engine
        t = C.c_uint64()
        self.realign = None
        if realign is not None:
            from . import sw

            prio = np.ascontiguousarray(np.asarray(realign["priority"], np.float64).reshape(-1))
            zeros = np.zeros(self.n_reads, np.uint16)
            cl = np.ascontiguousarray(np.asarray(realign.get("clip_left", zeros), np.uint16).reshape(-1))
            cr = np.ascontiguousarray(np.asarray(realign.get("clip_right", zeros), np.uint16).reshape(-1))
            if prio.size != self.n_haps or cl.size != self.n_reads or cr.size != self.n_reads:
                raise ValueError("realign: one priority per haplotype and one clip per read")
            lens = np.array([len(r) for r in rs], np.int64)
            cap = int(np.minimum(lens - cl - cr + max((len(h) for h in hs), default=0), sw.MAX_CIGAR).sum())
            cap = int(realign.get("cigar_capacity", cap))
            self.best_hap = np.empty(max(self.n_reads, 1), np.int32)
            self.sw_res = np.zeros(max(self.n_reads, 1), sw.SW_RESULT_DTYPE)
            self.cigars = np.empty(max(cap, 1), np.uint32)
            self.cigar_total = C.c_uint64()
            self._keepalive += [prio, cl, cr]
            self.realign = _lib.RegionRealign(prio.ctypes.data, cl.ctypes.data, cr.ctypes.data,
                                              self.best_hap.ctypes.data, self.sw_res.ctypes.data,
                                              self.cigars.ctypes.data, self.cigars.size,
                                              C.cast(C.byref(self.cigar_total), C.c_void_p))
            check(engine._lib.phmm_submit_region_realign(engine._h, C.byref(inp), ev_ptr, C.byref(self.realign),
                                                         _ptr(self.out), _ptr(self.keep), C.byref(self.n_kept),
                                                         C.byref(t)))
        else:
            check(engine._lib.phmm_submit_region(engine._h, C.byref(inp), ev_ptr, _ptr(self.out), _ptr(self.keep),
                                                 C.byref(self.n_kept), C.byref(t)))
        self.ticket = t.value

    def realignment(self):
        """(best haplotype per read, -1 for dropped reads; sw.SwResults of each read against it) after
        wait()."""
        from . import sw

        n = self.n_reads
        return self.best_hap[:n].copy(), sw.SwResults(self.sw_res[:n].copy(),
                                                     self.cigars[:self.cigar_total.value].copy(), sw.MAX_CIGAR)

    def wait(self):
        """Blocks until done; returns (matrix [n_haps][n_reads] with kept reads first or None, keep mask)."""
        self._engine.wait(self.ticket)
        mat = self.out.reshape(self.n_haps, self.n_reads) if self.out is not None else None
        return mat, self.keep[:self.n_reads].astype(bool)

    def genotypes(self):
        """Per event: (genotype log10 likelihoods, most likely genotype, allele likelihoods or None)."""
        res, go, ao = [], 0, 0
        for a in self._n_alleles.astype(int):
            g = a * (a + 1) // 2
            alk = None
            if self.allele_lk is not None:
                alk = self.allele_lk[ao:ao + a * self.n_reads].reshape(a, self.n_reads)
            res.append((self.gl[go:go + g].copy(), int(self.best[len(res)]), alk))
            go += g
            ao += a * self.n_reads
        return res


class ResidentBatch:
    """A batch uploaded once; run() recomputes it from HBM with no host transfers."""

    def __init__(self, engine: Engine, batch: PackedBatch, want_flags: bool = False):
        self._lib = engine._lib
        self.batch = batch
        self.want_flags = want_flags
        h = C.c_void_p()
        b = batch.as_c()
        check(self._lib.phmm_resident_create(engine._h, C.byref(b), int(want_flags), C.byref(h)))
        self._h = h

    def run(self, iterations: int = 1) -> dict:
        st = _lib.Stats()
        check(self._lib.phmm_resident_run(self._h, iterations, C.byref(st)))
        return st.as_dict()

    def profile(self) -> dict:
        """phmm_resident_profile: every kernel class alone, timed with CUDA events; returns
        class_ms and class_cells (FP32 classes first, then FP64) as arrays."""
        ms = np.zeros(_lib.FP32_CLASSES + _lib.FP64_CLASSES, np.float32)
        cells = np.zeros(_lib.FP32_CLASSES + _lib.FP64_CLASSES, np.uint64)
        check(self._lib.phmm_resident_profile(self._h, _ptr(ms), _ptr(cells)))
        return {"class_ms": ms, "class_cells": cells}

    def results(self):
        out = np.empty(self.batch.out_size, np.float64)
        fl = np.empty(self.batch.out_size, np.uint8) if self.want_flags else None
        check(self._lib.phmm_resident_results(self._h, _ptr(out), _ptr(fl)))
        return out, fl

    def check_fp64(self) -> np.ndarray:
        """phmm_resident_check_fp64: every pair of the batch recomputed on the device with the
        all-FP64 check arithmetic (the oracle's fp64_only model); overwrites the resident's results
        (run() again before results())."""
        out = np.empty(self.batch.out_size, np.float64)
        check(self._lib.phmm_resident_check_fp64(self._h, _ptr(out)))
        return out

    def close(self) -> None:
        if getattr(self, "_h", None):
            check(self._lib.phmm_resident_destroy(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def partition_regions(batch: PackedBatch, n_parts: int) -> tuple[np.ndarray, np.ndarray]:
    """phmm_partition_regions (host only): (part of every region, cells of every part), regions
    split by longest-processing-time greedy on their cells."""
    part = np.empty(batch.n_regions, np.uint32)
    cells = np.empty(n_parts, np.uint64)
    b = batch.as_c()
    check(_lib.load().phmm_partition_regions(C.byref(b), n_parts, _ptr(part), _ptr(cells)))
    return part, cells


class DeviceSet:
    """One engine per listed device behind one handle (phmm_device_set_*): batches split across
    the devices by region, serving requests routed to the least-loaded device."""

    def __init__(self, devices: Sequence[int], use_cuda_graph: bool = True, autotune: bool = True,
                 hbm_budget_bytes: int = 0, chunk_cells: int = 0):
        self._lib = _lib.load()
        devs = (C.c_int32 * len(devices))(*devices)
        cfg = _lib.Config(0, int(use_cuda_graph), int(autotune), 0, hbm_budget_bytes, chunk_cells)
        h = C.c_void_p()
        check(self._lib.phmm_device_set_create(devs, len(devices), C.byref(cfg), C.byref(h)))
        self._h = h
        self.devices = list(devices)

    def compute(self, batch: PackedBatch, want_flags: bool = False):
        """As Engine.compute, over every device of the set."""
        n = batch.out_size
        out = np.empty(n, np.float64)
        flags = np.empty(n, np.uint8) if want_flags else None
        st = _lib.Stats()
        b = batch.as_c()
        check(self._lib.phmm_device_set_compute_regions(self._h, C.byref(b), _ptr(out), _ptr(flags), C.byref(st)))
        return out, flags, st.as_dict()

    def submit(self, region: PackedBatch, out: np.ndarray, flags: np.ndarray | None = None) -> int:
        t = C.c_uint64()
        b = region.as_c()
        check(self._lib.phmm_device_set_submit(self._h, C.byref(b), _ptr(out), _ptr(flags), C.byref(t)))
        return t.value

    def wait(self, ticket: int, timeout_us: int = -1) -> tuple[float, float, int]:
        """(queued µs, total µs, index of the member that ran the request)."""
        q, tot, dev = C.c_double(), C.c_double(), C.c_uint32()
        check(self._lib.phmm_device_set_wait(self._h, ticket, timeout_us, C.byref(q), C.byref(tot), C.byref(dev)))
        return q.value, tot.value, dev.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            check(self._lib.phmm_device_set_destroy(self._h))
            self._h = None

    def __enter__(self) -> "DeviceSet":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_engine: Engine | None = None


def default_engine() -> Engine:
    global _default_engine
    if _default_engine is None:
        _default_engine = Engine()
    return _default_engine


def schedule_pairhmm(haplotypes, reads, quality, insertion_qualities, deletion_qualities, gap_contiguous_qualities,
                     engine: Engine | None = None):
    """Vector-API mirror: returns (ok, result) with result[read][hap] log10 likelihoods.

    Like the reference, no quality capping or PCR model is applied; ok is False (and result
    empty) when there are no haplotypes or no reads (roDV_schedule.cpp:179-181)."""
    if len(haplotypes) == 0 or len(reads) == 0:
        return False, np.zeros((0, 0))
    eng = engine or default_engine()
    reg = Region(list(haplotypes), list(reads), list(quality), list(insertion_qualities), list(deletion_qualities),
                 list(gap_contiguous_qualities))
    (mat,) = eng.compute_regions([reg])
    return True, np.ascontiguousarray(mat.T)


def call_pairhmm(haplotypes, reads, base_quals, mapq, min_quality_threshold: int = 18,
                 pcr_option: str | int = "CONSERVATIVE", engine: Engine | None = None):
    """HaplotypeCaller entry-point mirror: returns (result [hap][read], kept read indices).

    As in the reference, result has one column per input read; the first len(kept) columns hold the
    kept reads in order, the rest are NaN, and the caller erases the other reads."""
    eng = engine or default_engine()
    mat, keep = eng.call_region(haplotypes, reads, base_quals, mapq, min_quality_threshold, pcr_option)
    return mat, np.nonzero(keep)[0]


__all__ = ["Engine", "Region", "PackedBatch", "PhmmError", "schedule_pairhmm", "call_pairhmm", "default_engine",
           "plan_summary", "compute_noalloc", "partition_regions", "DeviceSet"]
