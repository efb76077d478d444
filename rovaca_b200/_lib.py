"""ctypes binding of include/phmm_b200.h (the engine's C ABI).

The library is built in-tree (``python -m rovaca_b200.build``).  There is no fallback: if the
library or a CUDA device is missing, calls raise instead of computing anything on the CPU.
"""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libphmm_b200.so"
HEADER_PATH = Path(__file__).resolve().parent.parent / "include" / "phmm_b200.h"

PHMM_OK = 0
PHMM_ERR_LIMIT_EXCEEDED = 2
STATUS_NAMES = {
    0: "PHMM_OK", 1: "PHMM_ERR_INVALID_ARGUMENT", 2: "PHMM_ERR_LIMIT_EXCEEDED", 3: "PHMM_ERR_OUT_OF_MEMORY",
    4: "PHMM_ERR_CUDA", 5: "PHMM_ERR_NOT_INITIALIZED", 6: "PHMM_ERR_TIMEOUT", 7: "PHMM_ERR_CANCELLED",
    8: "PHMM_ERR_QUEUE_FULL", 9: "PHMM_ERR_DEVICE_STATUS", 10: "PHMM_ERR_NO_DEVICE", 11: "PHMM_ERR_INTERNAL",
}
PCR_MODELS = {"NONE": 0, "HOSTILE": 1, "AGGRESSIVE": 2, "CONSERVATIVE": 3}


class PhmmError(RuntimeError):
    """A non-OK phmm_status, with the library's detail message."""

    def __init__(self, status: int, detail: str):
        self.status = status
        self.name = STATUS_NAMES.get(status, f"status {status}")
        super().__init__(f"{self.name}: {detail}" if detail else self.name)


class Config(C.Structure):
    _fields_ = [("device", C.c_int32), ("use_cuda_graph", C.c_int32), ("autotune", C.c_int32),
                ("reserved0", C.c_int32), ("hbm_budget_bytes", C.c_uint64), ("chunk_cells", C.c_uint64)]


class Batch(C.Structure):
    _fields_ = [("n_regions", C.c_uint32), ("n_haps", C.c_void_p), ("n_reads", C.c_void_p),
                ("hap_bases", C.c_void_p), ("hap_off", C.c_void_p), ("read_bases", C.c_void_p),
                ("read_qual", C.c_void_p), ("read_ins", C.c_void_p), ("read_del", C.c_void_p),
                ("read_gcp", C.c_void_p), ("read_off", C.c_void_p)]


class Stats(C.Structure):
    _fields_ = [("regions", C.c_uint64), ("pairs", C.c_uint64), ("cells", C.c_uint64), ("pairs_f64", C.c_uint64),
                ("work_items", C.c_uint64), ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64),
                ("kernel_launches", C.c_uint64), ("device_ms", C.c_double), ("fp32_ms", C.c_double),
                ("fp64_ms", C.c_double), ("host_ms", C.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


TILE_MODES, LEN_BUCKETS, FP32_CLASSES, FP64_CLASSES = 3, 24, 39, 27


class TileTable(C.Structure):
    """phmm_tile_table: row pairs per lane and multi-stripe flag per (mode, read-length bucket)."""
    _fields_ = [("rows_per_lane", (C.c_uint8 * LEN_BUCKETS) * TILE_MODES),
                ("multi_stripe", (C.c_uint8 * LEN_BUCKETS) * TILE_MODES)]

    def as_arrays(self):
        import numpy as np
        kh = np.array([[self.rows_per_lane[m][b] for b in range(LEN_BUCKETS)] for m in range(TILE_MODES)], np.uint8)
        mu = np.array([[self.multi_stripe[m][b] for b in range(LEN_BUCKETS)] for m in range(TILE_MODES)], np.uint8)
        return kh, mu

    @classmethod
    def from_arrays(cls, kh, multi) -> "TileTable":
        t = cls()
        for m in range(TILE_MODES):
            for b in range(LEN_BUCKETS):
                t.rows_per_lane[m][b] = int(kh[m][b])
                t.multi_stripe[m][b] = int(multi[m][b])
        return t


class TuneEntry(C.Structure):
    _fields_ = [("mode", C.c_uint8), ("bucket", C.c_uint8), ("rows_per_lane", C.c_uint8),
                ("multi_stripe", C.c_uint8), ("chosen", C.c_uint8), ("reserved", C.c_uint8 * 3),
                ("gcups", C.c_float)]


TUNE_MAX_ENTRIES = 512


class TuneReport(C.Structure):
    _fields_ = [("n_entries", C.c_uint32), ("reserved", C.c_uint32), ("seconds", C.c_double),
                ("entries", TuneEntry * TUNE_MAX_ENTRIES)]


class RegionInput(C.Structure):
    """phmm_region_input: one region for the region API."""
    _fields_ = [("n_haps", C.c_uint32), ("hap_bases", C.c_void_p), ("hap_off", C.c_void_p),
                ("n_reads", C.c_uint32), ("read_bases", C.c_void_p), ("read_qual", C.c_void_p),
                ("read_off", C.c_void_p), ("mapq", C.c_void_p), ("min_quality_threshold", C.c_int32),
                ("pcr_model", C.c_int32)]


class RegionEvents(C.Structure):
    """phmm_region_events: genotyping events of one region."""
    _fields_ = [("n_events", C.c_uint32), ("n_alleles", C.c_void_p), ("hap_allele", C.c_void_p),
                ("genotype_lk", C.c_void_p), ("best_genotype", C.c_void_p), ("allele_lk", C.c_void_p)]


class ServerStats(C.Structure):
    _fields_ = [("requests_submitted", C.c_uint64), ("requests_done", C.c_uint64), ("batches", C.c_uint64),
                ("max_batch_regions", C.c_uint64), ("queue_peak", C.c_uint64), ("cells_done", C.c_uint64),
                ("batch_ms", C.c_double), ("device_ms", C.c_double), ("max_batch_ms", C.c_double),
                ("max_queue_ms", C.c_double), ("arena_grows", C.c_uint64), ("graph_captures", C.c_uint64),
                ("max_setup_ms", C.c_double), ("max_host_ms", C.c_double), ("gather_ms", C.c_double),
                ("plan_ms", C.c_double), ("enqueue_ms", C.c_double), ("wait_ms", C.c_double), ("scatter_ms", C.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class RegionRealign(C.Structure):
    """phmm_region_realign: realignment of a region's kept reads to their best haplotypes."""
    _fields_ = [("hap_priority", C.c_void_p), ("clip_left", C.c_void_p), ("clip_right", C.c_void_p),
                ("best_hap", C.c_void_p), ("sw", C.c_void_p), ("cigars", C.c_void_p), ("cigar_capacity", C.c_uint64),
                ("cigar_total", C.c_void_p)]


class SwItem(C.Structure):
    """phmm_sw_item: one alignment (haplotype = seq1, read = seq2) as offsets into two base buffers."""
    _fields_ = [("hap_offset", C.c_uint64), ("read_offset", C.c_uint64), ("hap_len", C.c_uint32),
                ("read_len", C.c_uint32)]


class SwResult(C.Structure):
    _fields_ = [("score", C.c_int32), ("alignment_offset", C.c_int32), ("max_i", C.c_int32), ("max_j", C.c_int32),
                ("cigar_count", C.c_uint32), ("cigar_offset", C.c_uint32)]


_lib = None


def load() -> C.CDLL:
    """Loads libphmm_b200.so (once) and declares every entry point's signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m rovaca_b200.build`")
    lib = C.CDLL(str(LIB_PATH))
    P, U32, U64, I32, I64, D = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int32, C.c_int64, C.c_double
    sig = {
        "phmm_engine_create": (I32, [C.POINTER(Config), C.POINTER(P)]),
        "phmm_engine_destroy": (I32, [P]),
        "phmm_status_string": (C.c_char_p, [I32]),
        "phmm_last_error": (C.c_char_p, []),
        "phmm_version": (C.c_char_p, []),
        "phmm_compute_regions": (I32, [P, C.POINTER(Batch), P, P, C.POINTER(Stats)]),
        "phmm_call_region": (I32, [P, U32, P, P, U32, P, P, P, P, I32, I32, P, P, C.POINTER(U32)]),
        "phmm_host_prepare_quals": (None, [P, U32, C.c_uint8, I32, P]),
        "phmm_host_pcr_model": (None, [P, U32, P, I32]),
        "phmm_host_tandem_repeat_length": (I32, [P, U32, U32]),
        "phmm_host_normalize_filter": (None, [P, U32, U32, P, P, P, C.POINTER(U32)]),
        "phmm_resident_create": (I32, [P, C.POINTER(Batch), I32, C.POINTER(P)]),
        "phmm_resident_run": (I32, [P, I32, C.POINTER(Stats)]),
        "phmm_resident_results": (I32, [P, P, P]),
        "phmm_resident_check_fp64": (I32, [P, P]),
        "phmm_resident_destroy": (I32, [P]),
        "phmm_fp32_fma_peak": (I32, [P, C.POINTER(D), C.POINTER(D)]),
        "phmm_compute_regions_noalloc": (I32, [C.POINTER(Batch), P, P, I32]),
        "phmm_host_plan_summary": (I32, [C.POINTER(Batch), P, P, P, C.POINTER(U64), C.POINTER(U64)]),
        "phmm_tile_table_default": (None, [P]),
        "phmm_engine_get_tiles": (I32, [P, P]),
        "phmm_engine_set_tiles": (I32, [P, P]),
        "phmm_engine_autotune": (I32, [P, P]),
        "phmm_submit": (I32, [P, C.POINTER(Batch), P, P, C.POINTER(U64)]),
        "phmm_submit_region": (I32, [P, P, P, P, P, C.POINTER(U32), C.POINTER(U64)]),
        "phmm_resident_profile": (I32, [P, P, P]),
        "phmm_poll": (I32, [P, U64, C.POINTER(I32)]),
        "phmm_wait": (I32, [P, U64, I64, C.POINTER(D), C.POINTER(D)]),
        "phmm_cancel": (I32, [P, U64]),
        "phmm_server_stats_get": (I32, [P, P]),
        "phmm_submit_region_realign": (I32, [P, P, P, P, P, P, C.POINTER(U32), C.POINTER(U64)]),
        "phmm_sw_align": (I32, [P, P, I32, U32, P, P, U64, P, U64, U32, P, P, U64, C.POINTER(U64)]),
        "phmm_sw_resident_create": (I32, [P, P, I32, U32, P, P, U64, P, U64, U32, C.POINTER(P)]),
        "phmm_sw_resident_run": (I32, [P, I32, C.POINTER(C.c_float), P]),
        "phmm_sw_resident_results": (I32, [P, P, P, U64, C.POINTER(U64)]),
        "phmm_sw_resident_destroy": (I32, [P]),
        "phmm_partition_regions": (I32, [C.POINTER(Batch), U32, P, P]),
        "phmm_device_set_create": (I32, [P, U32, C.POINTER(Config), C.POINTER(P)]),
        "phmm_device_set_destroy": (I32, [P]),
        "phmm_device_set_engine": (I32, [P, U32, C.POINTER(P)]),
        "phmm_device_set_compute_regions": (I32, [P, C.POINTER(Batch), P, P, C.POINTER(Stats)]),
        "phmm_device_set_submit": (I32, [P, C.POINTER(Batch), P, P, C.POINTER(U64)]),
        "phmm_device_set_wait": (I32, [P, U64, I64, C.POINTER(D), C.POINTER(D), C.POINTER(U32)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def check(status: int) -> None:
    if status != PHMM_OK:
        detail = load().phmm_last_error().decode(errors="replace")
        raise PhmmError(status, detail)


def declared_symbols() -> list[str]:
    """Every function include/phmm_b200.h declares."""
    text = HEADER_PATH.read_text()
    return sorted(set(re.findall(r"^PHMM_API\s+[\w\s\*]+?\b(phmm_\w+)\s*\(", text, flags=re.M)))
