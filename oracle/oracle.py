"""Python access to the PairHMM oracle (test infrastructure only).

* ``Oracle`` -- the C restatement in oracle/phmm_oracle.c (built into oracle/_build/).
* ``Ref``    -- the reference's own kernels and vector-API scheduler, compiled from the reference
  sources by oracle/build_ref.sh into oracle/_ref/ (present wherever that recipe has run).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module, as the checker;
the engine in rovaca_b200/ never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SRC = HERE / "phmm_oracle.c"
ORACLE_SCHED_SRC = HERE / "phmm_oracle_sched.cpp"
ORACLE_SW_SRC = HERE / "sw_oracle.c"
ORACLE_LIB = HERE / "_build" / "libphmm_oracle.so"
REF_LIB = HERE / "_ref" / "libphmm_ref.so"

INTER, INTRA = 0, 1
UNFUSED, FUSED = 0, 1


def build_oracle(force: bool = False) -> Path:
    """Compiles oracle/_build/libphmm_oracle.so (no FMA contraction beyond the explicit fma calls)."""
    ORACLE_LIB.parent.mkdir(exist_ok=True)
    srcs = (ORACLE_SRC, ORACLE_SCHED_SRC, ORACLE_SW_SRC)
    if force or not ORACLE_LIB.exists() or any(ORACLE_LIB.stat().st_mtime < s.stat().st_mtime for s in srcs):
        flags = ["-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-Wall"]
        tmp = ORACLE_LIB.parent
        subprocess.run(["gcc", *flags, "-c", str(ORACLE_SRC), "-o", str(tmp / "phmm_oracle.o")], check=True)
        subprocess.run(["gcc", *flags, "-c", str(ORACLE_SW_SRC), "-o", str(tmp / "sw_oracle.o")], check=True)
        subprocess.run(["g++", *flags, "-std=c++17", "-c", str(ORACLE_SCHED_SRC), "-o", str(tmp / "phmm_oracle_sched.o")],
                       check=True)
        subprocess.run(["g++", "-shared", "-o", str(ORACLE_LIB), str(tmp / "phmm_oracle.o"),
                        str(tmp / "phmm_oracle_sched.o"), str(tmp / "sw_oracle.o"), "-lm"], check=True)
    return ORACLE_LIB


def reference_root() -> str | None:
    """The reference's source tree, read in place by the build recipes and the fixture generators:
    the REFERENCE_ROOT environment variable (None when unset; the build functions then keep the
    libraries already built).  Nothing on the GPU host reads it (the built oracle/_ref libraries
    travel instead)."""
    return os.environ.get("REFERENCE_ROOT") or None


def build_ref(root: str | None = None) -> Path | None:
    """Builds oracle/_ref from the reference sources when they are present; returns the library."""
    src = root or reference_root()
    if src is None or not Path(src, "src/haplotypecaller/pairhmm").is_dir():
        return REF_LIB if REF_LIB.exists() else None
    srcs = [HERE / "ref_shim.cpp", HERE / "ref_kernels.cpp", HERE / "ref_region.cpp", HERE / "ref_unreached.cpp",
            HERE / "build_ref.sh"]
    if REF_LIB.exists() and all(REF_LIB.stat().st_mtime >= s.stat().st_mtime for s in srcs):
        return REF_LIB
    subprocess.run(["bash", str(HERE / "build_ref.sh"), src], check=True)
    return REF_LIB


SW_REF_LIB = HERE / "_ref" / "libsw_ref.so"


def build_ref_sw(root: str | None = None) -> Path | None:
    """Builds oracle/_ref/libsw_ref.so (the reference's Smith-Waterman aligner) when the reference
    sources are present; returns the library."""
    src = root or reference_root()
    if src is None or not Path(src, "src/haplotypecaller/common/base/lib/ro_sw").is_dir():
        return SW_REF_LIB if SW_REF_LIB.exists() else None
    srcs = [HERE / "ref_sw_shim.c", HERE / "build_ref_sw.sh"]
    if SW_REF_LIB.exists() and all(SW_REF_LIB.stat().st_mtime >= s.stat().st_mtime for s in srcs):
        return SW_REF_LIB
    subprocess.run(["bash", str(HERE / "build_ref_sw.sh"), src], check=True)
    return SW_REF_LIB


GENOTYPE_REF_LIB = HERE / "_ref" / "libgenotype_ref.so"


def build_ref_genotype(root: str | None = None) -> Path | None:
    """Builds oracle/_ref/libgenotype_ref.so (the reference's allele marginalisation and diploid
    genotype-likelihood calculator) when the reference sources are present; returns the library."""
    src = root or reference_root()
    if src is None or not Path(src, "src/haplotypecaller/genotype/genotype_likelihood_calculator.cpp").is_file():
        return GENOTYPE_REF_LIB if GENOTYPE_REF_LIB.exists() else None
    deps = [HERE / "ref_genotype_shim.cpp", HERE / "build_ref_genotype.sh",
            *sorted((HERE / "ref_stubs" / "boost" / "math" / "special_functions").glob("*.hpp"))]
    if GENOTYPE_REF_LIB.exists() and all(GENOTYPE_REF_LIB.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return GENOTYPE_REF_LIB
    subprocess.run(["bash", str(HERE / "build_ref_genotype.sh"), src], check=True)
    return GENOTYPE_REF_LIB


class GenotypeRef:
    """The reference's own genotyping arithmetic (oracle/_ref/libgenotype_ref.so): for one sample
    at ploidy 2, AlleleLikelihoods::marginalize (allele_likelihoods.hpp:189-221,702-730) and
    GenotypeLikelihoodCalculator::genotype_likelihoods (genotype_likelihood_calculator.h:44-142)."""

    def __init__(self, path: Path | str | None = None):
        p = Path(path) if path else GENOTYPE_REF_LIB
        if not p.exists():
            raise FileNotFoundError(f"{p} not built (oracle/build_ref_genotype.sh needs the reference sources)")
        self.lib = C.CDLL(str(p))
        self.lib.ref_genotype.restype = C.c_int
        self.lib.ref_genotype.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                          C.c_void_p]

    def genotype(self, lk_hr: np.ndarray, hap_allele, n_alleles: int) -> tuple[np.ndarray, np.ndarray]:
        """lk_hr: [hap][read] normalised likelihoods of the kept reads; hap_allele: allele of each
        haplotype (-1: none).  Returns (allele likelihoods [allele][read], genotype likelihoods)."""
        lk = np.ascontiguousarray(lk_hr, np.float64)
        H, N = lk.shape
        ha = np.ascontiguousarray(np.asarray(hap_allele, np.int8))
        if ha.size != H:
            raise ValueError("hap_allele needs one entry per haplotype")
        alk = np.empty((n_alleles, N), np.float64)
        gl = np.empty(n_alleles * (n_alleles + 1) // 2, np.float64)
        rc = self.lib.ref_genotype(H, N, lk.ctypes.data, n_alleles, ha.ctypes.data, alk.ctypes.data, gl.ctypes.data)
        if rc != 0:
            raise ValueError(f"ref_genotype: alleles {n_alleles} outside the reference's limits")
        return alk, gl


class SwRef:
    """The reference's Smith-Waterman aligner (oracle/_ref/libsw_ref.so), as HaplotypeCaller calls
    it to realign a read to its best haplotype: seq1 = haplotype, seq2 = read."""

    GENOTYPING = (10, -15, -30, -5)   # sw_parameters_genotype, lib/sw_avx/sw_avx.c:15
    ASSEMBLY = (200, -150, -260, -11)  # sw_parameters_assemble, lib/sw_avx/sw_avx.c:14

    def __init__(self, path: Path | str | None = None):
        p = Path(path) if path else SW_REF_LIB
        if not p.exists():
            raise FileNotFoundError(f"{p} not built (oracle/build_ref_sw.sh)")
        self.lib = C.CDLL(str(p))
        self.lib.ref_sw_align.restype = C.c_int
        self.lib.ref_sw_align.argtypes = [C.c_char_p, C.c_int, C.c_char_p, C.c_int, C.c_void_p, C.c_int,
                                          C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                          C.POINTER(C.c_int32), C.c_void_p, C.c_int]
        self.lib.ref_sw_uses_int32.restype = C.c_int
        self.lib.ref_sw_uses_int32.argtypes = [C.c_int, C.c_int, C.c_int]

    def align(self, hap: bytes, read: bytes, params=GENOTYPING, variant: int = 0):
        """-> (score, alignment_offset, max_i, max_j, [cigar ops as (len << 4) | op])."""
        prm = (C.c_int32 * 4)(*params)
        cig = (C.c_uint32 * 4096)()
        sc, off, mi, mj = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        n = self.lib.ref_sw_align(bytes(hap), len(hap), bytes(read), len(read), C.cast(prm, C.c_void_p), variant,
                                  C.byref(sc), C.byref(off), C.byref(mi), C.byref(mj), C.cast(cig, C.c_void_p), 4096)
        return sc.value, off.value, mi.value, mj.value, list(cig[:max(n, 0)])

    def uses_int32(self, hap_len: int, read_len: int, match: int) -> bool:
        return bool(self.lib.ref_sw_uses_int32(hap_len, read_len, match))


class SwOracle:
    """The C restatement of the reference's Smith-Waterman aligner (oracle/sw_oracle.c)."""

    GENOTYPING = SwRef.GENOTYPING
    ASSEMBLY = SwRef.ASSEMBLY

    def __init__(self):
        self.lib = C.CDLL(str(build_oracle()))
        self.lib.sw_oracle_align.restype = C.c_int
        self.lib.sw_oracle_align.argtypes = [C.c_char_p, C.c_int, C.c_char_p, C.c_int, C.c_void_p, C.c_int,
                                             C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                             C.POINTER(C.c_int32), C.c_void_p, C.c_int]
        self.lib.sw_oracle_uses_int32.restype = C.c_int
        self.lib.sw_oracle_uses_int32.argtypes = [C.c_int, C.c_int, C.c_int]

    def align(self, hap: bytes, read: bytes, params=GENOTYPING, variant: int = 0):
        """-> (score, alignment_offset, max_i, max_j, [cigar ops as (len << 4) | op])."""
        prm = (C.c_int32 * 4)(*params)
        cig = (C.c_uint32 * 4096)()
        sc, off, mi, mj = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        n = self.lib.sw_oracle_align(bytes(hap), len(hap), bytes(read), len(read), C.cast(prm, C.c_void_p), variant,
                                     C.byref(sc), C.byref(off), C.byref(mi), C.byref(mj), C.cast(cig, C.c_void_p),
                                     4096)
        if n < 0:
            raise MemoryError("sw_oracle_align: allocation failed")
        return sc.value, off.value, mi.value, mj.value, list(cig[:n])

    def uses_int32(self, hap_len: int, read_len: int, match: int) -> bool:
        return bool(self.lib.sw_oracle_uses_int32(hap_len, read_len, match))


def cigar_string(ops) -> str:
    return "".join(f"{c >> 4}{'MIDNSHP=XB'[c & 15]}" for c in ops)


def _b(x) -> bytes:
    if isinstance(x, (bytes, bytearray)):
        return bytes(x)
    if isinstance(x, str):
        return x.encode()
    return np.ascontiguousarray(np.asarray(x, np.uint8)).tobytes()


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class Oracle:
    def __init__(self):
        lib = C.CDLL(str(build_oracle()))
        cp, u32, i32, D, F = C.c_char_p, C.c_uint32, C.c_int, C.c_double, C.c_float
        pair = [cp, u32, cp, u32, cp, cp, cp, cp]
        for name, res, extra in [("oracle_raw_f32", F, [i32, i32]), ("oracle_raw_f64", D, [i32, i32]),
                                 ("oracle_log10_f64", D, []),
                                 ("oracle_log10_switch", D, [i32, i32, C.POINTER(C.c_int)])]:
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = pair + extra
        lib.oracle_log10_from_f32.restype = D
        lib.oracle_log10_from_f32.argtypes = [F]
        for name, res in [("oracle_ph2pr_f32", F), ("oracle_ph2pr_f64", D)]:
            getattr(lib, name).restype = res
            getattr(lib, name).argtypes = [i32]
        for name, res in [("oracle_mm_f32", F), ("oracle_mm_f64", D)]:
            getattr(lib, name).restype = res
            getattr(lib, name).argtypes = [i32, i32]
        P = C.c_void_p
        lib.oracle_batch.restype = C.c_uint64
        lib.oracle_batch.argtypes = [u32, P, P, P, P, P, P, P, P, P, P, i32, i32, P, P]
        lib.oracle_schedule.restype = i32
        lib.oracle_schedule.argtypes = [u32, P, P, u32, P, P, P, P, P, P, D, D, u32, u32, P, P]
        self.lib = lib

    @staticmethod
    def _args(hap, read, q, i, d, c):
        hap, read = _b(hap), _b(read)
        return [hap, len(hap), read, len(read), _b(q), _b(i), _b(d), _b(c)]

    def raw_f32(self, hap, read, q, i, d, c, kernel=INTER, fused=FUSED) -> float:
        return self.lib.oracle_raw_f32(*self._args(hap, read, q, i, d, c), kernel, fused)

    def raw_f64(self, hap, read, q, i, d, c, kernel=INTER, fused=FUSED) -> float:
        return self.lib.oracle_raw_f64(*self._args(hap, read, q, i, d, c), kernel, fused)

    def log10_f64(self, hap, read, q, i, d, c) -> float:
        """All-FP64 oracle (plain multiply/add, inter prior)."""
        return self.lib.oracle_log10_f64(*self._args(hap, read, q, i, d, c))

    def pair(self, hap, read, q, i, d, c, kernel=None, fused=FUSED) -> tuple[float, bool]:
        """Reference semantics for one pair: FP32, FP64 below 1e-28; N pairs on the intra variant."""
        if kernel is None:
            kernel = INTRA if (b"N" in _b(hap) or b"N" in _b(read)) else INTER
        u = C.c_int()
        v = self.lib.oracle_log10_switch(*self._args(hap, read, q, i, d, c), kernel, fused, C.byref(u))
        return v, bool(u.value)

    def batch(self, pb, fused=FUSED, fp64_only=False):
        """A PackedBatch with reference semantics: (likelihoods, used_f64) in the engine's layout."""
        n = pb.out_size
        out = np.empty(n, np.float64)
        used = np.empty(n, np.uint8)
        self.lib.oracle_batch(pb.n_regions, _p(pb.n_haps), _p(pb.n_reads), _p(pb.hap_bases), _p(pb.hap_off),
                              _p(pb.read_bases), _p(pb.read_qual), _p(pb.read_ins), _p(pb.read_del), _p(pb.read_gcp),
                              _p(pb.read_off), fused, int(fp64_only), _p(out), _p(used))
        return out, used.astype(bool)


    # routes of oracle_schedule: which reference kernel and precision produced a pair
    ROUTE_F64 = (1, 3, 4)

    def schedule_region(self, pb, g: int, idle_f: float = 0.02, idle_d: float = 0.02, width_f: int = 16,
                        width_d: int = 8):
        """Region g through the restated vector-API scheduler (AVX-512 widths by default).

        Returns (log10 [hap][read], route [hap][read]); route codes are listed in
        oracle/phmm_oracle_sched.cpp, and route in ROUTE_F64 means the pair ended in FP64."""
        h0, r0 = int(pb.n_haps[:g].sum()), int(pb.n_reads[:g].sum())
        m, n = int(pb.n_haps[g]), int(pb.n_reads[g])
        hoff = np.ascontiguousarray(pb.hap_off[h0:h0 + m + 1])
        roff = np.ascontiguousarray(pb.read_off[r0:r0 + n + 1])
        out = np.empty(m * n, np.float64)
        route = np.empty(m * n, np.uint8)
        rc = self.lib.oracle_schedule(m, _p(pb.hap_bases), _p(hoff), n, _p(pb.read_bases), _p(pb.read_qual),
                                      _p(pb.read_ins), _p(pb.read_del), _p(pb.read_gcp), _p(roff), idle_f, idle_d,
                                      width_f, width_d, _p(out), _p(route))
        if rc != 0:
            raise ValueError("oracle_schedule: empty region")
        return out.reshape(m, n), route.reshape(m, n)


class Ref:
    """The reference's own PairHMM (oracle/_ref/libphmm_ref.so)."""

    def __init__(self, path: Path | str | None = None):
        p = Path(path) if path else REF_LIB
        if not p.exists():
            raise FileNotFoundError(f"{p} not built (oracle/build_ref.sh needs the reference sources)")
        lib = C.CDLL(str(p))
        cp, u32, i32, D, F, P = C.c_char_p, C.c_uint32, C.c_int, C.c_double, C.c_float, C.c_void_p
        pair = [cp, u32, cp, u32, cp, cp, cp, cp]
        lib.ref_init.restype = None
        lib.ref_isa_bits.restype = i32
        lib.ref_inter_width_f32.restype = i32
        lib.ref_inter_width_f64.restype = i32
        lib.ref_intra_raw_f32.restype = F
        lib.ref_intra_raw_f32.argtypes = pair
        lib.ref_intra_raw_f64.restype = D
        lib.ref_intra_raw_f64.argtypes = pair
        lib.ref_intra_log10.restype = D
        lib.ref_intra_log10.argtypes = pair + [i32]
        lib.ref_inter.restype = i32
        lib.ref_inter.argtypes = [i32, u32, P, P, P, P, P, P, P, P, i32, P]
        lib.ref_schedule.restype = i32
        lib.ref_schedule.argtypes = [u32, P, P, u32, P, P, P, P, P, P, D, D, P]
        lib.ref_init()
        self.lib = lib
        self.isa = lib.ref_isa_bits()
        self.width_f32 = lib.ref_inter_width_f32()
        self.width_f64 = lib.ref_inter_width_f64()

    def init_thread(self) -> None:
        """Flush-to-zero on the calling thread, as the reference sets it (pairhmm_engine.cpp:36)."""
        self.lib.ref_init()

    def intra_raw_f32(self, hap, read, q, i, d, c) -> float:
        return self.lib.ref_intra_raw_f32(*Oracle._args(hap, read, q, i, d, c))

    def intra_raw_f64(self, hap, read, q, i, d, c) -> float:
        return self.lib.ref_intra_raw_f64(*Oracle._args(hap, read, q, i, d, c))

    def intra_log10(self, hap, read, q, i, d, c, use_double=False) -> float:
        return self.lib.ref_intra_log10(*Oracle._args(hap, read, q, i, d, c), int(use_double))

    def inter(self, pairs, dbl=False, raw=True) -> np.ndarray:
        """pairs: exactly width_f32 (or width_f64) tuples (hap, read, q, i, d, c)."""
        n = len(pairs)
        cols = [[_b(p[k]) for p in pairs] for k in range(6)]
        arrs = [(C.c_char_p * n)(*col) for col in cols]
        hl = (C.c_uint32 * n)(*[len(x) for x in cols[0]])
        rl = (C.c_uint32 * n)(*[len(x) for x in cols[1]])
        out = (C.c_double * n)()
        rc = self.lib.ref_inter(int(dbl), n, arrs[0], hl, arrs[1], rl, arrs[2], arrs[3], arrs[4], arrs[5], int(raw), out)
        if rc != 0:
            raise ValueError(f"ref_inter returned {rc} (needs exactly the SIMD width of pairs)")
        return np.array(out[:], np.float64)

    def schedule_region(self, pb, g: int, idle_f: float = 0.02, idle_d: float = 0.02) -> np.ndarray:
        """Region g of a PackedBatch through schedule_pairhmm; returns [hap][read] (engine layout)."""
        h0, r0 = int(pb.n_haps[:g].sum()), int(pb.n_reads[:g].sum())
        m, n = int(pb.n_haps[g]), int(pb.n_reads[g])
        hoff = np.ascontiguousarray(pb.hap_off[h0:h0 + m + 1])
        roff = np.ascontiguousarray(pb.read_off[r0:r0 + n + 1])
        out = np.empty(n * m, np.float64)
        rc = self.lib.ref_schedule(m, _p(pb.hap_bases), _p(hoff), n, _p(pb.read_bases), _p(pb.read_qual),
                                   _p(pb.read_ins), _p(pb.read_del), _p(pb.read_gcp), _p(roff), idle_f, idle_d, _p(out))
        if rc != 0:
            raise RuntimeError(f"ref_schedule failed ({rc})")
        return out.reshape(n, m).T.copy()


def ref_available() -> bool:
    return REF_LIB.exists()


__all__ = ["Oracle", "Ref", "build_oracle", "build_ref", "ref_available", "INTER", "INTRA", "FUSED", "UNFUSED"]
