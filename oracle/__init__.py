"""PairHMM oracle: test infrastructure that checks the CUDA engine (see oracle/oracle.py)."""
from .oracle import (FUSED, INTER, INTRA, UNFUSED, GenotypeRef, Oracle, Ref, SwOracle, SwRef, build_oracle, build_ref,
                     build_ref_genotype, build_ref_sw, cigar_string, ref_available)

__all__ = ["GenotypeRef", "Oracle", "Ref", "SwOracle", "SwRef", "build_oracle", "build_ref", "build_ref_genotype",
           "build_ref_sw", "cigar_string", "ref_available",
           "INTER", "INTRA", "FUSED", "UNFUSED"]
