"""PairHMM oracle: test infrastructure that checks the CUDA engine (see oracle/oracle.py)."""
from .oracle import FUSED, INTER, INTRA, UNFUSED, Oracle, Ref, build_oracle, build_ref, ref_available

__all__ = ["Oracle", "Ref", "build_oracle", "build_ref", "ref_available", "INTER", "INTRA", "FUSED", "UNFUSED"]
