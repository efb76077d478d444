"""B200-native PairHMM likelihood engine (drop-in for the HaplotypeCaller PairHMM path).

The engine is libphmm_b200.so (C ABI in include/phmm_b200.h); this package is its Python host
interface, the seeded workload generators and the in-tree build.
"""
from .pairhmm import (DeviceSet, Engine, PackedBatch, PhmmError, Region, call_pairhmm, default_engine, partition_regions,
                      schedule_pairhmm)
from .sw import SwBatch, SwResident

__all__ = ["DeviceSet", "Engine", "PackedBatch", "PhmmError", "Region", "SwBatch", "SwResident", "call_pairhmm",
           "default_engine", "partition_regions", "schedule_pairhmm"]
