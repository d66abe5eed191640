"""tapas-reduce_b200: B200-native (sm_100a) Tapas N-body evaluation path.

The compute lives in libtapas_b200.so (hand-written CUDA, C ABI in
include/tapas_b200.h).  This package is its Python host side:

* ``Context``   - one GPU context: partition (octree build), upward, traverse,
                  downward, results; the phases of the reference's
                  ``TapasFMM::Partition`` / ``TapasFMM::Map`` calls in
                  sample/exafmm-dev-13274dd4ac68/examples/tapas_exafmm.cxx:550-641.
* ``datasets``  - seeded synthetic body sets.
* ``build``     - compiles the CUDA library in-tree.

Importing the package never falls back to a CPU path: without the built
library, ``Context`` raises.
"""
from ._lib import (DEVICE, FP64, HOST, MIXED, ORDER_ORIGINAL, ORDER_SORTED, Context,  # noqa: F401
                   TapasError, lib, read_sources, read_targets, write_main_csv, write_sources,
                   write_targets)
from . import datasets  # noqa: F401

__all__ = ["Context", "TapasError", "lib", "datasets", "FP64", "MIXED", "HOST", "DEVICE",
           "ORDER_SORTED", "ORDER_ORIGINAL", "read_sources", "read_targets", "write_sources",
           "write_targets", "write_main_csv"]
