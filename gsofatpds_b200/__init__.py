"""gsofatpds_b200 -- B200-native (sm_100a) fill-path symbolic LU factorization.

The compute path is libgsofa.so (CUDA kernels behind the C-ABI in
include/gsofa.h); this package is its Python host interface plus the seeded
input generators.  Importing works without a GPU; the first call that needs
the library loads it and raises if it is missing.
"""
from .api import (Batch, Context, GsofaError, Matrix, Result, Server, convert_dat,  # noqa: F401
                  read_binary, symbfact_min_id, write_binary)
from . import gen  # noqa: F401

__all__ = ["Batch", "Context", "GsofaError", "Matrix", "Result", "Server", "symbfact_min_id",
           "write_binary", "read_binary", "convert_dat", "gen"]
