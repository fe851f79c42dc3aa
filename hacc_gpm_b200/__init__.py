"""B200-native particle-mesh step for HACC_GPM's serial path.

The product is native: CUDA kernels for sm_100a and a C-ABI library
(``_lib/libhgpm.so``, declared in ``include/hgpm_c.h``) plus a C++ drop-in
driver (``_lib/haccgpm``).  This package holds the sources (``csrc/``,
``host/``), the in-tree build (``build.py``), the Python binding of the
C-ABI (``binding.py``), the batched ensemble / serving front ends and the
``.ipk`` writer.
"""
from .binding import (HgpmError, Params, Simulation, Timestepper, footprint_bytes, growth, lib, parse_params,
                      read_ipk, read_params, write_pk)

__all__ = ["HgpmError", "Params", "Simulation", "Timestepper", "footprint_bytes", "growth", "lib", "parse_params",
           "read_ipk", "read_params", "write_pk"]
