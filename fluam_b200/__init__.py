"""fluam_b200: a B200 (sm_100a) implementation of fluam's Stokes-limit
immersed-boundary step, as the C-ABI library libfluamsl.so plus a Python
mirror of its interface.

The package holds only what the path needs: ``csrc/`` (CUDA kernels, the C
ABI and the data.main driver), ``build.py`` (nvcc recipe), ``_lib.py``
(ctypes binding) and ``stokes.py`` (the Python interface).
"""
from .stokes import (PAIR_NONE, PAIR_SOFT, PAIR_TABLE_LJ, RFD_PAPER, RFD_REFERENCE,
                     SCHEME_FIRST_ORDER, SCHEME_INCOMPRESSIBLE, SCHEME_MIDPOINT, SCHEME_QUASI2D,
                     SCHEME_STOKES2D, Batch,
                     Server, StokesLimit, make_config,
                     parse_data_main, run_data_main)

__all__ = ["StokesLimit", "Batch", "Server", "make_config", "run_data_main", "parse_data_main", "PAIR_NONE",
           "PAIR_SOFT", "PAIR_TABLE_LJ", "RFD_PAPER", "RFD_REFERENCE", "SCHEME_MIDPOINT",
           "SCHEME_FIRST_ORDER", "SCHEME_QUASI2D", "SCHEME_STOKES2D", "SCHEME_INCOMPRESSIBLE"]
