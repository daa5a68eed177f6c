"""B200-native HPL single-process solve path.

The compute lives in libhplb200.so (sm_100a CUDA behind the C ABI declared in
include/hplb.h); this package is the thin host-side mirror of rocHPL's
interface for the path: HPL_pdmatgen / HPL_pdgesv / the HPL_pdtest residual
check (see rochpl_b200.hpl), plus the ctypes binding itself.

There is no CPU fallback: importing the binding without the built library, or
calling it without a CUDA device, raises.
"""
from .lib import HplError, Library, library  # noqa: F401
from .hpl import (Algo, Pmat, HPL_pdgesv, HPL_pdmatgen, HPL_pdtest, default_ld,  # noqa: F401
                  hpl_flops, parse_hpl_dat)

__all__ = ["HplError", "Library", "library", "Algo", "Pmat", "HPL_pdgesv", "HPL_pdmatgen",
           "HPL_pdtest", "default_ld", "hpl_flops", "parse_hpl_dat"]
