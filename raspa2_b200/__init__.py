"""B200-native GCMC energy hot path of RASPA2.

- `systems`: seeded synthetic adsorption systems (frameworks, adsorbates).
- `raspa_io`: writes a system as RASPA2 input files.
- `native`: ctypes binding of libraspa_gpu.so (include/raspa_gpu.h): the
  reference-named per-call energy routines, grids and the persistent batched
  GCMC engine. There is no CPU fallback.
- `build`: in-tree nvcc build of the library for sm_100a.
"""
from . import units, systems  # noqa: F401

__all__ = ["units", "systems"]
