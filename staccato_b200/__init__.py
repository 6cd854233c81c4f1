"""B200-native reduced-order frequency sweep (STACCATO KMOR ROM path).

Layers:
  * ``libstaccato_rom.so``  hand-written sm_100a kernels behind the C ABI of
    ``include/staccato_rom.h`` (built by ``staccato_b200/build.py``);
  * ``_capi``               ctypes binding of that ABI;
  * ``sweep``               batched sweep over device (torch) or host (numpy) buffers;
  * ``rom``                 ``KrylovROMSubstructure``: the reference's ROM interface;
  * ``workloads``           seeded synthetic ROMs of the benchmarked shapes.
"""
from . import _capi  # noqa: F401

__all__ = ["_capi", "sweep", "workloads", "rom"]
