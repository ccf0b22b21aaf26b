"""B200-native lighting hot path of the instantradiositytest renderer.

ReSTIR direct and VPL-indirect candidate generation, temporal and spatial
reservoir reuse, SDF soft-shadow visibility through a stackless BVH and SVGF,
as hand-written sm_100a CUDA behind the C-ABI of include/irt.h (libirt.so).

Modules:
  _lib      ctypes binding of libirt.so (fails loudly when it is not built)
  workload  seeded procedural rooms and the host input producers
  runtime   context / scene / session handles and a frame driver (torch for
            device memory and streams)
"""
from . import _lib  # noqa: F401  (raises ImportError when libirt.so is missing)
