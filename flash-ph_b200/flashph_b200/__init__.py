"""flashph_b200: exact Vietoris-Rips persistent homology on NVIDIA B200.

Drop-in for the public API of ot-triton-lab/flash-ph (``flash_ph``):
``rips_persistence``, ``auto_threshold``, ``enclosing_radius`` and
``RipsComplex``, computed by hand-written sm_100a CUDA kernels behind the C
ABI declared in ``include/flashph_b200.h``.
"""

__version__ = "0.1.0"

from .complex import RipsComplex
from .persistence import rips_persistence
from .threshold import auto_threshold, enclosing_radius

__all__ = ["rips_persistence", "auto_threshold", "enclosing_radius", "RipsComplex"]
