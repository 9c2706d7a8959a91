"""crystalgraphics_b200 — a B200-native (sm_100a) backend for the View()
spectral path-tracing hot path of ray847/CrystalGraphics.

The CUDA library (libcg_cuda.so, include/cg_cuda.h) does the work; this
package holds its Python mirror of the reference's crystal::graphics API
(``backend``), the ctypes layouts (``_abi``), the seeded benchmark scenes
(``scenes``) and the build recipe (``build``).  Importing ``backend`` loads
the CUDA library and fails loudly if it is missing.
"""
__all__ = ["backend", "scenes", "build"]
