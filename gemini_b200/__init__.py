"""B200-native (sm_100a) GEMINI3D multifluid fluid advance.

The MC-limited advection sweeps, the device ghost fill that replaces the MPI halo, and the
TRBDF2 field-aligned heat diffusion, on the reference's own memory blocks resident in GPU
memory.  ``gemini_b200.fluid`` holds the reference-named routines; the C ABI is in
``include/gem_fluid.h`` (device pointers) and ``include/gemini3d_fluid.h`` (the reference's
``*_C`` entry points over host memory).
"""
from . import grid, state  # noqa: F401  (numpy-only; the native library loads on first use)

__version__ = "0.1.0"
