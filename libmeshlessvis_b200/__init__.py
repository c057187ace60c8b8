"""B200-native (sm_100a) drop-in for libMeshlessVis's hot path: the direct
nonuniform Fourier sum of basis-function transforms over a 3D Hermitian
half-spectrum, Fourier-slice extraction per view and the batched 2D C2R, behind
the reference's C API (include/meshless.h, include/meshless_vis.h).

The product is libmeshless_vis.so (CUDA + C++ under csrc/); the Python modules
describe and call its C ABI.
"""
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libmeshless_vis.so"
