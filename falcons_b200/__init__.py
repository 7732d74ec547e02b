"""falcons_b200 — B200-native (sm_100a) implementation of the Falcons compression hot path.

Layers:
  libfalcons_b200.so   CUDA kernels + the C ABI (include/falcons_b200.h)
  falcons_b200._lib    ctypes binding of that ABI
  falcons_b200.device  stage-level entry points on device tensors
  falcons_b200.api     pyfalcons-compatible compress/decompress on NumPy arrays
"""
__version__ = "1.0.0"
