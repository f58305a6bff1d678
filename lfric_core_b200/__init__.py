"""B200-native LFRic linear-solver hot path.

The compute path is hand-written CUDA for sm_100a in liblfg.so (C ABI in
include/lfg.h); this package holds the host-side set-up (meshes, seeded
problems), the Python front end of the ABI and the autograd extension.
Importing the package does not load the library; api.Context() does, and
fails loudly if the library or a CUDA device is missing.
"""
__all__ = ["mesh", "problems", "api"]
