"""scadyn_b200 — B200-native T-matrix solve path of jherrane/scadyn.

The product is ``libscadyn_gpu.so`` (C ABI in include/scadyn_gpu.h, sm_100a
kernels in csrc/); ``api`` mirrors the reference's solver interface over it;
``meshgen`` builds seeded synthetic meshes; ``build`` compiles the library.
"""
