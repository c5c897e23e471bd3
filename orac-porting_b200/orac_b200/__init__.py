"""B200 implementation of ORAC's nonbonded force path (host-side package).

liborac_gpu.so (built from ../csrc) holds the CUDA kernels and the C ABI of
include/orac_gpu.h; this package binds it (lib), mirrors the reference's
routine interface over it (engine), and builds synthetic ORAC systems
(systems, units).
"""
__all__ = ["lib", "engine", "systems", "units"]
