"""B200 implementation of ORAC's nonbonded force path (host-side package).

liborac_gpu.so (built from ../csrc) holds the CUDA kernels and the C ABI of
include/orac_gpu.h; this package binds it (lib), mirrors the reference's
routine interface over it (engine), and builds synthetic ORAC systems
(systems, units).
"""
import os

# Independent systems of a batch run as parallel branches of one CUDA graph;
# the device executes at most CUDA_DEVICE_MAX_CONNECTIONS such branches at a
# time (8 unless set before the CUDA context is created).  Ask for the
# maximum when the caller has not chosen.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

__all__ = ["lib", "engine", "systems", "units"]
