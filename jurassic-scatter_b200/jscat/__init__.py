"""Python host side of the B200 JURASSIC-scatter forward model.

The computation lives in libjurassic_b200.so (C host code + sm_100a CUDA
kernels); this package only declares its C-ABI (lib), mirrors the boundary
structs (structs), wraps the calls (api) and generates the seeded synthetic
workloads used by the tests and the benchmark (synth).
"""
from . import structs
from .api import Batch, Model, brightness, formod, formod_batch, launch_count

__all__ = ["structs", "Batch", "Model", "brightness", "formod",
           "formod_batch", "launch_count"]
