"""B200-native WCSPH step for ultraballpit: sm_100a CUDA kernels behind a C ABI.

The CUDA library (``libsph_cuda.so``, built from ``csrc/``) is the product; this
package holds its host-side mirror of the reference ``SimulationKernel``
interface (``kernel.CudaKernel``), the particle containers and the scenario
builders.
"""
from .particles import (BoundaryParticles, ErrorMetrics, FluidType, GridSDF,  # noqa: F401
                        ParticleArrays)
