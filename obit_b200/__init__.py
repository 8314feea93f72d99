"""B200-native DFT sky-model predict / subtract for Obit-layout visibility data.

The compute path is libobit_dft.so (hand-written sm_100a CUDA behind a C ABI,
include/obit_dft.h); this package holds its ctypes bindings, the Python face of
the GPU sky-model class, and seeded synthetic workloads.
"""
from .uvdata import SkyComps, UVData, Workload  # noqa: F401

__version__ = "0.1.0"
