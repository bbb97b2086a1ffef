"""B200-native (sm_100a) Leeds Spherical Dynamo timestep hot path.

Submodules: capi (ABI structures), lsd (ctypes host interface), state (netCDF state
files), synthetic (seeded workloads), build (nvcc build of liblsd_b200.so).
Import with importlib.import_module("leeds-code_b200").
"""
from . import capi, state, synthetic  # noqa: F401
from .lsd import Context, Ensemble, LsdError, load_library  # noqa: F401
