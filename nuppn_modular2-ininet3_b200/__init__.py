"""B200-native stiff reaction-network integration (NuPPN's per-zone hot path) behind a C ABI.

Import as ``importlib.import_module("nuppn_modular2-ininet3_b200")`` (the directory name is not a
Python identifier). Submodules:

* ``abi``       ctypes mirror of include/nuppn.h
* ``synthnet``  seeded synthetic networks in the reference's slot layout
* ``workloads`` the benchmark / test workloads (zone batches)
* ``solver``    ``NetworkSolver``: the reference-shaped entry points over the CUDA library
* ``build``     in-tree compilation of the CUDA library (sm_100a)
"""
from . import abi, synthnet  # noqa: F401

__all__ = ["abi", "synthnet", "solver", "workloads", "build"]
