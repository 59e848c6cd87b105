"""simulon_b200 -- B200-native (sm_100a) implementation of Simulon's per-step force path.

Hand-written CUDA kernels behind a C ABI (include/simb200.h, libsimb200.so)
with a Python host layer that mirrors the reference's plugin interfaces:

    AtomFileReader, Box, EAMParser, EAMForceCUDAExt / EAMForce, LennardJonesForce,
    VerletIntegrator, BerendsenBarostat, AnisotropicNPTBarostat,
    UniaxialTensileLoader, SphericalIndenterForce, SumBackboneInterface, BaseModel, MDSimulator,
    find_neighbors_gpu_pbc, and the legacy ``simulon_cuda`` module.
"""
from __future__ import annotations

import sys

from . import _lib
from .barostat import AnisotropicNPTBarostat, BerendsenBarostat
from .batch import BatchedEngine, CrackObserver, Replica, crack_slab, crack_sweep, partition_replicas
from .box import Box
from .eam_parser import EAMDeviceTables, EAMParser
from .engine import MDEngine
from .forces import BackboneInterface, EAMForce, EAMForceCUDA, EAMForceCUDAExt, LennardJonesForce
from .integrator import IntegratorInterface, VerletIntegrator
from .md_model import BaseModel, SumBackboneInterface
from .md_simulation import MDSimulator
from .mechanics import SphericalIndenterForce, UniaxialTensileLoader
from .neighbor import find_neighbors_gpu_pbc
from .reader import AtomFileReader
from .restart import load_checkpoint, save_checkpoint

__version__ = "0.1.0"


def install_simulon_cuda():
    """Register the drop-in as the top-level module ``simulon_cuda``."""
    from . import simulon_cuda
    sys.modules["simulon_cuda"] = simulon_cuda
    return simulon_cuda


__all__ = ["AtomFileReader", "Box", "EAMParser", "EAMDeviceTables", "EAMForce", "EAMForceCUDA", "EAMForceCUDAExt",
           "LennardJonesForce", "BackboneInterface", "IntegratorInterface", "VerletIntegrator",
           "BerendsenBarostat", "SumBackboneInterface", "BaseModel", "MDSimulator", "MDEngine",
           "find_neighbors_gpu_pbc", "install_simulon_cuda", "BatchedEngine", "Replica", "crack_slab",
           "crack_sweep", "partition_replicas", "AnisotropicNPTBarostat", "UniaxialTensileLoader",
           "SphericalIndenterForce", "CrackObserver", "save_checkpoint", "load_checkpoint"]
