"""Force-field plugins with the reference's BackboneInterface contract.

``forward() -> {'energy', 'forces', 'virial', 'virial_tensor', ...}`` exactly as
core/force/lennard_jones_force.py:15-95 and core/force/eam_force_cu.py:461-579
return them, computed by the device kernels on the engine state.  The returned
mapping is lazy: 'forces' is gathered into the caller's atom order only when
it is read; the energies and virials are device scalars (no host sync).
"""
from __future__ import annotations

from collections.abc import Mapping

import numpy as np
import torch
import torch.nn as nn

from . import _lib
from .eam_parser import EAMDeviceTables, EAMParser
from .engine import DeviceStruct


class LazyOutputs(Mapping):
    """Mapping whose values are computed on first access and cached."""

    def __init__(self, **producers):
        self._producers = producers
        self._cache = {}

    def __getitem__(self, key):
        if key not in self._cache:
            self._cache[key] = self._producers[key]()
        return self._cache[key]

    def __iter__(self):
        return iter(self._producers)

    def __len__(self):
        return len(self._producers)


class BackboneInterface(nn.Module):
    """Force-field plugin (core/md_model.py:9-12)."""

    def forward(self):
        raise NotImplementedError


def _force_outputs(mol, extra=None):
    eng = mol.engine
    dt = mol.dtype
    red = eng.red_out
    prod = dict(
        energy=lambda: eng.potential_energy().to(dt),
        forces=lambda: eng.gather("f").to(dt),
        virial=lambda: red[_lib.RED_VIRIAL].to(dt),
        virial_tensor=lambda: eng.virial_tensor().to(dt),
    )
    prod.update(extra or {})
    return LazyOutputs(**prod)


class EAMForceCUDAExt(BackboneInterface):
    """Two-pass EAM on the device (EAMForceCUDAExt, eam_force_cu.py:316-579)."""

    def __init__(self, eam_parser: EAMParser, molecular, n_r: int = 8192, n_rho: int = 4096,
                 use_extension: bool = True):
        super().__init__()
        if not use_extension:
            raise ValueError("simulon_b200 has no host fallback; use_extension must be True")
        self.parser = eam_parser
        self.molecular = molecular
        self.device = molecular.device
        self.cutoff = float(eam_parser.cutoff)
        self.n_r, self.n_rho = n_r, n_rho
        missing = [a for a in molecular.elements if a not in eam_parser.element_map]
        if missing:
            raise KeyError(f"elements {missing} not in the potential file")
        # the engine's type ids follow first appearance in the structure; the
        # tables follow the file's element order -> remap when they differ
        order = [eam_parser.element_map[a] for a in molecular.elements]
        if order != list(range(len(order))) or len(order) != len(eam_parser.elements):
            raise NotImplementedError("structure element order must match the potential file's element order")
        self.tables = EAMDeviceTables(eam_parser, self.device, n_r=n_r, n_rho=n_rho)
        self.E = len(eam_parser.elements)
        self.force_precision = 0

    def compute(self):
        self.molecular.engine.eam_forces(self.tables)

    def compute_and_finish(self, integrator):
        """Forces plus the integrator's second half in one pass over the atoms."""
        self.molecular.engine.eam_forces_integrate(self.tables, integrator.params)

    def compute_finish_and_drift(self, integrator):
        """Forces, the integrator's second half and the next step's first half
        in one pass over the atoms."""
        self.molecular.engine.eam_forces_integrate_drift(self.tables, integrator.params)

    def compute_finish_with_indenter(self, integrator, indenter, mode: int):
        """Forces with a SphericalIndenterForce added in the same pass, and the
        integrator's second half (mode 1) or both half-steps (mode 2)."""
        self.molecular.engine.eam_forces_integrate_indenter(self.tables, integrator.params, indenter._ref, mode)

    def step_drift_with_indenter(self, integrator, indenter):
        """compute_finish_with_indenter(mode 2), the step's log row and the
        conditional list rebuild, the last two decided inside the force pass."""
        self.molecular.engine.eam_step_drift_indenter(self.tables, integrator.params, indenter._ref)

    def step_and_drift(self, integrator):
        """compute_finish_and_drift, the step's log row and the conditional
        list rebuild, with the last two decided inside the force pass."""
        self.molecular.engine.eam_step_drift(self.tables, integrator.params)

    def forward(self):
        self.compute()
        red = self.molecular.engine.red_out
        dt = self.molecular.dtype
        return _force_outputs(self.molecular, dict(
            embedding_energy=lambda: red[_lib.RED_EPOT_EMBED].to(dt),
            pair_potential=lambda: red[_lib.RED_EPOT_PAIR].to(dt)))


class EAMForce(EAMForceCUDAExt):
    """core/force/eam_force.py:5-391 (table path) -- same device kernels."""

    def __init__(self, eam_parser: EAMParser, molecular, use_tables: bool = True, n_r: int = 8192,
                 n_rho: int = 4096):
        if not use_tables:
            raise ValueError("only the uniform-table EAM path is provided")
        super().__init__(eam_parser, molecular, n_r=n_r, n_rho=n_rho)


EAMForceCUDA = EAMForceCUDAExt


def lj_type_pair_params(parameter: dict, n_types: int, rc: float, device):
    """Per type-pair constants formed exactly as the reference forms them.

    The reference keeps per-edge epsilon/sigma as float32 tensors
    (reader.py:193-207), so 4*eps, 24*eps and the force-shift constants
    (lennard_jones_force.py:66-75) are float32 products; they are reproduced
    here with float32 torch ops and handed to the kernels as doubles.
    """
    keys = {}
    for a in range(n_types):
        for b in range(n_types):
            k = str(np.array([a, b]))
            if k not in parameter:
                k = str(np.array([b, a]))
            if k not in parameter:
                raise KeyError(f"no LJ parameters for pair {a}-{b}")
            keys[(a, b)] = k
    eps = torch.tensor([parameter[keys[(a, b)]]["epsilon"] for a in range(n_types) for b in range(n_types)],
                       dtype=torch.float32)
    sig = torch.tensor([parameter[keys[(a, b)]]["sigma"] for a in range(n_types) for b in range(n_types)],
                       dtype=torch.float32)
    c4 = 4.0 * eps
    c24 = 24.0 * eps
    sr_rc = sig / rc
    sr6_rc = sr_rc ** 6
    sr12_rc = sr6_rc ** 2
    u_rc = 4.0 * eps * (sr12_rc - sr6_rc)
    f_rc = 24.0 * eps * (1.0 / rc) * (2.0 * sr12_rc - sr6_rc)
    to = dict(device=device, dtype=torch.float64)
    return {k: v.to(**to) for k, v in dict(c4eps=c4, c24eps=c24, sigma=sig, u_rc=u_rc, f_rc=f_rc).items()}


class LennardJonesForce(BackboneInterface):
    """Lennard-Jones on the device (lennard_jones_force.py:7-95), modes raw /
    force-shift (is_fs) / quintic switch (is_switch).  FP64 pair arithmetic
    when the system's dtype is float64, FP32 otherwise."""

    def __init__(self, molecular):
        super().__init__()
        self.molecular = molecular
        eng = molecular.engine
        rc = float(molecular.cutoff)
        self.is_switch = bool(getattr(molecular, "is_switch", False))
        self.is_fs = bool(getattr(molecular, "is_fs", False))
        mode = _lib_mode(self.is_switch, self.is_fs)
        rs = float(molecular.switch_ratio) * rc if self.is_switch else 0.0
        self.tensors = lj_type_pair_params(molecular.parameter, eng.n_types, rc, eng.device)
        s = _lib.SimLJParams()
        for k, t in self.tensors.items():
            setattr(s, k, _lib.ptr(t))
        s.n_types, s.mode, s.rc, s.rs = eng.n_types, mode, rc, rs
        self.params = DeviceStruct(s, list(self.tensors.values()))
        self.ref = self.params.ref
        self.force_precision = 1 if molecular.dtype == torch.float64 else 0

    def compute(self):
        self.molecular.engine.lj_forces(self.params, self.force_precision)

    def add_to_engine(self, force_precision: int = 0):
        """As a further backbone of a SumBackboneInterface (md_model.py:39-46):
        the LJ forces, energy and virials are added to the engine's, which the
        first backbone wrote (FP32 pairs)."""
        if force_precision != 0:
            raise NotImplementedError("LJ is summed onto FP32 forces only (the first force field computes FP32 "
                                      "forces)")
        eng = self.molecular.engine
        _lib.call("sim_lj_forces_add", eng.st_ref, self.params.ref, eng.stream)

    def compute_and_finish(self, integrator):
        """Forces plus the integrator's second half (one pass over the atoms for
        FP32 pairs; the FP64 path runs the two separately)."""
        eng = self.molecular.engine
        if self.force_precision == 0:
            eng.lj_forces_integrate(self.params, integrator.params, 1)
        else:
            eng.lj_forces(self.params, 1)
            eng.integrate_second(integrator.params, 1)

    def compute_finish_and_drift(self, integrator):
        """Forces, the integrator's second half and the next step's first half
        (one pass for FP32 pairs; FP64: forces, then sim_integrate_second_first)."""
        eng = self.molecular.engine
        if self.force_precision == 0:
            eng.lj_forces_integrate(self.params, integrator.params, 2)
        else:
            eng.lj_forces(self.params, 1)
            eng.integrate_second_first(integrator.params, 1)

    def forward(self):
        self.compute()
        return _force_outputs(self.molecular)


def _lib_mode(is_switch: bool, is_fs: bool) -> int:
    if is_switch:
        return 2
    if is_fs:
        return 1
    return 0
