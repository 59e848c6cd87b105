"""Barostats with the interfaces of core/barostat.py: Berendsen (:21-75) and
the diagonal anisotropic controller (:78-208).

Pressure, the scaling factor and the box update are computed on the device
in FP64 from the FP64 kinetic and virial tensors; ``step`` returns the
pressure in bar as a device scalar (``float(p)`` synchronises).

The reference scales ``molecular.coordinates`` and ``graph_data.pos`` -- the
same tensor -- so coordinates are multiplied by mu twice while the box and
velocities are multiplied by mu once, and ``last_positions`` is reset after
every step.  Those behaviours are the defaults here
(``coordinate_scale_power=2``, ``reset_reference=True``) so that results
match; pass 1 / False to scale coordinates and box consistently and keep the
skin/2 reference across steps.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from .engine import berendsen_params

_EV_ANG3_TO_BAR = 1_602_176.6208


class BerendsenBarostat:
    def __init__(self, molecular, target_pressure: float, tau_p: float, compressibility: float = 4.57e-5,
                 mu_max: float = 0.05, coordinate_scale_power: int = 2, reset_reference: bool = True):
        self.molecular = molecular
        self.target_P = float(target_pressure)
        self.tau_p = float(tau_p)
        self.kappa = float(compressibility)
        self.mu_max = float(mu_max)
        self.coordinate_scale_power = int(coordinate_scale_power)
        self.reset_reference = bool(reset_reference)
        self._params = {}

    def params(self, dt: float):
        if dt not in self._params:
            self._params[dt] = berendsen_params(dt, self.target_P, self.tau_p, self.kappa, self.mu_max,
                                                self.coordinate_scale_power, self.reset_reference)
        return self._params[dt]

    def step(self, dt: float, kinetic_energy=None, virial=None, kinetic_tensor=None, virial_tensor=None):
        """Uses the device's kinetic and virial tensors of the current step."""
        eng = self.molecular.engine
        eng.berendsen(self.params(dt))
        return eng.extra[0]

    def controller(self, dt: float):
        """step() without the atoms' scaling, which the next step's first half
        applies (deferred_first_half); for runs of several steps."""
        self.molecular.engine.berendsen_mu(self.params(dt))
        return self.molecular.engine.extra[0]

    def deferred_first_half(self, integrator):
        """The atoms' scaling of the last controller() call, then
        integrator.first_half() (kick, drift, skin/2 trigger, conditional
        rebuild), with the scaling and the half-step in one pass."""
        eng = self.molecular.engine
        eng.berendsen_scale_first(self.params(integrator.dt), integrator.params, integrator.force_precision)
        eng.rebuild_if_needed()

    def pressure(self) -> torch.Tensor:
        """Pressure (bar) of the last step (device scalar)."""
        return self.molecular.engine.extra[0]

    def sync_box(self):
        """Copy the device box back into molecular.box (synchronises)."""
        self.molecular.box.H = self.molecular.engine.box_matrix()


class AnisotropicNPTBarostat:
    """Diagonal anisotropic pressure controller (barostat.py:78-208) on the
    device in FP64: the log strain rate eta_dot of each lattice axis follows
    d eta_dot / dt = kappa (P_axis - P_target) / tau_p^2 - gamma_p eta_dot with
    a deadband of pressure_tolerance_bar, is clamped to +-max_eta_dot, and
    scales the box rows by exp(dt eta_dot) and the velocities by
    exp(-dt eta_dot); positions follow through fractional coordinates and are
    wrapped.  ``step`` returns the axis pressures (bar) as a device tensor.
    stochastic=True adds the reference's thermal noise from Philox normals
    (the reference draws torch.randn; the distributions agree, the draws do
    not).  As in the reference the skin reference is reset every step
    (reset_reference=False keeps it)."""

    def __init__(self, molecular, target_pressure_bar, temperature_k: float, tau_p: float = 0.2,
                 gamma_p: float = 2.0, control_axes=(True, True, True), max_eta_dot: float = 0.05,
                 compressibility_bar_inv: float = 3.2e-7, pressure_tolerance_bar: float = 25.0,
                 stochastic: bool = False, seed: int = 0, reset_reference: bool = True):
        self.molecular = molecular
        eng = molecular.engine
        self.device = eng.device
        tp = [float(v) for v in torch.as_tensor(target_pressure_bar, dtype=torch.float64).reshape(-1).tolist()]
        if len(tp) == 1:
            tp = tp * 3
        if len(tp) != 3:
            raise ValueError("target_pressure_bar must be scalar or length-3")
        ca = [bool(v) for v in control_axes]
        if len(ca) != 3:
            raise ValueError("control_axes must have length 3")
        self.target_pressure_bar = torch.tensor(tp, dtype=torch.float64, device=self.device)
        self.control_axes = torch.tensor(ca, dtype=torch.bool, device=self.device)
        self.temperature_k = float(temperature_k)
        self.tau_p, self.gamma_p, self.max_eta_dot = float(tau_p), float(gamma_p), float(max_eta_dot)
        self.compressibility_bar_inv = float(compressibility_bar_inv)
        self.pressure_tolerance_bar = float(pressure_tolerance_bar)
        self.stochastic = bool(stochastic)
        self.eta_dot = torch.zeros(3, dtype=torch.float64, device=self.device)
        self.counter = torch.zeros(1, dtype=torch.int64, device=self.device)
        self.work = torch.zeros(_lib.BOXSCALE_WORK, dtype=torch.float64, device=self.device)
        self._st = _lib.SimAniso()
        s = self._st
        s.target_bar[:] = tp
        s.tau_p, s.gamma_p, s.max_eta_dot = self.tau_p, self.gamma_p, self.max_eta_dot
        s.kappa_bar_inv, s.tol_bar = self.compressibility_bar_inv, self.pressure_tolerance_bar
        s.temperature = self.temperature_k
        s.eta_dot, s.counter = _lib.ptr(self.eta_dot), _lib.ptr(self.counter)
        s.control[:] = [int(v) for v in ca]
        s.stochastic = int(self.stochastic)
        s.reset_reference = int(bool(reset_reference))
        s.seed = int(seed) & 0xFFFFFFFF
        self._ref = ctypes.byref(s)

    def step(self, dt: float, kinetic_energy=None, virial=None, kinetic_tensor=None, virial_tensor=None):
        """Uses the device's kinetic and virial tensors of the current step."""
        eng = self.molecular.engine
        self._st.dt = float(dt)
        _lib.call("sim_aniso_npt", eng.st_ref, self._ref, _lib.ptr(self.work), eng.stream)
        return self.work[0:3]

    def controller(self, dt: float):
        """step() without moving the atoms: the axis pressures, the strain-rate
        update and the new box are prepared in ``work``; a loader's next
        update moves the atoms for both (UniaxialTensileLoader.launch_after)."""
        eng = self.molecular.engine
        self._st.dt = float(dt)
        _lib.call("sim_aniso_control", eng.st_ref, self._ref, _lib.ptr(self.work), eng.stream)
        return self.work[0:3]

    def pressure(self) -> torch.Tensor:
        """Axis pressures (bar) of the last step (device tensor)."""
        return self.work[0:3]

    def sync_box(self):
        """Copy the device box back into molecular.box (synchronises)."""
        self.molecular.box.H = self.molecular.engine.box_matrix()
