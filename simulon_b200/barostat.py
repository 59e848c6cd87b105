"""Berendsen barostat with the interface of core/barostat.py:21-75.

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

    def sync_box(self):
        """Copy the device box back into molecular.box (synchronises)."""
        self.molecular.box.H = self.molecular.engine.box_matrix()
