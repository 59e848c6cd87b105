"""Velocity-Verlet integrator with the interface of core/integrator/integrator.py.

NVE, NVT (Langevin) and NPT (Langevin + a Berendsen barostat driven by
BaseModel).  Units eV, A, ps, amu; ``dt`` in ps, ``gamma`` in 1/ps.  The
state is FP64 on the device; the Langevin noise is Philox4x32-10 keyed by
(seed, original atom index, step), so it is reproducible and independent of
the cell order.
"""
from __future__ import annotations

import torch
import torch.nn as nn

from .engine import MASS_TO_INTERNAL, integrator_params
from .forces import LazyOutputs


class IntegratorInterface(nn.Module):
    """Integrator plugin (core/md_model.py:14-17)."""

    def forward(self, force):
        raise NotImplementedError


class VerletIntegrator(IntegratorInterface):
    BOLTZMAN = 8.617333262e-5
    N_a = 6.02214076e23
    J_per_ev = 1.60218e-19

    def __init__(self, molecular, dt: float, ensemble: str | None = None, temperature=None, gamma=None,
                 force_field=None, seed: int = 0):
        super().__init__()
        self.molecular = molecular
        self.dt = dt
        self.ensemble = (ensemble or "NVE").upper()
        self.atom_mass = (molecular.atom_mass.to(molecular.dtype).unsqueeze(-1).expand(-1, 3)
                          * (10.0 / (self.N_a * self.J_per_ev)))
        self.is_langevin_thermostat = self.ensemble in ("NVT", "NPT")
        if self.is_langevin_thermostat:
            if temperature is None or gamma is None:
                raise ValueError(f"ensemble='{self.ensemble}' needs both temperature and gamma")
            self.temperature = torch.tensor(float(temperature[1]), device=molecular.device)
            self.gamma = torch.tensor(float(gamma), device=molecular.device)
            molecular.set_maxwell_boltzmann_velocity(torch.tensor(float(temperature[0]), device=molecular.device))
            self.params = integrator_params(molecular.engine, dt, langevin=True, temperature=float(temperature[1]),
                                            gamma=float(gamma), seed=seed)
        else:
            self.params = integrator_params(molecular.engine, dt)
        self.force_precision = 0

    @property
    def new_coords(self):
        return self.molecular.coordinates

    @property
    def vel_half(self):
        return self.molecular.atom_velocities

    def first_half(self, forces_old=None):
        """v += 0.5 F/m dt; x += v dt; skin/2 trigger; conditional list rebuild."""
        eng = self.molecular.engine
        eng.integrate_first(self.params, self.force_precision)
        eng.rebuild_if_needed()

    def second_half(self, forces_new=None):
        eng = self.molecular.engine
        eng.integrate_second(self.params, self.force_precision)
        return self._outputs()

    def _outputs(self):
        eng = self.molecular.engine
        dt = self.molecular.dtype
        n = self.molecular.atom_count
        ke = lambda: eng.red_out[9].to(dt)
        return LazyOutputs(update_coordinates=lambda: self.molecular.coordinates,
                           kinetic_energy=ke,
                           temperature=lambda: (2.0 / 3.0) * ke() / (n * self.BOLTZMAN))

    def forward(self, force=None):
        self.first_half()
        self.second_half()
        return self._outputs()


__all__ = ["IntegratorInterface", "VerletIntegrator", "MASS_TO_INTERNAL"]
