"""Oracle integrator, barostat and step order (TEST INFRASTRUCTURE ONLY).

Restates, on CPU tensors in a chosen dtype:

* VerletIntegrator (core/integrator/integrator.py:45-124)
    mass [N,3] in eV ps^2/A^2 = amu * 10/(N_A * 1.60218e-19)          (:61-64)
    Langevin: damp = exp(-g dt), rff = sqrt(kB T/m (1 - exp(-2 g dt)))  (:84-88)
    first_half : a = F/m; v_half = v + 0.5 a dt; x += v_half dt          (:91-99)
    second_half: v = v_half damp + xi rff; v += 0.5 (F'/m) dt;
                 K = sum 0.5 m v^2; T = 2K/(3 N kB)                      (:102-124)
* BerendsenBarostat.step (core/barostat.py:36-68)
    P = tr(K_t + W_t)/(3V) [eV/A^3] -> bar (x 1 602 176.6208);
    mu^3 = 1 + kappa dt/tau (P - P0), clamped to [(1-mu_max)^3, (1+mu_max)^3];
    box scaled by mu; coordinates scaled by mu TWICE (the reference scales
    ``coordinates`` and ``graph_data.pos``, which are the same tensor);
    velocities by mu; last_positions reset to the scaled coordinates.
* BaseModel.forward order (core/md_model.py:88-166): first call computes
  forces; first_half -> update_coordinates (skin/2 trigger, rebuild) ->
  forces -> second_half -> K recomputed -> optional barostat with
  K_t = sum m v (x) v (:83-86).
"""
from __future__ import annotations

import numpy as np
import torch

from .box import OracleBox
from . import neighbor as onb

BOLTZMAN = 8.617333262e-5
N_A = 6.02214076e23
J_PER_EV = 1.60218e-19
EV_ANG3_TO_BAR = 1_602_176.6208


def mass_internal(masses_amu, dtype=torch.float64):
    m = torch.as_tensor(np.asarray(masses_amu, np.float64)).to(dtype)
    return m.unsqueeze(-1).expand(-1, 3) * (10.0 / (N_A * J_PER_EV))


class OracleVerlet:
    def __init__(self, masses_amu, dt: float, ensemble: str = "NVE", temperature=None, gamma=None,
                 dtype=torch.float64):
        self.dtype = dtype
        self.dt = dt
        self.ensemble = (ensemble or "NVE").upper()
        self.atom_mass = mass_internal(masses_amu, dtype)
        self.langevin = self.ensemble in ("NVT", "NPT")
        if self.langevin:
            T = torch.tensor(float(temperature), dtype=dtype)
            g = torch.tensor(float(gamma), dtype=dtype)
            self.damp = torch.exp(-g * dt)
            self.rff = torch.sqrt((BOLTZMAN * T) / self.atom_mass * (1.0 - torch.exp(-2.0 * g * dt)))

    def first_half(self, x, v, F):
        accel = F / self.atom_mass
        vh = v + 0.5 * accel * self.dt
        return x + vh * self.dt, vh

    def second_half(self, vh, F, xi=None):
        vel = vh
        if self.langevin:
            vel = vel * self.damp + xi.to(self.dtype) * self.rff
        accel = F / self.atom_mass
        vel = vel + 0.5 * accel * self.dt
        ke = (0.5 * self.atom_mass * vel.pow(2)).sum()
        return vel, ke, (2.0 / 3.0) * ke / (vel.shape[0] * BOLTZMAN)


def berendsen(box: OracleBox, coords, vel, dt, K_t, W_t, P0, tau, kappa=4.57e-5, mu_max=0.05,
              coordinate_scale_power: int = 2):
    V = box.volume
    stress = (K_t.to(torch.float64) + W_t.to(torch.float64)) / V
    P = float(torch.trace(stress) / 3.0) * EV_ANG3_TO_BAR
    mu3 = 1.0 + kappa * (dt / tau) * (P - P0)
    mu3 = max(mu3, (1.0 - mu_max) ** 3)
    mu3 = min(mu3, (1.0 + mu_max) ** 3)
    mu = mu3 ** (1.0 / 3.0)
    box.scale(mu)
    for _ in range(coordinate_scale_power):
        coords = coords * mu
    return coords, vel * mu, P, mu


def aniso_npt(box: OracleBox, coords, vel, eta_dot, dt, K_t, W_t, target_bar, tau_p=0.2, gamma_p=2.0,
              control=(True, True, True), max_eta_dot=0.05, kappa=3.2e-7, tol=25.0):
    """AnisotropicNPTBarostat.step without its optional noise (barostat.py:137-208):
    returns (new wrapped coordinates, velocities, axis pressures in bar, eta_dot);
    box.H is updated."""
    f64 = torch.float64
    p_int = (K_t.to(f64) + W_t.to(f64)) / box.volume
    axes = box.H / torch.linalg.norm(box.H, dim=1, keepdim=True).clamp_min(1e-12)
    p_axis_bar = torch.einsum("ai,ij,aj->a", axes, p_int, axes) * EV_ANG3_TO_BAR
    target = torch.as_tensor(target_bar, dtype=f64).reshape(-1).expand(3)
    ctrl = torch.as_tensor(control, dtype=torch.bool)
    delta = p_axis_bar - target
    within = delta.abs() <= tol
    accel = kappa * torch.where(within, torch.zeros_like(delta), delta) / max(tau_p ** 2, 1e-12)
    if gamma_p > 0.0:
        accel = accel - gamma_p * eta_dot
    if bool(within.any()):
        accel = torch.where(within, -max(gamma_p, 5.0) * eta_dot, accel)
    eta = torch.clamp(eta_dot + dt * accel, -max_eta_dot, max_eta_dot)
    eta = torch.where(ctrl, eta, torch.zeros_like(eta))
    eta = torch.where(within & (eta.abs() < 1e-7), torch.zeros_like(eta), eta)
    scale = torch.where(ctrl, torch.exp(dt * eta), torch.ones_like(eta))
    frac = coords.to(f64) @ box.H_inv
    box.H = torch.diag(scale) @ box.H
    box._refresh()
    new = box.wrap_positions(frac @ box.H)
    vs = torch.where(ctrl, torch.exp(-dt * eta), torch.ones_like(eta))
    return new, vel * vs.unsqueeze(0), p_axis_bar, eta


def uniaxial_box_step(box: OracleBox, coords, dt, axis=0, strain_rate=1e-3, lateral_mode="fixed",
                      poisson_ratio=0.28, max_lateral_scale_step=2e-3):
    """UniaxialTensileLoader.step's box and coordinate update (loading.py:41-73):
    returns the new wrapped coordinates; box.H is updated."""
    dstrain = strain_rate * float(dt)
    scale = torch.ones(3, dtype=torch.float64)
    scale[axis] = 1.0 + dstrain
    if lateral_mode == "poisson":
        lat = max(1.0 - poisson_ratio * dstrain, 1.0 - max_lateral_scale_step)
        for ax in range(3):
            if ax != axis:
                scale[ax] = lat
    frac = coords.to(torch.float64) @ box.H_inv
    box.H = torch.diag(scale) @ box.H
    box._refresh()
    return box.wrap_positions(frac @ box.H)


def indenter(x, center, radius, stiffness):
    """SphericalIndenterForce.forward (indenter.py:40-68): forces, energy,
    virial (F (x) x), force on the indenter and contact count, FP64."""
    x = x.to(torch.float64)
    disp = x - torch.as_tensor(center, dtype=torch.float64)
    dist = torch.linalg.norm(disp, dim=1).clamp_min(1e-12)
    pen = radius - dist
    act = pen > 0.0
    F = torch.zeros_like(x)
    W = torch.zeros(3, 3, dtype=torch.float64)
    E = torch.zeros((), dtype=torch.float64)
    if bool(act.any()):
        fv = stiffness * pen[act].pow(2).unsqueeze(1) * (disp[act] / dist[act].unsqueeze(1))
        F[act] = fv
        E = stiffness / 3.0 * pen[act].pow(3).sum()
        W = torch.einsum("ni,nj->ij", fv, x[act])
    return dict(forces=F, energy=E, virial=torch.trace(W), virial_tensor=W, force_on_indenter=-F.sum(0),
                contact_atoms=int(act.sum()))


class OracleMD:
    """CPU restatement of one reference MD step (the timed CPU baseline too).

    ``force_fn(x, i, j) -> dict`` computes forces from a half list.
    ``noise_fn(step) -> [N,3]`` supplies Langevin normals (Philox by default).
    """

    def __init__(self, x, v, masses_amu, box: OracleBox, force_fn, cutoff: float, skin: float,
                 dt: float, ensemble="NVE", temperature=None, gamma=None, dtype=torch.float64,
                 noise_fn=None, barostat=None):
        self.dtype = dtype
        self.x = torch.as_tensor(x).to(dtype).clone()
        self.v = torch.as_tensor(v).to(dtype).clone()
        self.box = box
        self.force_fn = force_fn
        self.integ = OracleVerlet(masses_amu, dt, ensemble, temperature, gamma, dtype)
        self.rc2 = onb.rc2_like_reference(cutoff, skin, np.float32 if dtype == torch.float32 else np.float64)
        self.skin = skin
        self.skin_half = torch.tensor(skin, dtype=dtype) / 2
        self.noise_fn = noise_fn
        self.barostat = barostat
        self.last = None
        self.F = None
        self.step_index = 0
        self.rebuilds = 0
        self.eta_dot = torch.zeros(3, dtype=torch.float64)
        self._rebuild()

    def _rebuild(self):
        hl = onb.half_list(self.x.numpy(), self.box, self.rc2)
        self.i = torch.as_tensor(hl["i"])
        self.j = torch.as_tensor(hl["j"])
        self.rebuilds += 1

    def update_coordinates(self, xn):
        """reader.py:136-163 (skin/2 trigger)."""
        if self.last is not None:
            disp = self.box.minimum_image(xn - self.last)
            if torch.max(torch.norm(disp, dim=1)) > self.skin_half:
                self.last = xn.clone()
                self.x = xn
                self._rebuild()
                return
        else:
            self.last = xn.clone()
            self.x = xn
            self._rebuild()
            return
        self.x = xn

    def load_step(self, **loader):
        """UniaxialTensileLoader.step (loading.py:41-80): box and coordinates,
        update_coordinates, last_positions reset; returns the axis strain."""
        L0 = float(torch.linalg.norm(self.box.H[loader.get("axis", 0)]))
        xn = uniaxial_box_step(self.box, self.x, self.integ.dt, **loader)
        self.update_coordinates(xn.to(self.dtype))
        self.last = self.x.clone()
        return float(torch.linalg.norm(self.box.H[loader.get("axis", 0)])) / L0

    def step(self):
        if self.F is None:
            self.F = self.force_fn(self.x, self.i, self.j)["forces"].to(self.dtype)
        xn, vh = self.integ.first_half(self.x, self.v, self.F)
        self.update_coordinates(xn)
        out = self.force_fn(self.x, self.i, self.j)
        self.F = out["forces"].to(self.dtype)
        xi = self.noise_fn(self.step_index) if self.integ.langevin else None
        self.v, ke, T = self.integ.second_half(vh, self.F, None if xi is None else torch.as_tensor(xi))
        res = dict(energy=out["energy"], kinetic_energy=ke, temperature=T,
                   virial=out["virial"], virial_tensor=out["virial_tensor"])
        if self.barostat is not None:
            m = self.integ.atom_mass[:, :1]
            K_t = torch.einsum("ni,nj->ij", m * self.v, self.v)
            if self.barostat.get("kind") == "aniso":
                kw = {k: v for k, v in self.barostat.items() if k != "kind"}
                xn, self.v, P, self.eta_dot = aniso_npt(self.box, self.x, self.v, self.eta_dot, self.integ.dt, K_t,
                                                        out["virial_tensor"], **kw)
                self.update_coordinates(xn.to(self.dtype))
            else:
                self.x, self.v, P, mu = berendsen(self.box, self.x, self.v, self.integ.dt, K_t,
                                                  out["virial_tensor"], **self.barostat)
            self.last = self.x.clone()
            res["pressure"] = P
        self.step_index += 1
        return res
