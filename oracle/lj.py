"""Oracle Lennard-Jones forward (TEST INFRASTRUCTURE ONLY).

Restates core/force/lennard_jones_force.py:15-95 on CPU tensors in the dtype
of the coordinates (FP64 when the caller passes FP64, as the reference runs
under torch.set_default_dtype(torch.float64)).

  rij = min_image(pos_i - pos_j); r2 = clamp(sum rij^2, 1e-24)       (:35-36)
  sr = sigma/r; U = 4 eps (sr^12 - sr^6); F = 24 eps/r (2 sr^12 - sr^6) (:42-46)
  modes: quintic switch on [rs, rc] (:48-63), force shift (:65-75), raw (:77-79)
  mask r < rc (:82-84); f_i += F e_ij, f_j -= F e_ij (:87-90)
  energy = sum U; virial = sum F r (scalar, sign of sum f.r) (:92-93)
  virial_tensor = sum_e f_e (x) r_e (:94)
"""
from __future__ import annotations

import torch


def lj_forward(pos, i, j, eps, sigma, box, rc: float, mode: str = "raw", rs: float | None = None):
    pos = torch.as_tensor(pos)
    i = torch.as_tensor(i, dtype=torch.long)
    j = torch.as_tensor(j, dtype=torch.long)
    # Per-edge parameters keep their own dtype (the reference stores them as
    # float32, reader.py:193-207), so scalar products such as 24*eps and
    # sigma/rc are formed in float32 exactly as the reference does.
    eps = torch.as_tensor(eps)
    sigma = torch.as_tensor(sigma)
    rij = box.minimum_image(pos[i] - pos[j])
    r2 = (rij * rij).sum(dim=1).clamp_min(1e-24)
    r = torch.sqrt(r2)
    inv_r = 1.0 / r
    e_ij = rij * inv_r.unsqueeze(1)
    sr = sigma * inv_r
    sr6 = sr ** 6
    sr12 = sr6 ** 2
    U_raw = 4.0 * eps * (sr12 - sr6)
    F_raw = 24.0 * eps * inv_r * (2.0 * sr12 - sr6)
    if mode == "switch":
        x = ((r - rs) / (rc - rs)).clamp(0.0, 1.0)
        S_poly = 1.0 - 10.0 * x ** 3 + 15.0 * x ** 4 - 6.0 * x ** 5
        dS_poly = (-30.0 * x ** 2 + 60.0 * x ** 3 - 30.0 * x ** 4) / (rc - rs)
        in_mid = (r > rs) & (r < rc)
        S = torch.where(r <= rs, torch.ones_like(r), torch.where(in_mid, S_poly, torch.zeros_like(r)))
        dS = torch.where(in_mid, dS_poly, torch.zeros_like(r))
        U = U_raw * S
        F = F_raw * S - U_raw * dS
    elif mode == "fs":
        sr_rc = sigma / rc
        sr6_rc = sr_rc ** 6
        sr12_rc = sr6_rc ** 2
        U_rc = 4.0 * eps * (sr12_rc - sr6_rc)
        F_rc = 24.0 * eps * (1.0 / rc) * (2.0 * sr12_rc - sr6_rc)
        U = U_raw - U_rc + (r - rc) * F_rc
        F = F_raw - F_rc
    elif mode == "raw":
        U, F = U_raw, F_raw
    else:
        raise ValueError(mode)
    mask = (r < rc).to(pos.dtype)
    F = F * mask
    U = U * mask
    forces = torch.zeros_like(pos)
    fij = F.unsqueeze(1) * e_ij
    forces.index_add_(0, i, fij)
    forces.index_add_(0, j, -fij)
    return dict(energy=U.sum(), forces=forces, virial=(F * r * mask).sum(),
                virial_tensor=torch.einsum("ei,ej->ij", fij, rij))
