"""Checkpoint and restart with the interface and file layout of io_utils/restart.py:32-149.

``save_checkpoint(model, step, path)`` writes a ``torch.save`` dict with the
reference's keys -- step, coordinates, velocities (original atom order, the
molecular's dtype), box_H, rng_cpu, rng_cuda, force_cache, energy_cache,
virial_cache -- so the reference's ``load_checkpoint`` can read it, plus the
engine's Philox step counter (``philox_step``), with which the Langevin noise
of the resumed run continues exactly (the noise is keyed by seed, original
atom index and step).  ``load_checkpoint(model, path)`` reads either
layout (tensors only: ``weights_only=True``; the box from ``box_H``, or from
``box_length`` as a cubic box when the reference wrote that key instead),
reloads positions, velocities and box into the device state (cell sort and list build), restores the RNG
states and the step counter, and returns the next step.  The forces of the
restored positions are recomputed on the first step (the reference restores
its force cache instead; both give the same forces).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import torch


def save_checkpoint(model, step: int, path: str | Path) -> None:
    mol = model.molecular
    eng = model.engine
    dt = mol.dtype
    ckpt = {
        "step": int(step),
        "coordinates": mol.coordinates.detach().to(dt).cpu(),
        "velocities": mol.atom_velocities.detach().to(dt).cpu(),
        "box_H": torch.as_tensor(eng.box_matrix(), dtype=torch.float64),
        "rng_cpu": torch.get_rng_state(),
        "rng_cuda": torch.cuda.get_rng_state(eng.device),
        "force_cache": eng.gather("f").to(dt).cpu(),
        "energy_cache": eng.potential_energy().to(dt).cpu(),
        "virial_cache": eng.red_out[2].to(dt).cpu(),
        "philox_step": eng.step_ctr.cpu().clone(),
    }
    torch.save(ckpt, path)


def load_checkpoint(model, path: str | Path) -> int:
    ckpt = torch.load(path, map_location="cpu", weights_only=True)
    mol = model.molecular
    eng = model.engine
    H = None
    if "box_H" in ckpt:
        H = np.asarray(ckpt["box_H"], np.float64)
    elif "box_length" in ckpt:
        # the reference's layout for a molecular without a Box object
        # (restart.py:55-58): a cubic box of that side
        H = np.diag([float(ckpt["box_length"])] * 3)
    if H is not None:
        eng.set_box(H)
        if hasattr(mol, "box"):
            mol.box.H = torch.as_tensor(H)
        if not eng.cells_valid(H):
            eng.regrid()
    mol.update_coordinates(ckpt["coordinates"].to(torch.float64))
    mol.atom_velocities = ckpt["velocities"].to(eng.device)
    if "philox_step" in ckpt:
        eng.step_ctr.copy_(ckpt["philox_step"].to(eng.device))
    if "rng_cpu" in ckpt:
        torch.set_rng_state(ckpt["rng_cpu"])
    if "rng_cuda" in ckpt:
        torch.cuda.set_rng_state(ckpt["rng_cuda"], eng.device)
    eng.forces_valid = False
    return int(ckpt["step"]) + 1


__all__ = ["save_checkpoint", "load_checkpoint"]
