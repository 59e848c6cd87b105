"""Uniaxial tensile loading with the interface of core/mechanics/loading.py:6-81.

The box update runs on the device in FP64 (``sim_box_scale``): H <- diag(s) H,
positions through fractional coordinates of the old box into the new one and
wrapped (box.py:132-142), posq refreshed, the skin test against the last
rebuild, and the reference's reset of last_positions.  ``step`` returns the
engineering strain of the loading axis as a Python float (it reads the
device box, which also holds a barostat's changes of the other axes).

Beyond the reference: the cell grid is rebuilt when the box shrinks below
rc + skin per cell (``MDEngine.regrid``), and the list is rebuilt whenever
the box has strained by more than a quarter of the skin over the list
cutoff since the last such rebuild (the skin test compares fractional
positions, which an affine box change leaves unchanged).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib


class UniaxialTensileLoader:
    def __init__(self, molecular, axis: int = 0, strain_rate: float = 1.0e-3, lateral_mode: str = "fixed",
                 poisson_ratio: float = 0.28, max_lateral_scale_step: float = 2.0e-3):
        self.molecular = molecular
        self.axis = int(axis)
        self.strain_rate = float(strain_rate)
        self.lateral_mode = str(lateral_mode).lower()
        self.poisson_ratio = float(poisson_ratio)
        self.max_lateral_scale_step = float(max_lateral_scale_step)
        if self.axis not in (0, 1, 2):
            raise ValueError(f"axis must be 0/1/2, got {axis}")
        if not hasattr(molecular, "engine"):
            raise NotImplementedError("UniaxialTensileLoader requires a device-resident molecular (engine)")
        if self.lateral_mode not in ("fixed", "poisson"):
            raise ValueError(f"unsupported lateral_mode={lateral_mode}")
        eng = molecular.engine
        H = eng.box_matrix()
        self.initial_lengths = torch.tensor(np.linalg.norm(H, axis=1), dtype=torch.float64)
        self.total_engineering_strain = 0.0
        self.work = torch.zeros(_lib.BOXSCALE_WORK, dtype=torch.float64, device=eng.device)
        self._H_list = H
        self.forced_rebuilds = 0
        self.regrids = 0

    def _scale_vector(self, dt: float) -> list:
        dstrain = self.strain_rate * float(dt)
        scale = [1.0, 1.0, 1.0]
        scale[self.axis] = 1.0 + dstrain
        if self.lateral_mode == "poisson":
            lat = max(1.0 - self.poisson_ratio * dstrain, 1.0 - self.max_lateral_scale_step)
            for ax in range(3):
                if ax != self.axis:
                    scale[ax] = lat
        return scale

    def step(self, dt: float) -> float:
        mol = self.molecular
        eng = mol.engine
        s = _lib.SimBoxScale()
        s.scale[:] = self._scale_vector(dt)
        s.vel_scale[:] = [1.0, 1.0, 1.0]
        s.reset_reference = 1
        _lib.call("sim_box_scale", eng.st_ref, ctypes.byref(s), _lib.ptr(self.work), eng.stream)
        H = eng.box_matrix()
        if not eng.cells_valid(H):
            eng.regrid()
            self.regrids += 1
            self._H_list = H
        else:
            dev = np.abs(np.linalg.solve(self._H_list.T, H.T).T - np.eye(3)).max()
            if dev * eng.x_rc > 0.25 * eng.skin:
                eng.rebuild(only_if_flagged=False)
                self.forced_rebuilds += 1
                self._H_list = H
        if hasattr(mol, "box"):
            mol.box.H = torch.as_tensor(H)
        lengths = np.linalg.norm(H, axis=1)
        self.total_engineering_strain = float(lengths[self.axis] / float(self.initial_lengths[self.axis]) - 1.0)
        return self.total_engineering_strain

    def current_lengths(self) -> torch.Tensor:
        return torch.tensor(np.linalg.norm(self.molecular.engine.box_matrix(), axis=1), dtype=torch.float64)
