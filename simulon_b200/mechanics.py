"""Mechanics callers of the force path: uniaxial tensile loading
(core/mechanics/loading.py:6-81) and the spherical indenter backbone
(core/mechanics/indenter.py:7-68).

Loader:
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
from .forces import BackboneInterface, _force_outputs


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


class SphericalIndenterForce(BackboneInterface):
    """Repulsive sphere (indenter.py:7-68): for atoms with d = |x - c| < R,
    U = K/3 (R - d)^3 and F = K (R - d)^2 (x - c)/d.  On the device: added to
    the engine's forces, energy and virial after the force field's pass (as a
    further backbone of SumBackboneInterface), with its own energy, force on
    the indenter and contact count in ``out``.  The centre is device memory,
    so ``set_center`` between CUDA-graph replays takes effect.  Positions are
    the unwrapped ones, without periodic images (as the reference).  The
    engine's virial tensor is symmetric: the indenter's F (x) x enters it with
    its upper triangle."""

    # its force depends on the atom's own position only, so an EAM force pass
    # can add it in its per-atom epilogue (sim_eam_force_integrate_indenter)
    fusable_into_force_pass = True

    def __init__(self, molecular, radius: float, stiffness: float, center):
        super().__init__()
        self.molecular = molecular
        self.device = molecular.device
        self.radius = float(radius)
        self.stiffness = float(stiffness)
        c = torch.as_tensor(center, dtype=torch.float64).reshape(-1)
        if c.numel() != 3:
            raise ValueError("center must have three components")
        self._center = c.to(self.device).clone()
        self.out = torch.zeros(11, dtype=torch.float64, device=self.device)
        self._st = _lib.SimIndenter()
        self._st.center, self._st.out = _lib.ptr(self._center), _lib.ptr(self.out)
        self._st.radius, self._st.stiffness = self.radius, self.stiffness
        self._ref = ctypes.byref(self._st)
        self.force_precision = 0

    @property
    def center(self) -> torch.Tensor:
        return self._center

    def set_center(self, center) -> None:
        self._center.copy_(torch.as_tensor(center, dtype=torch.float64).reshape(3))

    @property
    def force_on_indenter(self) -> torch.Tensor:
        return self.out[1:4]

    @property
    def last_energy(self) -> torch.Tensor:
        return self.out[0]

    @property
    def contact_atoms(self) -> int:
        return int(self.out[4].item())

    def add_to_engine(self, force_precision: int = 0):
        eng = self.molecular.engine
        _lib.call("sim_indenter_add", eng.st_ref, self._ref, int(force_precision), eng.stream)

    def compute(self):
        """Alone (the only backbone): the engine's forces and sums are zeroed first."""
        eng = self.molecular.engine
        eng.f32.zero_()
        if eng.f64 is not None:
            eng.f64.zero_()
        eng.red_out.zero_()
        self.add_to_engine(self.force_precision)
        eng.forces_valid = True

    def forward(self):
        self.compute()
        return _force_outputs(self.molecular)
