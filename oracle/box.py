"""Oracle box math (TEST INFRASTRUCTURE ONLY).

Restates core/box.py:39-153 on CPU tensors:
  * H rows are lattice vectors; H_inv = inv(H); orthogonal iff off-diagonal
    entries are all within 1e-8 of zero                          (box.py:54-57)
  * minimum_image: orthogonal -> r - d*round(r/d);
    triclinic -> s = r @ H_inv; s -= round(s); s @ H              (box.py:109-130)
  * wrap_positions                                                 (box.py:132-142)
  * scale (isotropic, Berendsen) and volume = |det H|              (box.py:78-80,145-148)
"""
from __future__ import annotations

import numpy as np
import torch


class OracleBox:
    def __init__(self, h):
        h = torch.as_tensor(np.asarray(h, dtype=np.float64))
        if h.numel() == 1:
            self.H = torch.diag(torch.full((3,), float(h.reshape(())), dtype=torch.float64))
        elif h.dim() == 1 and h.numel() == 3:
            self.H = torch.diag(h.double())
        elif tuple(h.shape) == (3, 3):
            self.H = h.double().clone()
        else:
            raise ValueError(f"h must be scalar, [3] or [3,3]; got {tuple(h.shape)}")
        self._refresh()

    def _refresh(self):
        self.H_inv = torch.linalg.inv(self.H)
        off = self.H - torch.diag(torch.diag(self.H))
        self.is_orthogonal = bool(torch.allclose(off, torch.zeros_like(off), atol=1e-8))

    @property
    def volume(self) -> float:
        return float(torch.det(self.H).abs())

    def minimum_image(self, rij: torch.Tensor) -> torch.Tensor:
        if self.is_orthogonal:
            d = torch.diag(self.H).to(rij)
            return rij - d * torch.round(rij / d)
        H_inv = self.H_inv.to(rij)
        H = self.H.to(rij)
        s = rij @ H_inv
        s = s - torch.round(s)
        return s @ H

    def wrap_positions(self, pos: torch.Tensor) -> torch.Tensor:
        if self.is_orthogonal:
            d = torch.diag(self.H).to(pos)
            return pos - torch.floor(pos / d) * d
        s = pos @ self.H_inv.to(pos)
        s = s - torch.floor(s)
        return s @ self.H.to(pos)

    def scale(self, factor: float):
        self.H = self.H * factor
        self._refresh()

    def perpendicular_widths(self) -> np.ndarray:
        """Distance between opposite faces along each fractional axis."""
        H = self.H.numpy()
        V = abs(np.linalg.det(H))
        a, b, c = H
        return np.array([V / np.linalg.norm(np.cross(b, c)),
                         V / np.linalg.norm(np.cross(c, a)),
                         V / np.linalg.norm(np.cross(a, b))])
