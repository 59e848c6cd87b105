"""Periodic box with the interface of core/box.py (rows of H are lattice vectors).

Host-side description of the cell used to configure the device kernels and
available to user code.  The hot path never calls these torch methods: the
kernels carry their own minimum image (fixed-point fractional displacements
for the FP32 pair kernels, the reference's exact op order for the FP64 and
neighbour-export kernels).
"""
from __future__ import annotations

import torch


class Box:
    def __init__(self, h, device=None):
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda" if torch.cuda.is_available() else "cpu")
        h_t = torch.as_tensor(h, dtype=torch.float64)
        if h_t.dim() == 0 or h_t.numel() == 1:
            L = float(h_t)
            self._H = torch.diag(torch.tensor([L, L, L], dtype=torch.float64, device=self.device))
        elif h_t.dim() == 1 and h_t.numel() == 3:
            self._H = torch.diag(h_t.to(self.device))
        elif tuple(h_t.shape) == (3, 3):
            self._H = h_t.to(self.device)
        else:
            raise ValueError(f"h must be a scalar, [3] or [3,3]; got shape {tuple(h_t.shape)}")
        self._refresh()

    def _refresh(self):
        self._H_inv = torch.linalg.inv(self._H)
        off = self._H - torch.diag(torch.diag(self._H))
        self._is_orthogonal = bool(torch.allclose(off, torch.zeros_like(off), atol=1e-8))

    @property
    def H(self) -> torch.Tensor:
        return self._H

    @H.setter
    def H(self, value):
        self._H = torch.as_tensor(value).double().to(self.device)
        self._refresh()

    @property
    def H_inv(self) -> torch.Tensor:
        return self._H_inv

    @property
    def is_orthogonal(self) -> bool:
        return self._is_orthogonal

    @property
    def volume(self) -> float:
        return float(torch.det(self._H).abs())

    @property
    def lengths(self) -> torch.Tensor:
        return torch.norm(self._H, dim=1)

    @property
    def diag(self) -> torch.Tensor:
        return torch.diag(self._H)

    @property
    def box_length(self) -> torch.Tensor:
        d = torch.diag(self._H)
        if not self._is_orthogonal or not torch.allclose(d, d[0].expand_as(d), rtol=1e-5):
            raise ValueError("box_length is defined for cubic boxes only; use box.diag or box.H")
        return d[0].to(torch.float32)

    @property
    def box_length_cpu(self) -> float:
        return float(self.box_length)

    def minimum_image(self, rij: torch.Tensor) -> torch.Tensor:
        if self._is_orthogonal:
            d = torch.diag(self._H).to(rij)
            return rij - d * torch.round(rij / d)
        s = rij @ self._H_inv.to(rij)
        s = s - torch.round(s)
        return s @ self._H.to(rij)

    def wrap_positions(self, pos: torch.Tensor) -> torch.Tensor:
        if self._is_orthogonal:
            d = torch.diag(self._H).to(pos)
            return pos - torch.floor(pos / d) * d
        s = pos @ self._H_inv.to(pos)
        return (s - torch.floor(s)) @ self._H.to(pos)

    def scale(self, factor: float):
        self._H = self._H * factor
        self._refresh()

    def scale_anisotropic(self, mu: torch.Tensor):
        self._H = mu.double().to(self.device) @ self._H
        self._refresh()

    def to(self, device) -> "Box":
        self.device = torch.device(device)
        self._H = self._H.to(self.device)
        self._H_inv = self._H_inv.to(self.device)
        return self

    def state_dict(self) -> dict:
        return {"H": self._H.cpu()}

    @classmethod
    def from_state_dict(cls, d: dict, device=None) -> "Box":
        return cls(d["H"], device=device)

    def __repr__(self) -> str:
        kind = "orthogonal" if self._is_orthogonal else "triclinic"
        return f"Box({kind}, H=\n{self._H.cpu().numpy()})"
