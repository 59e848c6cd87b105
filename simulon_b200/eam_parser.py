"""EAM potential files -> splines -> FP32 uniform tables for the device kernels.

``EAMParser`` mirrors io_utils/eam_parser.py (same constructor, same
attributes: elements, element_map, n_rho, d_rho, n_r, d_r, cutoff,
embedding_splines, density_splines_by_pair, pair_potential_splines and their
derivative splines, is_fs_format).  Format handling follows eam_parser.py:23-210:
DYNAMO setfl for a single element, LAMMPS eam/alloy or eam/fs otherwise;
non-numeric lines (element lines such as "74 183.84 3.165 bcc") are skipped
whole; the pair blocks store r*phi(r); every function is a scipy
CubicSpline(bc_type='not-a-knot') with its first-derivative spline.

``EAMDeviceTables`` evaluates those splines on the uniform grids that
EAMForceCUDAExt uses (eam_force_cu.py:334-396: n_r = 8192 points on
[0, cutoff], n_rho = 4096 points on the embedding knot range), in FP64, and
uploads them as FP32.  Derivative tables come from the derivative splines
(not from differencing the value tables), as in the reference.
"""
from __future__ import annotations

from collections import defaultdict

import numpy as np
import torch
from scipy.interpolate import CubicSpline

from . import _lib
from .engine import DeviceStruct


def _spline(x, y):
    s = CubicSpline(x, y, bc_type="not-a-knot")
    return s, s.derivative(1)


class EAMParser:
    def __init__(self, filepath: str, device=None):
        self.filepath = str(filepath)
        self.device = device
        self.embedding_splines, self.embedding_deriv_splines = {}, {}
        self.density_splines, self.density_deriv_splines = {}, {}
        self.density_splines_by_pair = defaultdict(dict)
        self.density_deriv_splines_by_pair = defaultdict(dict)
        self.pair_potential_splines = defaultdict(dict)
        self.pair_potential_deriv_splines = defaultdict(dict)
        self._parse()

    def _parse(self):
        with open(self.filepath) as fh:
            lines = fh.readlines()
        start = 0
        for k, line in enumerate(lines):
            if k > 2 and line.strip():
                start = k
                break
        head = lines[start:]
        parts = head[0].split()
        if len(parts) > 1 and all(tok.isalpha() for tok in parts[1:]):
            self._read_multi(head)
        else:
            self._read_setfl(lines)

    def _grid(self, line):
        g = line.split()
        self.n_rho, self.d_rho = int(g[0]), float(g[1])
        self.n_r, self.d_r, self.cutoff = int(g[2]), float(g[3]), float(g[4])

    def _read_setfl(self, lines):
        first = next((k for k, l in enumerate(lines) if l.strip() and l[0] != "#"), 0)
        self.elements = [lines[first + 3].split()[3]]
        self.element_map = {self.elements[0]: 0}
        self._grid(lines[first + 4])
        vals = np.array([float(v) for line in lines[first + 5:] for v in line.split()])
        self.is_fs_format = False
        rho_k = np.arange(self.n_rho) * self.d_rho
        r_k = np.arange(self.n_r) * self.d_r
        F = vals[:self.n_rho]
        f = vals[self.n_rho:self.n_rho + self.n_r]
        rphi = vals[self.n_rho + self.n_r:self.n_rho + 2 * self.n_r]
        self.embedding_splines[0], self.embedding_deriv_splines[0] = _spline(rho_k, F)
        s, ds = _spline(r_k, f)
        self.density_splines[0], self.density_deriv_splines[0] = s, ds
        self.density_splines_by_pair[0][0], self.density_deriv_splines_by_pair[0][0] = s, ds
        phi = np.divide(rphi, r_k, out=np.zeros_like(rphi), where=r_k != 0)
        self.pair_potential_splines[0][0], self.pair_potential_deriv_splines[0][0] = _spline(r_k, phi)

    def _read_multi(self, lines):
        head = lines[0].split()
        ne = int(head[0])
        self.elements = head[1:]
        self.element_map = {name: k for k, name in enumerate(self.elements)}
        self._grid(lines[1])
        values = []
        for line in lines[2:]:
            toks = line.split()
            if not toks:
                continue
            try:
                row = [float(t) for t in toks]
            except ValueError:
                continue          # element header line ("74 183.84 3.165 bcc")
            values.extend(row)
        values = np.asarray(values)
        n_alloy = ne * (self.n_rho + self.n_r) + ne * (ne + 1) // 2 * self.n_r
        n_fs = ne * (self.n_rho + ne * self.n_r) + ne * (ne + 1) // 2 * self.n_r
        self.is_fs_format = (self.filepath.lower().endswith(".eam.fs")
                             or any("eam.fs" in l.lower() for l in lines[:3])
                             or (len(values) >= n_fs and len(values) - n_alloy >= ne * (ne - 1) * self.n_r))
        rho_k = np.arange(self.n_rho) * self.d_rho
        r_k = np.arange(self.n_r) * self.d_r
        pos = 0

        def take(n, what):
            nonlocal pos
            if pos + n > len(values):
                raise ValueError(f"{what}: need {n} values, {len(values) - pos} left")
            block = values[pos:pos + n]
            pos += n
            return block
        for b in range(ne):
            self.embedding_splines[b], self.embedding_deriv_splines[b] = _spline(rho_k, take(self.n_rho, "F(rho)"))
            if self.is_fs_format:
                for a in range(ne):
                    s, ds = _spline(r_k, take(self.n_r, "FS density"))
                    self.density_splines_by_pair[a][b], self.density_deriv_splines_by_pair[a][b] = s, ds
                self.density_splines[b] = self.density_splines_by_pair[b][b]
                self.density_deriv_splines[b] = self.density_deriv_splines_by_pair[b][b]
            else:
                s, ds = _spline(r_k, take(self.n_r, "density"))
                self.density_splines[b], self.density_deriv_splines[b] = s, ds
                for a in range(ne):
                    self.density_splines_by_pair[a][b], self.density_deriv_splines_by_pair[a][b] = s, ds
        for a in range(ne):
            for b in range(a, ne):
                rphi = take(self.n_r, "pair")
                phi = np.divide(rphi, r_k, out=np.zeros_like(rphi), where=r_k != 0)
                s, ds = _spline(r_k, phi)
                self.pair_potential_splines[a][b], self.pair_potential_deriv_splines[a][b] = s, ds
                if a != b:
                    self.pair_potential_splines[b][a], self.pair_potential_deriv_splines[b][a] = s, ds


def eval_spline(spline, x: np.ndarray) -> np.ndarray:
    """Piecewise-polynomial evaluation with the clamp/search rule of
    eam_force_cu.py:397-415, in FP64."""
    knots = spline.x
    c = spline.c
    x = np.clip(np.asarray(x, np.float64), knots[0], knots[-1])
    idx = np.clip(np.searchsorted(knots, x, side="right") - 1, 0, len(knots) - 2)
    dx = x - knots[idx]
    val = np.zeros_like(x)
    for k in range(c.shape[0]):
        val = val * dx + c[k, idx]
    return val


class EAMDeviceTables:
    """FP32 uniform tables on the device + the SimEAMTables struct."""

    def __init__(self, parser: EAMParser, device, n_r: int = 8192, n_rho: int = 4096):
        E = len(parser.elements)
        self.n_types, self.n_r, self.n_rho = E, int(n_r), int(n_rho)
        self.cutoff = float(parser.cutoff)
        self.r_max = self.cutoff
        self.dr = self.r_max / (n_r - 1)
        self.inv_dr = 1.0 / self.dr
        r = np.linspace(0.0, self.r_max, n_r)

        def grid(table):
            return np.stack([np.stack([eval_spline(table[h][n], r) for n in range(E)]) for h in range(E)])
        zero = np.zeros(n_r)

        def pair_grid(table):
            return np.stack([np.stack([eval_spline(table[a][b], r) if b in table[a] else zero
                                       for b in range(E)]) for a in range(E)])
        host = dict(density=grid(parser.density_splines_by_pair),
                    density_deriv=grid(parser.density_deriv_splines_by_pair),
                    pair=pair_grid(parser.pair_potential_splines),
                    pair_deriv=pair_grid(parser.pair_potential_deriv_splines))
        emb, emb_d, lo, inv, hi = [], [], [], [], []
        for t in range(E):
            knots = parser.embedding_splines[t].x
            a, b = float(knots[0]), float(knots[-1])
            d = (b - a) / (n_rho - 1)
            g = np.linspace(a, b, n_rho)
            emb.append(eval_spline(parser.embedding_splines[t], g))
            emb_d.append(eval_spline(parser.embedding_deriv_splines[t], g))
            lo.append(a)
            inv.append(1.0 / d)
            hi.append(a + d * (n_rho - 1) * (1 - 1e-7))
        host["embed"] = np.stack(emb)
        host["embed_deriv"] = np.stack(emb_d)
        self.host64 = host
        self.rho_min64, self.inv_drho64, self.rho_hi64 = lo, inv, hi
        to = dict(device=device, dtype=torch.float32)
        self.tensors = {k: torch.as_tensor(v.astype(np.float32)).contiguous().to(device) for k, v in host.items()}
        self.tensors["rho_min"] = torch.tensor(lo, **to)
        self.tensors["inv_drho"] = torch.tensor(inv, **to)
        self.tensors["rho_clamp_hi"] = torch.tensor(hi, **to)

        def vd(*tabs):
            # value and forward difference, interleaved: (..., n_r, 2*len(tabs))
            vals = [t.astype(np.float32) for t in tabs]
            diffs = [np.concatenate([v[..., 1:] - v[..., :-1], np.zeros_like(v[..., :1])], -1) for v in vals]
            return np.ascontiguousarray(np.stack(vals + diffs, -1))
        self.tensors["dens_vd"] = torch.as_tensor(vd(host["density"])).to(device)
        self.tensors["deriv_vd"] = torch.as_tensor(vd(host["density_deriv"], host["pair_deriv"])).to(device)
        self.tensors["pair_vd"] = torch.as_tensor(vd(host["pair"])).to(device)
        s = _lib.SimEAMTables()
        for k in ("density", "density_deriv", "pair", "pair_deriv", "embed", "embed_deriv", "rho_min",
                  "inv_drho", "rho_clamp_hi", "dens_vd", "deriv_vd", "pair_vd"):
            setattr(s, k, _lib.ptr(self.tensors[k]))
        s.n_types, s.n_r, s.n_rho = E, self.n_r, self.n_rho
        s.cutoff = self.cutoff
        s.inv_dr = self.inv_dr
        s.r_clamp_hi = self.r_max * (1 - 1e-7)
        self.dev = DeviceStruct(s, list(self.tensors.values()))
        self.ref = self.dev.ref
