"""Oracle EAM: file parser, uniform tables and the two-pass forward.

TEST INFRASTRUCTURE ONLY.

Parser -- restates io_utils/eam_parser.py:23-210:
  * format detection: the first non-empty line after three comment lines; a
    multi-element header ("n El1 El2 ...", all-alphabetic names) selects the
    alloy/fs reader, anything else the single-element DYNAMO setfl reader
    (:30-48);
  * alloy/fs: grid line (n_rho d_rho n_r d_r cutoff), every following line
    flattened when it parses as floats -- element lines with a lattice token
    are skipped (:133-144); FS when the file name / header says eam.fs or the
    value count fits the FS layout (:146-152); per element F(rho) then
    (FS) one density block per neighbour element or (alloy) one block;
    then the pair blocks i<=j storing r*phi, divided by r (phi(0)=0) (:154-210);
  * every function is scipy CubicSpline(bc_type='not-a-knot') with its
    .derivative(1) -- scipy is the third-party algorithm the reference
    relies on and the same library is used here.

Tables -- restates core/force/eam_force_cu.py:334-415 (EAMForceCUDAExt):
  r grid linspace(0, cutoff, n_r=8192); rho grid linspace(knot0, knotN, n_rho=4096);
  splines (and derivative splines) evaluated by clamping to the knot range,
  searchsorted(right)-1, Horner.  ``dtype`` selects the evaluation precision:
  float32 reproduces the reference as-is, float64 is the FP64 restatement.

Forward -- restates eam_force_cu.py:437-579:
  cutoff filter r < rc on the Verlet half list; rho_i += f_{ti,tj}(r),
  rho_j += f_{tj,ti}(r); F(rho), F'(rho) by clamped lerp; pair energy
  sum phi_{ti,tj}(r); s = F'_i f'_{tj,ti}... exactly as :546-550;
  force_i += -s rij/(r+1e-8), force_j -= ...; virial = sum s r (note: the
  opposite sign of the LJ scalar convention); virial_tensor = sum f (x) rij.
"""
from __future__ import annotations

from collections import defaultdict

import numpy as np
import torch
from scipy.interpolate import CubicSpline


class ParsedEAM:
    pass


def parse_eam(path: str) -> ParsedEAM:
    with open(path) as fh:
        lines = fh.readlines()
    first = 0
    for k, line in enumerate(lines):
        if k > 2 and len(line.strip()) > 0:
            first = k
            break
    header = lines[first:]
    parts = header[0].split()
    if len(parts) > 1 and all(c.isalpha() for c in parts[1:]):
        return _parse_alloy(header, path)
    return _parse_setfl(lines)


def _new(path=None):
    p = ParsedEAM()
    p.filepath = path
    p.embedding_splines = {}
    p.embedding_deriv_splines = {}
    p.density_splines = {}
    p.density_deriv_splines = {}
    p.density_splines_by_pair = defaultdict(dict)
    p.density_deriv_splines_by_pair = defaultdict(dict)
    p.pair_potential_splines = defaultdict(dict)
    p.pair_potential_deriv_splines = defaultdict(dict)
    return p


def _parse_setfl(lines) -> ParsedEAM:
    """Single-element DYNAMO setfl (eam_parser.py:50-102)."""
    p = _new()
    start = 0
    for k in range(len(lines)):
        if len(lines[k].strip()) > 0 and lines[k][0] != "#":
            start = k
            break
    p.elements = [lines[start + 3].split()[3]]
    p.element_map = {p.elements[0]: 0}
    g = lines[start + 4].split()
    p.n_rho, p.d_rho, p.n_r, p.d_r, p.cutoff = int(g[0]), float(g[1]), int(g[2]), float(g[3]), float(g[4])
    data = [float(v) for line in lines[start + 5:] for v in line.split()]
    p.is_fs_format = False
    rho_v = np.arange(p.n_rho) * p.d_rho
    r_v = np.arange(p.n_r) * p.d_r
    s = CubicSpline(rho_v, np.array(data[:p.n_rho]), bc_type="not-a-knot")
    p.embedding_splines[0], p.embedding_deriv_splines[0] = s, s.derivative(1)
    s = CubicSpline(r_v, np.array(data[p.n_rho:p.n_rho + p.n_r]), bc_type="not-a-knot")
    p.density_splines[0], p.density_deriv_splines[0] = s, s.derivative(1)
    p.density_splines_by_pair[0][0] = s
    p.density_deriv_splines_by_pair[0][0] = p.density_deriv_splines[0]
    rphi = np.array(data[p.n_rho + p.n_r:p.n_rho + 2 * p.n_r])
    phi = np.divide(rphi, r_v, out=np.zeros_like(rphi), where=r_v != 0)
    s = CubicSpline(r_v, phi, bc_type="not-a-knot")
    p.pair_potential_splines[0][0], p.pair_potential_deriv_splines[0][0] = s, s.derivative(1)
    return p


def _parse_alloy(lines, path) -> ParsedEAM:
    """Multi-element eam/alloy or eam/fs (eam_parser.py:104-210)."""
    p = _new(path)
    h = lines[0].split()
    ne = int(h[0])
    p.elements = h[1:]
    p.element_map = {name: k for k, name in enumerate(p.elements)}
    g = lines[1].split()
    p.n_rho, p.d_rho, p.n_r, p.d_r, p.cutoff = int(g[0]), float(g[1]), int(g[2]), float(g[3]), float(g[4])
    data = []
    for line in lines[2:]:
        line = line.strip()
        if line:
            try:
                values = [float(v) for v in line.split()]   # all-or-nothing per line
            except ValueError:
                continue
            data.extend(values)
    exp_alloy = ne * (p.n_rho + p.n_r) + (ne * (ne + 1) // 2) * p.n_r
    exp_fs = ne * (p.n_rho + ne * p.n_r) + (ne * (ne + 1) // 2) * p.n_r
    p.is_fs_format = (str(path).lower().endswith(".eam.fs")
                      or any("eam.fs" in line.lower() for line in lines[:3])
                      or (len(data) >= exp_fs and len(data) - exp_alloy >= ne * (ne - 1) * p.n_r))
    ptr = 0
    rho_v = np.arange(p.n_rho) * p.d_rho
    r_v = np.arange(p.n_r) * p.d_r
    for beta in range(ne):
        if ptr + p.n_rho > len(data):
            raise ValueError("embedding block truncated")
        s = CubicSpline(rho_v, np.array(data[ptr:ptr + p.n_rho]), bc_type="not-a-knot")
        ptr += p.n_rho
        p.embedding_splines[beta], p.embedding_deriv_splines[beta] = s, s.derivative(1)
        if p.is_fs_format:
            for alpha in range(ne):
                if ptr + p.n_r > len(data):
                    raise ValueError("FS density block truncated")
                s = CubicSpline(r_v, np.array(data[ptr:ptr + p.n_r]), bc_type="not-a-knot")
                ptr += p.n_r
                p.density_splines_by_pair[alpha][beta] = s
                p.density_deriv_splines_by_pair[alpha][beta] = s.derivative(1)
            p.density_splines[beta] = p.density_splines_by_pair[beta][beta]
            p.density_deriv_splines[beta] = p.density_deriv_splines_by_pair[beta][beta]
        else:
            if ptr + p.n_r > len(data):
                raise ValueError("density block truncated")
            s = CubicSpline(r_v, np.array(data[ptr:ptr + p.n_r]), bc_type="not-a-knot")
            ptr += p.n_r
            p.density_splines[beta], p.density_deriv_splines[beta] = s, s.derivative(1)
            for alpha in range(ne):
                p.density_splines_by_pair[alpha][beta] = s
                p.density_deriv_splines_by_pair[alpha][beta] = s.derivative(1)
    for a in range(ne):
        for b in range(a, ne):
            rphi = np.array(data[ptr:ptr + p.n_r])
            ptr += p.n_r
            phi = np.divide(rphi, r_v, out=np.zeros_like(rphi), where=r_v != 0)
            s = CubicSpline(r_v, phi, bc_type="not-a-knot")
            p.pair_potential_splines[a][b], p.pair_potential_deriv_splines[a][b] = s, s.derivative(1)
            if a != b:
                p.pair_potential_splines[b][a] = s
                p.pair_potential_deriv_splines[b][a] = p.pair_potential_deriv_splines[a][b]
    return p


def spline_eval(spline, x: torch.Tensor, dtype=torch.float64) -> torch.Tensor:
    """eam_force_cu.py:397-415: clamp to knots, searchsorted(right)-1, Horner."""
    knots = torch.from_numpy(spline.x).to(dtype)
    c = torch.from_numpy(spline.c).to(dtype)
    x = torch.clamp(x.to(dtype), knots[0], knots[-1])
    idx = torch.searchsorted(knots, x, right=True) - 1
    idx = torch.clamp(idx, 0, len(knots) - 2)
    dx = x - knots[idx]
    if c.shape[0] == 4:
        return c[3, idx] + dx * (c[2, idx] + dx * (c[1, idx] + dx * c[0, idx]))
    if c.shape[0] == 3:
        return c[2, idx] + dx * (c[1, idx] + dx * c[0, idx])
    if c.shape[0] == 2:
        return c[1, idx] + dx * c[0, idx]
    raise RuntimeError("unsupported spline order")


class EAMTables:
    """Uniform lookup tables (eam_force_cu.py:334-396) in a chosen precision."""

    def __init__(self, parsed: ParsedEAM, n_r: int = 8192, n_rho: int = 4096, dtype=torch.float64):
        E = len(parsed.elements)
        self.E, self.n_r, self.n_rho, self.dtype = E, n_r, n_rho, dtype
        self.cutoff = float(parsed.cutoff)
        self.r_max = self.cutoff
        self.dr = self.r_max / (n_r - 1)
        self.inv_dr = 1.0 / self.dr
        r_grid = torch.linspace(0.0, self.r_max, n_r, dtype=dtype)
        self.density = torch.stack([torch.stack([spline_eval(parsed.density_splines_by_pair[h][n], r_grid, dtype)
                                                 for n in range(E)]) for h in range(E)])
        self.density_deriv = torch.stack([torch.stack([spline_eval(parsed.density_deriv_splines_by_pair[h][n], r_grid, dtype)
                                                       for n in range(E)]) for h in range(E)])
        zero = torch.zeros_like(r_grid)
        self.pair = torch.stack([torch.stack([spline_eval(parsed.pair_potential_splines[a][b], r_grid, dtype)
                                              if b in parsed.pair_potential_splines[a] else zero
                                              for b in range(E)]) for a in range(E)])
        self.pair_deriv = torch.stack([torch.stack([spline_eval(parsed.pair_potential_deriv_splines[a][b], r_grid, dtype)
                                                    if b in parsed.pair_potential_deriv_splines[a] else zero
                                                    for b in range(E)]) for a in range(E)])
        self.rho_min, self.drho, self.inv_drho = [], [], []
        emb, emb_d = [], []
        for t in range(E):
            x = torch.from_numpy(parsed.embedding_splines[t].x).to(dtype)
            lo, hi = float(x[0]), float(x[-1])
            d = (hi - lo) / (n_rho - 1)
            grid = torch.linspace(lo, hi, n_rho, dtype=dtype)
            emb.append(spline_eval(parsed.embedding_splines[t], grid, dtype))
            emb_d.append(spline_eval(parsed.embedding_deriv_splines[t], grid, dtype))
            self.rho_min.append(lo)
            self.drho.append(d)
            self.inv_drho.append(1.0 / d)
        self.embed = torch.stack(emb)
        self.embed_deriv = torch.stack(emb_d)

    def interp_r(self, r, table):
        """eam_force_cu.py:437-446."""
        rc = torch.clamp(r, 0.0, self.r_max * (1 - 1e-7))
        idx_f = rc * self.inv_dr
        idx = idx_f.long()
        frac = idx_f - idx
        nxt = torch.clamp(idx + 1, max=self.n_r - 1)
        v0 = table[..., idx]
        v1 = table[..., nxt]
        return v0 + frac * (v1 - v0)

    def interp_rho(self, rho, t: int, deriv: bool = False):
        """eam_force_cu.py:448-459."""
        lo, d, inv = self.rho_min[t], self.drho[t], self.inv_drho[t]
        n = self.n_rho
        rc = torch.clamp(rho, lo, lo + d * (n - 1) * (1 - 1e-7))
        idx_f = (rc - lo) * inv
        idx = idx_f.long()
        frac = idx_f - idx
        nxt = torch.clamp(idx + 1, max=n - 1)
        tab = self.embed_deriv[t] if deriv else self.embed[t]
        v0 = tab[idx]
        v1 = tab[nxt]
        return v0 + frac * (v1 - v0)


def eam_forward(coords, i, j, types, box, tables: EAMTables, edge_attr=None):
    """Two-pass EAM on a half list (eam_force_cu.py:461-579) in ``tables.dtype``.

    ``coords`` may be FP32 or FP64; pair arithmetic runs in ``tables.dtype``
    (the reference casts distances and rij to FP32, :484,493).
    """
    dt = tables.dtype
    coords = torch.as_tensor(coords)
    row = torch.as_tensor(i, dtype=torch.long)
    col = torch.as_tensor(j, dtype=torch.long)
    types = torch.as_tensor(types, dtype=torch.long)
    N = coords.shape[0]
    if row.numel() == 0:
        z = torch.zeros((), dtype=coords.dtype)
        return dict(energy=z, forces=torch.zeros_like(coords), virial=z,
                    virial_tensor=torch.zeros(3, 3, dtype=coords.dtype), rho=torch.zeros(N, dtype=dt))
    if edge_attr is None:
        edge_attr = torch.norm(box.minimum_image(coords[row] - coords[col]), dim=1)
    d_all = torch.as_tensor(edge_attr)
    mask = d_all < tables.cutoff
    dist = d_all[mask].contiguous().to(dt)
    row_m, col_m = row[mask], col[mask]
    rij = box.minimum_image(coords[row_m] - coords[col_m]).contiguous().to(dt)
    rho = torch.zeros(N, dtype=dt)
    rt, ct = types[row_m], types[col_m]
    E = tables.E
    for h in range(E):
        for nb in range(E):
            m = (rt == h) & (ct == nb)
            if m.any():
                rho.scatter_add_(0, row_m[m], tables.interp_r(dist[m], tables.density[h, nb]))
            m = (ct == h) & (rt == nb)
            if m.any():
                rho.scatter_add_(0, col_m[m], tables.interp_r(dist[m], tables.density[h, nb]))
    emb = torch.zeros_like(rho)
    dF = torch.zeros_like(rho)
    for t in range(E):
        am = types == t
        if am.any():
            emb[am] = tables.interp_rho(rho[am], t, False)
            dF[am] = tables.interp_rho(rho[am], t, True)
    e_emb = emb.sum()
    pe = torch.zeros_like(dist)
    d_row = torch.zeros_like(dist)
    d_col = torch.zeros_like(dist)
    d_pair = torch.zeros_like(dist)
    for a in range(E):
        for b in range(E):
            sel = (rt == a) & (ct == b)
            if sel.any():
                rs = dist[sel]
                pe[sel] = tables.interp_r(rs, tables.pair[a, b])
                d_row[sel] = tables.interp_r(rs, tables.density_deriv[b, a])
                d_col[sel] = tables.interp_r(rs, tables.density_deriv[a, b])
                d_pair[sel] = tables.interp_r(rs, tables.pair_deriv[a, b])
    e_pair = pe.sum()
    s = dF[row_m] * d_col + dF[col_m] * d_row + d_pair
    fvec = -s.unsqueeze(1) * (rij / (dist.unsqueeze(1) + 1e-8))
    forces = torch.zeros((N, 3), dtype=dt)
    forces.scatter_add_(0, row_m.unsqueeze(1).expand_as(fvec), fvec)
    forces.scatter_add_(0, col_m.unsqueeze(1).expand_as(fvec), -fvec)
    return dict(energy=e_emb + e_pair, forces=forces,
                virial=(s * dist).sum(), virial_tensor=torch.einsum("ei,ej->ij", fvec, rij),
                embedding_energy=e_emb, pair_potential=e_pair, rho=rho, dF=dF)
