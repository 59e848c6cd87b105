"""Seeded synthetic inputs for the oracle, the tests and the benchmark.

TEST INFRASTRUCTURE (also used by bench.py to create its synthetic systems).

Systems follow the benchmark configurations of the reference project:

* FCC argon:  4 n^3 atoms, a = 5.26 A, cubic box of side n*a, Gaussian
  jitter (sigma 0.05 A), mass 39.948 u.
* BCC tungsten: 2 n^3 atoms, a = 3.165 A, mass 183.84 u.  The basis and the
  row-vector convention match io_utils/w_bcc.py:22-71 (orientation "100").
* Triclinic variant: box rows (L,0,0), (0.02 L, L, 0), (0,0,L) -- an xy tilt
  of 0.02; atoms are the BCC fractional coordinates mapped through H.
* The synthetic Finnis-Sinclair tungsten potential
  phi(r) = (r-c)^2 (c0 + c1 r + c2 r^2)  (r < c),  rho(r) = (r-d)^2  (r < d),
  F(rho) = -A sqrt(rho), tabulated in the LAMMPS eam/fs ("setfl") layout that
  io_utils/eam_parser.py:104-210 reads: 3 comment lines, "1 W", the grid
  line, an element line with a non-numeric lattice token (skipped by
  eam_parser.py:136-144), F(rho), rho(r), then r*phi(r) (eam_parser.py:200-201).

Velocities follow io_utils/reader.py:319-339 (Maxwell-Boltzmann in internal
units, centre-of-mass momentum removed) but draw from numpy's PCG64 so the
inputs are reproducible without torch.
"""
from __future__ import annotations

import numpy as np

# Synthetic Finnis-Sinclair W parameters (config of the EAM-W benchmark).
FS_W = dict(c=3.25, d=4.400224, A=1.896373,
            c0=47.1346499, c1=-33.7665655, c2=6.2541999)
W_MASS = 183.84
AR_MASS = 39.948
W_A = 3.165
AR_A = 5.26

KB_EV = 8.617333262e-5          # eV/K                     (reader.py:326)
MASS_CONV = 1.036427e-4         # amu*(A/ps)^2 -> eV       (reader.py:327)


def fcc_lattice(n: int, a: float = AR_A):
    """FCC n x n x n conventional cells -> (coords [4n^3,3] float64, L)."""
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.arange(n)
    cells = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    coords = (cells[:, None, :] + basis[None, :, :]).reshape(-1, 3) * a
    return coords.astype(np.float64), n * a


def bcc_lattice(n: int, a: float = W_A):
    """BCC n x n x n conventional cells -> (coords [2n^3,3] float64, L)."""
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0.5]])
    g = np.arange(n)
    cells = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    coords = (cells[:, None, :] + basis[None, :, :]).reshape(-1, 3) * a
    return coords.astype(np.float64), n * a


def triclinic_box(L: float, tilt: float = 0.02):
    """Rows = lattice vectors: (L,0,0), (tilt*L, L, 0), (0,0,L)."""
    return np.array([[L, 0.0, 0.0], [tilt * L, L, 0.0], [0.0, 0.0, L]])


def bcc_triclinic(n: int, a: float = W_A, tilt: float = 0.02):
    """BCC fractional sites mapped through a tilted box (row-vector convention)."""
    coords, L = bcc_lattice(n, a)
    H = triclinic_box(L, tilt)
    frac = coords / L
    return frac @ H, H


def jitter(coords, sigma: float, seed: int):
    rng = np.random.default_rng(seed)
    return coords + rng.normal(0.0, sigma, size=coords.shape)


def maxwell_boltzmann(masses_amu, temperature: float, seed: int):
    """v ~ N(0, kB T / m) per component, COM momentum removed (reader.py:319-339)."""
    rng = np.random.default_rng(seed)
    m = np.asarray(masses_amu, dtype=np.float64)[:, None] * MASS_CONV
    sigma = np.sqrt(KB_EV * temperature / m)
    v = rng.standard_normal((m.shape[0], 3)) * sigma
    p = (v * m).sum(0)
    return v - p / m.sum()


def fs_w_functions(r=None, rho=None, p=FS_W):
    """Closed forms of the synthetic FS-W potential (vectorised numpy)."""
    out = {}
    if r is not None:
        r = np.asarray(r, dtype=np.float64)
        out["phi"] = np.where(r < p["c"], (r - p["c"]) ** 2 * (p["c0"] + p["c1"] * r + p["c2"] * r * r), 0.0)
        out["rho"] = np.where(r < p["d"], (r - p["d"]) ** 2, 0.0)
    if rho is not None:
        rho = np.asarray(rho, dtype=np.float64)
        out["F"] = -p["A"] * np.sqrt(np.maximum(rho, 0.0))
    return out


def write_fs_w_setfl(path, n_rho: int = 5000, d_rho: float = 0.012,
                     n_r: int = 5000, d_r: float = 4.4 / 5000, cutoff: float = 4.4):
    """Write the synthetic FS-W potential in eam/fs layout; returns the path.

    Grid: rho_k = k d_rho (k < n_rho, so rho_max = 59.988, about twice the
    equilibrium density 31.18) and r_k = k d_r (k < n_r).  The pair block
    stores r*phi(r) as the eam/fs format requires.
    """
    rk = np.arange(n_r) * d_r
    rhok = np.arange(n_rho) * d_rho
    f = fs_w_functions(r=rk, rho=rhok)
    blocks = [f["F"], f["rho"], rk * f["phi"]]
    lines = ["synthetic Finnis-Sinclair tungsten (eam/fs layout)",
             "phi=(r-c)^2(c0+c1 r+c2 r^2), rho=(r-d)^2, F=-A sqrt(rho)",
             "c=3.25 d=4.400224 A=1.896373 c0=47.1346499 c1=-33.7665655 c2=6.2541999",
             "1 W",
             f"{n_rho} {d_rho!r} {n_r} {d_r!r} {cutoff!r}",
             f"74 {W_MASS} {W_A} bcc"]
    for blk in blocks:
        for i in range(0, len(blk), 5):
            lines.append(" ".join(f"{v:.16e}" for v in blk[i:i + 5]))
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    return str(path)


# Two-element Finnis-Sinclair variant (elements W and Li, the second a scaled
# copy of the first): F_b(rho) = -A_b sqrt(rho); the density that a neighbour
# of element a contributes to a host of element b is s[a][b] (r-d)^2, with an
# asymmetric s so that a swapped [host, neighbour] index shows; pair terms
# p_ab phi(r).  Used to check multi-element table indexing.
FS_2E = dict(elements=("W", "Li"), A=(1.896373, 1.70673), s=((1.0, 0.85), (0.7, 0.9)),
             p=((1.0, 0.9), (0.9, 0.8)))


def write_fs_two_element_setfl(path, n_rho: int = 5000, d_rho: float = 0.012,
                               n_r: int = 5000, d_r: float = 4.4 / 5000, cutoff: float = 4.4):
    """Write the two-element FS potential of FS_2E in eam/fs layout (per
    element b: F_b, then the density blocks for neighbour a = 0, 1; then the
    pair blocks (0,0), (0,1), (1,1) as r*phi); returns the path."""
    rk = np.arange(n_r) * d_r
    rhok = np.arange(n_rho) * d_rho
    f = fs_w_functions(r=rk)
    sq = np.sqrt(rhok)
    lines = ["synthetic two-element Finnis-Sinclair (eam/fs layout)",
             "scaled copies of phi=(r-c)^2(c0+c1 r+c2 r^2), rho=(r-d)^2, F=-A sqrt(rho)",
             "elements W, Li",
             "2 W Li",
             f"{n_rho} {d_rho!r} {n_r} {d_r!r} {cutoff!r}"]
    blocks = []
    for b, (el, mass) in enumerate(((FS_2E["elements"][0], W_MASS), (FS_2E["elements"][1], 6.94))):
        lines_b = [f"{74 if b == 0 else 3} {mass} {W_A} bcc"]
        data = [-FS_2E["A"][b] * sq] + [FS_2E["s"][a][b] * f["rho"] for a in range(2)]
        blocks.append((lines_b, data))
    for head, data in blocks:
        lines += head
        for blk in data:
            for i in range(0, len(blk), 5):
                lines.append(" ".join(f"{v:.16e}" for v in blk[i:i + 5]))
    for a in range(2):
        for b in range(a, 2):
            blk = FS_2E["p"][a][b] * rk * f["phi"]
            for i in range(0, len(blk), 5):
                lines.append(" ".join(f"{v:.16e}" for v in blk[i:i + 5]))
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    return str(path)


def write_xyz_symbols(path, coords, symbols):
    """XYZ file with one symbol per atom (round-trip precision)."""
    coords = np.asarray(coords, dtype=np.float64)
    with open(path, "w") as fh:
        fh.write(f"{coords.shape[0]}\nmixed synthetic\n")
        for s, (x, y, z) in zip(symbols, coords):
            fh.write(f"{s} {float(x)!r} {float(y)!r} {float(z)!r}\n")
    return str(path)


def perfect_bcc_known_answer(a: float = W_A, p=FS_W):
    """Analytic E/atom of the perfect BCC lattice for the synthetic FS-W form.

    First shell: 8 atoms at a*sqrt(3)/2; second: 6 at a; third: 12 at a*sqrt(2)
    (4.476 A, outside the 4.4 A cutoff).  Returns (rho, F(rho), half pair sum, E/atom).
    """
    r1, r2 = a * np.sqrt(3.0) / 2.0, a
    f = fs_w_functions(r=np.array([r1, r2]))
    rho = 8 * f["rho"][0] + 6 * f["rho"][1]
    F = -p["A"] * np.sqrt(rho)
    half_phi = 0.5 * (8 * f["phi"][0] + 6 * f["phi"][1])
    return float(rho), float(F), float(half_phi), float(F + half_phi)


def write_xyz(path, coords, symbol: str):
    """XYZ file with round-trip precision so a reader recovers the exact doubles."""
    coords = np.asarray(coords, dtype=np.float64)
    with open(path, "w") as fh:
        fh.write(f"{coords.shape[0]}\n{symbol} synthetic\n")
        for x, y, z in coords:
            fh.write(f"{symbol} {float(x)!r} {float(y)!r} {float(z)!r}\n")
    return str(path)
