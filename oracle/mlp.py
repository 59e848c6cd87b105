"""CPU restatement of the descriptor-MLP EAM surrogate (test infrastructure).

The surrogate has no counterpart in the reference (which has no learned
potential on this path), so this module is the definition the CUDA kernels
are checked against; its parity with the reference is unpinned by nature.

Per atom i, with d_ij = x_j - x_i under the minimum image, r = |d_ij| and the
cosine cutoff fc(r) = (cos(pi r / rc) + 1) / 2 for r < rc (rc = 4.4 A):

* 8 radial terms  G_k = sum_j exp(-eta (r_ij - R_k)^2) fc(r_ij),
  eta = 4 A^-2, R_k = 2.0 + 2.4 k / 7;
* 8 angular terms G_(zeta,lam) = 2^(1-zeta) sum_{j<k} (1 + lam cos t_jik)^zeta
  exp(-eta_a (r_ij^2 + r_ik^2)) fc(r_ij) fc(r_ik), zeta in (1, 2, 4, 8),
  lam in (+1, -1), eta_a = 0.01 A^-2; ordered (zeta=1,+1), (1,-1), (2,+1), ...

Network: per-atom energy E_i = w3 . silu(W2^T silu(W1^T g_i + b1) + b2) + b3
with g_i = (G_i - mu) / sigma; E = sum_i E_i; forces = -dE/dx (autograd here).
"""
from __future__ import annotations

import math

import numpy as np
import torch

RC = 4.4
ETA_R = 4.0
R_S = tuple(2.0 + 2.4 * k / 7.0 for k in range(8))
ETA_A = 0.01
ZETAS = (1, 2, 4, 8)
N_DESC = 16
H = 64


def _fc(r):
    return 0.5 * (torch.cos(math.pi * r / RC) + 1.0) * (r < RC)


def descriptors(x, box, pairs_i, pairs_j):
    """G [N,16] in FP64 from positions x [N,3] (torch, may require grad) and a
    full pair list (both directions) within the list cutoff."""
    x = x if torch.is_tensor(x) else torch.tensor(x, dtype=torch.float64)
    N = x.shape[0]
    i = torch.as_tensor(pairs_i, dtype=torch.long)
    j = torch.as_tensor(pairs_j, dtype=torch.long)
    d = box.minimum_image(x[j] - x[i])
    r = torch.linalg.norm(d, dim=1)
    keep = r < RC
    i, j, d, r = i[keep], j[keep], d[keep], r[keep]
    fc = _fc(r)
    G = []
    for Rk in R_S:
        G.append(torch.zeros(N, dtype=x.dtype).index_add(0, i, torch.exp(-ETA_R * (r - Rk) ** 2) * fc))
    # angular: all ordered pairs (j, k) of neighbours of the same centre with j < k (by slot in the pair list)
    order = torch.argsort(i, stable=True)
    i, d, r, fc = i[order], d[order], r[order], fc[order]
    counts = torch.bincount(i, minlength=N)
    starts = torch.cumsum(counts, 0) - counts
    ci, a_idx, b_idx = [], [], []
    for c in range(N):
        s, n = int(starts[c]), int(counts[c])
        if n < 2:
            continue
        aa, bb = torch.triu_indices(n, n, offset=1)
        ci.append(torch.full((aa.numel(),), c, dtype=torch.long))
        a_idx.append(aa + s)
        b_idx.append(bb + s)
    if ci:
        ci, a_idx, b_idx = torch.cat(ci), torch.cat(a_idx), torch.cat(b_idx)
        cos = (d[a_idx] * d[b_idx]).sum(1) / (r[a_idx] * r[b_idx])
        rad = torch.exp(-ETA_A * (r[a_idx] ** 2 + r[b_idx] ** 2)) * fc[a_idx] * fc[b_idx]
    for z in ZETAS:
        for lam in (1.0, -1.0):
            if len(ci) if isinstance(ci, list) else ci.numel():
                val = 2.0 ** (1 - z) * (1.0 + lam * cos) ** z * rad
                G.append(torch.zeros(N, dtype=x.dtype).index_add(0, ci, val))
            else:
                G.append(torch.zeros(N, dtype=x.dtype))
    return torch.stack(G, 1)


def silu(z):
    return z * torch.sigmoid(z)


def atom_energies(G, net):
    """net: dict of torch tensors W1 [16,64], b1 [64], W2 [64,64], b2 [64],
    w3 [64], b3 [], mu [16], sigma [16]."""
    g = (G - net["mu"]) / net["sigma"]
    h1 = silu(g @ net["W1"] + net["b1"])
    h2 = silu(h1 @ net["W2"] + net["b2"])
    return h2 @ net["w3"] + net["b3"]


def energy_forces(x, box, pairs_i, pairs_j, net):
    """(E_i [N], forces [N,3]) in FP64 with forces = -dE/dx by autograd."""
    xt = torch.tensor(np.asarray(x), dtype=torch.float64, requires_grad=True)
    G = descriptors(xt, box, pairs_i, pairs_j)
    e = atom_energies(G, {k: torch.as_tensor(v, dtype=torch.float64) for k, v in net.items()})
    (grad,) = torch.autograd.grad(e.sum(), xt)
    return e.detach(), -grad.detach(), G.detach()


def eam_atom_energies(coords, i, j, types, box, tables):
    """Per-atom EAM energies E_i = F(rho_i) + 1/2 sum_j phi(r_ij) on a half
    list, the decomposition the surrogate is trained on."""
    coords = torch.as_tensor(coords, dtype=torch.float64)
    N = coords.shape[0]
    row = torch.as_tensor(i, dtype=torch.long)
    col = torch.as_tensor(j, dtype=torch.long)
    dist = torch.linalg.norm(box.minimum_image(coords[row] - coords[col]), dim=1)
    m = dist < tables.cutoff
    row, col, dist = row[m], col[m], dist[m].to(tables.dtype)
    dens = tables.interp_r(dist, tables.density[0, 0])
    rho = torch.zeros(N, dtype=tables.dtype).index_add(0, row, dens).index_add(0, col, dens)
    F = tables.interp_rho(rho, 0, False)
    phi = tables.interp_r(dist, tables.pair[0, 0])
    half = torch.zeros(N, dtype=tables.dtype).index_add(0, row, 0.5 * phi).index_add(0, col, 0.5 * phi)
    return F + half


def random_net(seed: int = 0, mu=None, sigma=None):
    rng = np.random.default_rng(seed)
    net = dict(W1=rng.normal(0, 1 / math.sqrt(16), (16, H)), b1=rng.normal(0, 0.1, H),
               W2=rng.normal(0, 1 / math.sqrt(H), (H, H)), b2=rng.normal(0, 0.1, H),
               w3=rng.normal(0, 1 / math.sqrt(H), H), b3=np.array(-8.0),
               mu=np.zeros(16) if mu is None else np.asarray(mu), sigma=np.ones(16) if sigma is None else np.asarray(sigma))
    return {k: np.asarray(v, dtype=np.float64) for k, v in net.items()}
