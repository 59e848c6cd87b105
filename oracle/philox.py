"""Philox4x32-10 counter-based generator + Box-Muller (TEST INFRASTRUCTURE ONLY).

The published algorithm of Salmon, Moraes, Dror and Shaw, "Parallel random
numbers: as easy as 1, 2, 3" (SC'11): ten rounds of two 32x32->64 multiplies
with the Weyl key schedule.  The CUDA Langevin kernel draws its noise with the
same generator and the same counter layout, so the oracle can reproduce the
GPU's noise exactly (up to the last ulp of the float32 transcendentals).

Counter layout for Langevin noise of atom ``a`` (original, unsorted index) at
step ``s``:  ctr = (a, s & 0xffffffff, s >> 32, stream), key = (seed_lo, seed_hi).
Normals: u_k = (x_k + 0.5) * 2^-32 in float32 arithmetic, then
z0 = sqrt(-2 ln u0) cos(pi 2u1), z1 = sqrt(-2 ln u0) sin(pi 2u1),
z2 = sqrt(-2 ln u2) cos(pi 2u3) -- three normals per atom.  The
transcendentals are evaluated in float64 and rounded to float32 (the device
uses float32 logf/sincospif, accurate to about one ulp).
"""
from __future__ import annotations

import numpy as np

M0 = np.uint64(0xD2511F53)
M1 = np.uint64(0xCD9E8D57)
W0 = np.uint32(0x9E3779B9)
W1 = np.uint32(0xBB67AE85)
MASK = np.uint64(0xFFFFFFFF)


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    c0 = np.asarray(c0, np.uint32).astype(np.uint64)
    c1 = np.asarray(c1, np.uint32).astype(np.uint64)
    c2 = np.asarray(c2, np.uint32).astype(np.uint64)
    c3 = np.asarray(c3, np.uint32).astype(np.uint64)
    k0 = np.uint64(np.uint32(k0))
    k1 = np.uint64(np.uint32(k1))
    with np.errstate(over="ignore"):
        for _ in range(10):
            p0 = M0 * c0
            p1 = M1 * c2
            hi0, lo0 = p0 >> np.uint64(32), p0 & MASK
            hi1, lo1 = p1 >> np.uint64(32), p1 & MASK
            c0, c1, c2, c3 = (hi1 ^ c1 ^ k0) & MASK, lo1, (hi0 ^ c3 ^ k1) & MASK, lo0
            k0 = (k0 + np.uint64(W0)) & MASK
            k1 = (k1 + np.uint64(W1)) & MASK
    return [x.astype(np.uint32) for x in (c0, c1, c2, c3)]


def langevin_normals(n_atoms: int, step: int, seed: int, stream: int = 0, orig_index=None):
    """[n,3] float64 standard normals for each atom at ``step`` (float32 Box-Muller)."""
    a = np.arange(n_atoms, dtype=np.uint32) if orig_index is None else np.asarray(orig_index, np.uint32)
    s = np.uint64(step)
    x = philox4x32_10(a, np.full_like(a, np.uint32(s & MASK)), np.full_like(a, np.uint32(s >> np.uint64(32))),
                      np.full_like(a, np.uint32(stream)), seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF)
    f = np.float32
    u = [(xk.astype(np.float32) + f(0.5)) * f(2.0 ** -32) for xk in x]
    def lg(x):
        return np.log(x.astype(np.float64)).astype(np.float32)

    def cs(x, fn):
        return fn(np.pi * (f(2.0) * x).astype(np.float64)).astype(np.float32)
    r0 = np.sqrt(f(-2.0) * lg(u[0]))
    r1 = np.sqrt(f(-2.0) * lg(u[2]))
    z = np.stack([r0 * cs(u[1], np.cos), r0 * cs(u[1], np.sin), r1 * cs(u[3], np.cos)], 1)
    return z.astype(np.float64)
