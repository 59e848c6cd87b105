"""The surrogate's FP64 restatement on CPU: descriptors are invariant under
translation and periodic relabelling, and autograd forces agree with central
finite differences of the total energy (1e-6 relative)."""
import numpy as np
import torch

from oracle import inputs as oin
from oracle import mlp as omlp
from oracle import neighbor as onb
from oracle.box import OracleBox


def _pairs(x, H):
    hl = onb.half_list(x, OracleBox(H), 4.9 ** 2)
    return np.concatenate([hl["i"], hl["j"]]), np.concatenate([hl["j"], hl["i"]])


def test_descriptors_translation_invariant():
    x, L = oin.bcc_lattice(3)
    x = oin.jitter(x, 0.1, 1)
    H = np.diag([L] * 3)
    pi, pj = _pairs(x, H)
    G0 = omlp.descriptors(torch.tensor(x), OracleBox(H), pi, pj)
    G1 = omlp.descriptors(torch.tensor(x + np.array([1.3, -0.7, 2.2])), OracleBox(H), pi, pj)
    assert torch.allclose(G0, G1, rtol=1e-12, atol=1e-12)
    assert G0.shape == (len(x), 16) and torch.all(G0[:, :8] > 0)


def test_autograd_forces_match_finite_differences():
    x, L = oin.bcc_lattice(3)
    x = oin.jitter(x, 0.1, 2)
    H = np.diag([L] * 3)
    pi, pj = _pairs(x, H)
    G = omlp.descriptors(torch.tensor(x), OracleBox(H), pi, pj)
    net = omlp.random_net(0, mu=G.mean(0).numpy(), sigma=G.std(0).numpy())
    _, f, _ = omlp.energy_forces(x, OracleBox(H), pi, pj, net)
    h = 1e-5
    rng = np.random.default_rng(3)
    for a in rng.choice(len(x), 4, replace=False):
        for c in range(3):
            xp, xm = x.copy(), x.copy()
            xp[a, c] += h
            xm[a, c] -= h
            ep = omlp.energy_forces(xp, OracleBox(H), pi, pj, net)[0].sum()
            em = omlp.energy_forces(xm, OracleBox(H), pi, pj, net)[0].sum()
            fd = -(float(ep) - float(em)) / (2 * h)
            assert abs(fd - float(f[a, c])) <= 1e-6 * max(1.0, abs(fd)), (a, c, fd, float(f[a, c]))
