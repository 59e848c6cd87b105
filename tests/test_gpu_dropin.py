"""GPU parity of the drop-in for the reference's native module ``simulon_cuda``
(cuda source/ops.cpp:47-53), called with the arguments the reference's own
wrappers pass it.

The golden files ``legacy_*`` were written by running the reference's
wrappers (core/force/eam_force_cu.py:461-579 with its extension branch,
core/force/lennard_jones_force_cu.py:16-118) against a recording stand-in for
the native module: each call's arguments as the wrapper formed them, and the
values the call must produce from the reference's PyTorch evaluation of the
same quantities (tests/golden/make_golden.py, group "legacy").  The EAM
tables are rebuilt here by the oracle and checked bit for bit against the
digests of the reference's own tables before use.

Tolerances (FP32 kernels with atomics, as the reference's):
  * rho after pass 1: 2e-6 relative per atom;
  * F'(rho) computed from the drop-in's rho as the wrapper does: 1e-5 relative;
  * pass-2 forces: 5e-5 eV/A per component (8e-5 with F'(rho) from the
    drop-in's own rho; |F| reaches 3 eV/A), and the reference's own
    acceptance (cuda_test/test_eam_cuda.py:71: |dF|_2 < 1e-2) far inside;
  * LJ energy 2e-6 relative, forces 1e-6 eV/A per component, against the
    reference's FP64 PyTorch LJ on the same in-cutoff edges;
  * neighbor_search_cuda: the pair set bit-exact against the reference's.
"""
import hashlib
import os
import sys

import numpy as np
import pytest
import torch

from oracle import eam as oeam
from oracle import inputs as oin

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
DEV = torch.device("cuda")


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


def digest(t):
    return hashlib.sha256(np.ascontiguousarray(t.detach().cpu().numpy().astype(np.float32)).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def sc():
    import simulon_b200
    simulon_b200._lib.load()
    return simulon_b200.install_simulon_cuda()


POTENTIALS = {"legacy_eam_w250_f32": oin.write_fs_w_setfl, "legacy_eam_wli250_f32": oin.write_fs_two_element_setfl}


@pytest.fixture(scope="module", params=sorted(POTENTIALS))
def eam_case(request, tmp_path_factory):
    name = request.param
    g = load(name)
    pot = POTENTIALS[name](str(tmp_path_factory.mktemp("pot") / (name + ".eam.fs")))
    t = oeam.EAMTables(oeam.parse_eam(pot), dtype=torch.float32)
    for key, tab in (("density_table", t.density), ("density_deriv_table", t.density_deriv),
                     ("pair_table", t.pair), ("pair_deriv_table", t.pair_deriv), ("embed_table", t.embed),
                     ("embed_deriv_table", t.embed_deriv)):
        assert digest(tab) == str(g[key]), f"{key}: oracle table differs from the reference's"
    tabs = {k: v.to(DEV) for k, v in (("density", t.density), ("density_deriv", t.density_deriv),
                                      ("pair", t.pair), ("pair_deriv", t.pair_deriv), ("embed", t.embed),
                                      ("embed_deriv", t.embed_deriv))}
    return name, g, tabs


def interp_rho(g, tabs, rho, types, deriv):
    """F(rho) / F'(rho) exactly as the wrapper forms them (eam_force_cu.py:448-459,518-526)."""
    out = torch.zeros_like(rho)
    for t in range(len(g["embed_n"])):
        m = types == t
        if not bool(m.any()):
            continue
        lo, d, n = float(g["embed_rho_min"][t]), float(g["embed_drho"][t]), int(g["embed_n"][t])
        r = torch.clamp(rho[m], lo, lo + d * (n - 1) * (1 - 1e-7))
        idx_f = (r - lo) * (1.0 / d)
        idx = idx_f.long()
        frac = idx_f - idx
        nxt = torch.clamp(idx + 1, max=n - 1)
        tab = (tabs["embed_deriv"] if deriv else tabs["embed"])[t]
        v0, v1 = tab[idx], tab[nxt]
        out[m] = v0 + frac * (v1 - v0)
    return out


def cuda(a):
    return torch.as_tensor(a).to(DEV)


def test_eam_density_and_force_pass_match_reference(sc, eam_case):
    name, g, tabs = eam_case
    types = cuda(g["types"])
    n = types.shape[0]
    assert tuple(g["s0_d_table_shape"]) == tuple(tabs["density"].shape)
    for s in range(int(g["evaluations"])):
        d = {k: cuda(g[f"s{s}_d_{k}"]) for k in ("distances", "row", "col")}
        rho = torch.zeros(n, device=DEV)
        sc.density_pass(d["distances"], d["row"], d["col"], types, tabs["density"], float(g[f"s{s}_d_inv_dr"]),
                        int(g[f"s{s}_d_n_r"]), rho)
        torch.cuda.synchronize()
        want = g[f"s{s}_rho"]
        got = rho.cpu().numpy()
        assert np.max(np.abs(got - want) / np.abs(want)) < 2e-6, (name, s)
        # F'(rho) from this rho as the wrapper forms it, against the one the wrapper passed
        dF = interp_rho(g, tabs, rho, types, deriv=True)
        assert np.max(np.abs(dF.cpu().numpy() - g[f"s{s}_f_dF"]) / np.abs(g[f"s{s}_f_dF"])) < 1e-5, (name, s)

        f = {k: cuda(g[f"s{s}_f_{k}"]) for k in ("distances", "dist_vec", "row", "col", "dF")}
        for dFin in (f["dF"], dF):
            forces = torch.zeros(n, 3, device=DEV)
            sc.force_pass(f["distances"], f["dist_vec"], f["row"], f["col"], types, tabs["density_deriv"],
                          tabs["pair_deriv"], dFin, float(g[f"s{s}_d_inv_dr"]), int(g[f"s{s}_d_n_r"]), forces)
            torch.cuda.synchronize()
            err = forces.cpu().numpy() - g[f"s{s}_forces"]
            assert np.max(np.abs(err)) < (5e-5 if dFin is f["dF"] else 8e-5), (name, s, float(np.max(np.abs(err))))
            assert np.linalg.norm(err) < 1e-2


def test_eam_calls_accumulate_into_caller_buffers(sc, eam_case):
    """density_pass / force_pass add to what the buffers hold (the wrapper zeroes them first)."""
    name, g, tabs = eam_case
    types = cuda(g["types"])
    n = types.shape[0]
    d = {k: cuda(g[f"s0_d_{k}"]) for k in ("distances", "row", "col")}
    rho = torch.full((n,), 1.5, device=DEV)
    sc.density_pass(d["distances"], d["row"], d["col"], types, tabs["density"], float(g["s0_d_inv_dr"]),
                    int(g["s0_d_n_r"]), rho)
    assert np.max(np.abs(rho.cpu().numpy() - 1.5 - g["s0_rho"]) / g["s0_rho"]) < 3e-6
    f = {k: cuda(g[f"s0_f_{k}"]) for k in ("distances", "dist_vec", "row", "col", "dF")}
    forces = torch.ones(n, 3, device=DEV)
    sc.force_pass(f["distances"], f["dist_vec"], f["row"], f["col"], types, tabs["density_deriv"],
                  tabs["pair_deriv"], f["dF"], float(g["s0_d_inv_dr"]), int(g["s0_d_n_r"]), forces)
    assert np.max(np.abs(forces.cpu().numpy() - 1.0 - g["s0_forces"])) < 6e-5


def test_eam_recorded_md_sequence_through_installed_module(sc, eam_case):
    """The module registered by install_simulon_cuda() replays the native calls
    of the reference's MD steps: the wrapper's choice of function names
    (eam_force_cu.py:422-430), then per force evaluation pass 1 into a zeroed
    rho, F'(rho) from that rho, pass 2 into zeroed forces."""
    name, g, tabs = eam_case
    import simulon_cuda
    assert simulon_cuda is sc
    dens_fn = "density_pass_cuda" if hasattr(simulon_cuda, "density_pass_cuda") else "density_pass"
    force_fn = "force_pass_cuda" if hasattr(simulon_cuda, "force_pass_cuda") else "force_pass"
    types = cuda(g["types"])
    n = types.shape[0]
    for s in range(int(g["evaluations"])):
        rho = torch.zeros(n, device=DEV)
        getattr(simulon_cuda, dens_fn)(cuda(g[f"s{s}_d_distances"]), cuda(g[f"s{s}_d_row"]), cuda(g[f"s{s}_d_col"]),
                                       types, tabs["density"], float(g[f"s{s}_d_inv_dr"]), int(g[f"s{s}_d_n_r"]), rho)
        dF = interp_rho(g, tabs, rho, types, deriv=True)
        forces = torch.zeros(n, 3, device=DEV)
        getattr(simulon_cuda, force_fn)(cuda(g[f"s{s}_f_distances"]), cuda(g[f"s{s}_f_dist_vec"]),
                                        cuda(g[f"s{s}_f_row"]), cuda(g[f"s{s}_f_col"]), types,
                                        tabs["density_deriv"], tabs["pair_deriv"], dF, float(g[f"s{s}_d_inv_dr"]),
                                        int(g[f"s{s}_d_n_r"]), forces)
        torch.cuda.synchronize()
        assert np.max(np.abs(forces.cpu().numpy() - g[f"s{s}_forces"])) < 8e-5, (name, s)
        # total energy as the wrapper then forms it (eam_force_cu.py:527-538):
        # sum F(rho) over atoms + sum phi(r) over the in-cutoff edges
        F = interp_rho(g, tabs, rho, types, deriv=False)
        r = cuda(g[f"s{s}_d_distances"])
        tr, tc = types[cuda(g[f"s{s}_d_row"])], types[cuda(g[f"s{s}_d_col"])]
        rc = torch.clamp(r, 0.0, float(g["r_max"]) * (1 - 1e-7))
        idx_f = rc * float(g[f"s{s}_d_inv_dr"])
        idx = idx_f.long()
        frac = idx_f - idx
        nxt = torch.clamp(idx + 1, max=int(g[f"s{s}_d_n_r"]) - 1)
        v0, v1 = tabs["pair"][tr, tc, idx], tabs["pair"][tr, tc, nxt]
        energy = float(F.sum() + (v0 + frac * (v1 - v0)).sum())
        e_ref = float(g[f"s{s}_energy"])
        assert abs(energy - e_ref) < 2e-6 * abs(e_ref), (name, s, energy, e_ref)


@pytest.mark.parametrize("mode", ["raw", "fs", "switch"])
def test_lj_energy_force_cuda_matches_reference(sc, mode):
    g = load(f"legacy_lj_arcl108_{mode}_f32")
    sc.configure_lj_smoothing(int(g["mode"]), float(g["rc"]), float(g["rs"]))
    energy, forces = sc.lj_energy_force_cuda(cuda(g["pos"]), cuda(g["edge_index"]), cuda(g["sigma"]),
                                             cuda(g["epsilon"]), float(g["box_length"]))
    torch.cuda.synchronize()
    assert energy.dtype == torch.float32 and energy.shape == (1,)
    assert forces.dtype == torch.float32 and forces.shape == tuple(g["forces"].shape)
    e_ref = float(g["energy"])
    assert abs(float(energy[0]) - e_ref) <= 2e-6 * abs(e_ref), (float(energy[0]), e_ref)
    assert np.max(np.abs(forces.cpu().numpy() - g["forces"])) < 1e-6
    sc.configure_lj_smoothing(0, 0.0, 0.0)


def test_lj_energy_force_cuda_empty_edges(sc):
    g = load("legacy_lj_arcl108_raw_f32")
    energy, forces = sc.lj_energy_force_cuda(cuda(g["pos"]), torch.zeros(2, 0, dtype=torch.int64, device=DEV),
                                             torch.zeros(0, device=DEV), torch.zeros(0, device=DEV),
                                             float(g["box_length"]))
    assert float(energy[0]) == 0.0 and float(forces.abs().max()) == 0.0


@pytest.mark.parametrize("name", ["nbr_w250_f32", "nbr_far3_f32"])
def test_neighbor_search_cuda_pair_set_matches_reference(sc, name):
    """The reference calls it with FP32 positions, float(cutoff + skin) and
    the cubic box length (gpu_kdtree.py:77-83), then keeps i < j and
    recomputes the distances (reader.py:477-484)."""
    g = load(name)
    pos = cuda(g["pos"]).float()
    rc = float(torch.tensor(float(g["cutoff"]), dtype=torch.float32) + torch.tensor(float(g["skin"]),
                                                                                     dtype=torch.float32))
    L = float(np.asarray(g["box"]).reshape(-1)[0])
    ei, dist = sc.neighbor_search_cuda(pos, rc, L)
    assert ei.dtype == torch.int64 and ei.shape[0] == 2 and dist.dtype == torch.float32
    keep = ei[0] < ei[1]
    assert bool(keep.all())
    assert np.array_equal(ei[0].cpu().numpy(), g["i"]) and np.array_equal(ei[1].cpu().numpy(), g["j"])
    if len(g["i"]):
        np.testing.assert_allclose(dist.cpu().numpy(), g["dist"], rtol=1e-6)


def test_installed_module_is_the_dropin(sc):
    import simulon_b200
    mod = simulon_b200.install_simulon_cuda()
    assert sys.modules["simulon_cuda"] is mod
    for fn in ("lj_energy_force_cuda", "neighbor_search_cuda", "density_pass", "force_pass",
               "configure_lj_smoothing", "density_pass_cuda", "force_pass_cuda"):
        assert callable(getattr(mod, fn))
    with pytest.raises(RuntimeError):
        mod.density_pass(torch.zeros(1), torch.zeros(1, dtype=torch.int64), torch.zeros(1, dtype=torch.int64),
                         torch.zeros(1, dtype=torch.int64), torch.zeros(1, 1, 8), 1.0, 8, torch.zeros(1))
