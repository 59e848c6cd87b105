"""Pin the CPU oracle against golden vectors produced by the reference itself.

The fixtures in tests/golden/ were written by tests/golden/make_golden.py,
which runs the unmodified reference (core/, io_utils/) on seeded inputs.
Tolerances:
  * neighbor pair sets: bit-exact (same (i, j) set, same order);
  * LJ FP64: 1e-12 relative (same arithmetic, scatter order may differ);
  * EAM: the oracle in float32-table mode against the FP32 reference at
    float32 round-off; the FP64 oracle against the FP32 reference at 2e-5;
  * MD trajectories: 1e-9 (FP64 LJ) / 1e-4 relative energies (FP32 EAM).
"""
import os

import numpy as np
import pytest
import torch

from oracle import eam as oeam
from oracle import inputs as oin
from oracle import neighbor as onb
from oracle.box import OracleBox
from oracle.integrator import OracleMD
from oracle.lj import lj_forward
from oracle.philox import langevin_normals, philox4x32_10

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


NBR_CASES = ["nbr_ar108_f64", "nbr_w250_f32", "nbr_wtri432_f32", "nbr_wtri432_f64",
             "nbr_gas300_orth_f32", "nbr_pair2_f64", "nbr_far3_f32"]


@pytest.mark.parametrize("name", NBR_CASES)
@pytest.mark.parametrize("mode", ["brute", "auto"])
def test_neighbor_pair_set_bit_exact(name, mode):
    g = load(name)
    box = OracleBox(g["box"])
    pos = g["pos"]
    rc2 = onb.rc2_like_reference(float(g["cutoff"]), float(g["skin"]), pos.dtype)
    hl = onb.half_list(pos, box, rc2, mode=mode)
    assert np.array_equal(hl["i"], g["i"]) and np.array_equal(hl["j"], g["j"])
    if len(g["i"]):
        d = onb.edge_distances(pos, hl["i"], hl["j"], box)
        np.testing.assert_allclose(d, g["dist"], rtol=1e-6 if pos.dtype == np.float32 else 1e-14)
        assert (hl["d2"] < rc2).all()


def test_cell_mode_equals_brute_force_large():
    x, L = oin.bcc_lattice(12)                     # 3456 atoms, 9 cells per axis
    x = oin.jitter(x, 0.08, 11).astype(np.float32)
    box = OracleBox(L)
    rc2 = onb.rc2_like_reference(4.4, 0.5, np.float32)
    a = onb.half_list(x, box, rc2, mode="brute")
    b = onb.half_list(x, box, rc2, mode="cell")
    assert np.array_equal(a["i"], b["i"]) and np.array_equal(a["j"], b["j"])
    assert np.array_equal(a["image"], b["image"]) and np.array_equal(a["d2"], b["d2"])


def test_cell_mode_equals_brute_force_triclinic():
    x, H = oin.bcc_triclinic(10)
    x = oin.jitter(x, 0.08, 12)
    box = OracleBox(H)
    rc2 = onb.rc2_like_reference(4.4, 0.5, np.float64)
    a = onb.half_list(x, box, rc2, mode="brute")
    b = onb.half_list(x, box, rc2, mode="cell")
    assert np.array_equal(a["i"], b["i"]) and np.array_equal(a["j"], b["j"])


@pytest.mark.parametrize("mode", ["raw", "fs", "switch"])
def test_lj_fp64_matches_reference(mode):
    g = load(f"lj_ar108_{mode}_f64")
    box = OracleBox(g["box"])
    out = lj_forward(torch.tensor(g["pos"]), g["i"], g["j"], g["eps"], g["sigma"], box,
                     float(g["rc"]), mode, float(g["rs"]))
    np.testing.assert_allclose(out["energy"].item(), g["energy"], rtol=1e-12)
    np.testing.assert_allclose(out["forces"].numpy(), g["forces"], rtol=1e-10, atol=1e-13)
    np.testing.assert_allclose(out["virial"].item(), g["virial"], rtol=1e-12)
    np.testing.assert_allclose(out["virial_tensor"].numpy(), g["virial_tensor"], rtol=1e-11, atol=1e-14)


@pytest.fixture(scope="module")
def fsw(tmp_path_factory):
    path = oin.write_fs_w_setfl(str(tmp_path_factory.mktemp("pot") / "W_synthetic.eam.fs"))
    return oeam.parse_eam(path)


def test_eam_tables_fp32_bit_exact(fsw):
    g = load("eam_w250_jitter_f32")
    t32 = oeam.EAMTables(fsw, dtype=torch.float32)
    for key, tab in (("density_table", t32.density[0, 0]), ("density_deriv_table", t32.density_deriv[0, 0]),
                     ("pair_table", t32.pair[0, 0]), ("pair_deriv_table", t32.pair_deriv[0, 0]),
                     ("embed_table", t32.embed[0]), ("embed_deriv_table", t32.embed_deriv[0])):
        assert np.array_equal(tab.numpy(), g[key]), key


@pytest.mark.parametrize("name", ["eam_w250_jitter_f32", "eam_w250_perfect_f32", "eam_wtri432_f32"])
def test_eam_oracle_matches_reference(fsw, name):
    g = load(name)
    box = OracleBox(g["box"])
    types = np.zeros(len(g["pos"]), np.int64)
    t32 = oeam.EAMTables(fsw, dtype=torch.float32)
    o32 = oeam.eam_forward(torch.tensor(g["pos"]), g["i"], g["j"], types, box, t32)
    np.testing.assert_allclose(o32["energy"].item(), g["energy"], rtol=2e-6)
    np.testing.assert_allclose(o32["forces"].numpy(), g["forces"], atol=5e-5)
    np.testing.assert_allclose(o32["virial_tensor"].numpy(), g["virial_tensor"], rtol=1e-4, atol=2e-2)
    t64 = oeam.EAMTables(fsw, dtype=torch.float64)
    o64 = oeam.eam_forward(torch.tensor(g["pos"]).double(), g["i"], g["j"], types, box, t64)
    np.testing.assert_allclose(o64["energy"].item(), g["energy"], rtol=2e-5)
    rmse = np.sqrt(((o64["forces"].numpy() - g["forces"]) ** 2).mean())
    assert rmse < 1e-4, rmse


def test_eam_perfect_lattice_known_answer(fsw):
    rho, F, half_phi, e_atom = oin.perfect_bcc_known_answer()
    assert abs(rho - 31.179650) < 1e-5 and abs(e_atom - (-8.900002)) < 1e-5
    g = load("eam_w250_perfect_f32")
    t64 = oeam.EAMTables(fsw, dtype=torch.float64)
    out = oeam.eam_forward(torch.tensor(g["pos"]).double(), g["i"], g["j"], np.zeros(250, np.int64),
                           OracleBox(g["box"]), t64)
    assert abs(out["energy"].item() / 250 - e_atom) < 2e-5
    assert float(g["energy"]) / 250 == pytest.approx(-8.9000010, abs=2e-6)
    # positions are float32-rounded lattice sites, so forces vanish only to ~1e-5
    assert np.abs(out["forces"].numpy()).max() < 2e-5


def test_philox_known_answer():
    # Random123 known-answer vector for philox4x32-10 with counter = key = 0.
    out = philox4x32_10(0, 0, 0, 0, 0, 0)
    assert [int(v) for v in out] == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    # and with all-ones counter/key
    m = 0xFFFFFFFF
    out = philox4x32_10(m, m, m, m, m, m)
    assert [int(v) for v in out] == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    z = langevin_normals(20000, 3, 77)
    assert abs(z.mean()) < 0.02 and abs(z.std() - 1) < 0.02


def _lj_force_fn(box, eps, sigma):
    def fn(x, i, j):
        # the reference keeps per-edge LJ parameters in float32 (reader.py:193-195)
        return lj_forward(x, i, j, np.full(len(i), eps, np.float32), np.full(len(i), sigma, np.float32),
                          box, 7.0, "raw")
    return fn


@pytest.mark.parametrize("ens", ["nve", "nvt"])
def test_md_lj_fp64_matches_reference(ens):
    g = load(f"md_ar108_{ens}_f64")
    box = OracleBox(float(g["box"]))
    eps, sigma = 0.0104, 3.405
    md = OracleMD(g["x0"], g["v0"], np.full(108, oin.AR_MASS), box, _lj_force_fn(box, eps, sigma),
                  cutoff=7.0, skin=0.5, dt=float(g["dt"]), ensemble=ens.upper(),
                  temperature=float(g["T"]), gamma=float(g["gamma"]),
                  noise_fn=lambda s: langevin_normals(108, s, int(g["noise_seed"])))
    e = [md.step() for _ in range(int(g["steps"]))]
    np.testing.assert_allclose([float(r["energy"]) for r in e], g["energy"], rtol=1e-9)
    np.testing.assert_allclose([float(r["kinetic_energy"]) for r in e], g["kinetic_energy"], rtol=1e-9)
    np.testing.assert_allclose(md.x.numpy(), g["x"], atol=1e-10)
    np.testing.assert_allclose(md.v.numpy(), g["v"], atol=1e-9)
    # the reference counts rebuilds from the first step on (the list built at
    # construction, reader.py:83, precedes its profile counter, reader.py:87)
    assert md.rebuilds - 1 == int(g["rebuilds"])


@pytest.mark.parametrize("ens", ["nve", "npt"])
def test_md_eam_fp32_matches_reference(fsw, ens):
    g = load(f"md_w250_{ens}_f32")
    box = OracleBox(float(g["box0"]))
    t32 = oeam.EAMTables(fsw, dtype=torch.float32)
    types = np.zeros(250, np.int64)

    def ff(x, i, j):
        return oeam.eam_forward(x, i, j, types, box, t32)
    baro = dict(P0=0.0, tau=float(g["tau_p"])) if ens == "npt" else None
    md = OracleMD(np.asarray(g["x0"], np.float32), np.asarray(g["v0"], np.float32), np.full(250, oin.W_MASS),
                  box, ff, cutoff=fsw.cutoff, skin=0.5, dt=float(g["dt"]),
                  ensemble="NPT" if ens == "npt" else "NVE", temperature=float(g["T"]), gamma=float(g["gamma"]),
                  dtype=torch.float32, noise_fn=lambda s: langevin_normals(250, s, int(g["noise_seed"])),
                  barostat=baro)
    e = [md.step() for _ in range(int(g["steps"]))]
    np.testing.assert_allclose([float(r["energy"]) for r in e], g["energy"], rtol=1e-5)
    np.testing.assert_allclose([float(r["kinetic_energy"]) for r in e], g["kinetic_energy"], rtol=1e-3)
    if ens == "npt":
        np.testing.assert_allclose([r["pressure"] for r in e], g["pressure"], rtol=1e-3, atol=50.0)
        np.testing.assert_allclose(box.H.numpy(), g["box"], rtol=1e-6)
    np.testing.assert_allclose(md.x.numpy(), g["x"], atol=1e-4)


@pytest.mark.parametrize("name", ["tensile", "aniso"])
def test_tensile_and_aniso_npt_match_reference(name):
    """UniaxialTensileLoader + AnisotropicNPTBarostat (lateral axes) and the
    barostat alone, LJ argon FP64: the oracle's restatement against the
    reference's own run (energies, axis pressures, box, strain rates, final
    positions and velocities)."""
    import json
    g = load(f"mech_ar108_{name}_f64")
    box = OracleBox(float(g["box0"]))
    load_kw = json.loads(str(g["load"]))
    baro_kw = json.loads(str(g["baro"]))
    baro = dict(kind="aniso", target_bar=baro_kw["target_pressure_bar"], control=tuple(baro_kw["control_axes"]),
                tau_p=0.2, gamma_p=2.0, kappa=3.2e-5, tol=25.0)
    md = OracleMD(g["x0"], g["v0"], np.full(108, oin.AR_MASS), box, _lj_force_fn(box, 0.0104, 3.405),
                  cutoff=7.0, skin=0.5, dt=float(g["dt"]), barostat=baro)
    E, P, H, eta = [], [], [], []
    for _ in range(int(g["steps"])):
        if load_kw:
            md.load_step(**load_kw)
        r = md.step()
        E.append(float(r["energy"]))
        P.append(r["pressure"].numpy())
        H.append(box.H.numpy().copy())
        eta.append(md.eta_dot.numpy().copy())
    np.testing.assert_allclose(E, g["energy"], rtol=1e-9)
    np.testing.assert_allclose(np.array(P), g["pressure"], rtol=1e-8, atol=1e-6)
    np.testing.assert_allclose(np.array(H), g["H"], rtol=1e-12)
    np.testing.assert_allclose(np.array(eta), g["eta_dot"], rtol=1e-8, atol=1e-12)
    np.testing.assert_allclose(md.x.numpy(), g["x"], atol=1e-9)
    np.testing.assert_allclose(md.v.numpy(), g["v"], atol=1e-9)


def test_indenter_backbone_matches_reference():
    """LJ + SphericalIndenterForce (summed backbones) over 20 NVE steps with a
    moving centre: the oracle's restatement against the reference's run."""
    from oracle.integrator import indenter
    g = load("ind_ar108_f64")
    box = OracleBox(float(g["box0"]))
    lj = _lj_force_fn(box, 0.0104, 3.405)
    state = {"c": g["center"][0], "last": None}

    def ff(x, i, j):
        a = lj(x, i, j)
        b = indenter(x, state["c"], float(g["radius"]), float(g["stiffness"]))
        state["last"] = b
        return dict(forces=a["forces"] + b["forces"], energy=a["energy"] + b["energy"],
                    virial=a["virial"] + b["virial"], virial_tensor=a["virial_tensor"] + b["virial_tensor"])
    md = OracleMD(g["x0"], g["v0"], np.full(108, oin.AR_MASS), box, ff, cutoff=7.0, skin=0.5, dt=float(g["dt"]))
    E, Fi, n, W = [], [], [], []
    for s in range(int(g["steps"])):
        state["c"] = g["center"][s]
        r = md.step()
        E.append(float(r["energy"]))
        W.append(r["virial_tensor"].numpy())
        Fi.append(state["last"]["force_on_indenter"].numpy())
        n.append(state["last"]["contact_atoms"])
    np.testing.assert_allclose(E, g["energy"], rtol=1e-10)
    np.testing.assert_allclose(np.array(W), g["virial_tensor"], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(np.array(Fi), g["force_on_indenter"], rtol=1e-9, atol=1e-14)
    assert n == list(g["contact_atoms"])
    np.testing.assert_allclose(md.x.numpy(), g["x"], atol=1e-10)
    np.testing.assert_allclose(md.v.numpy(), g["v"], atol=1e-9)


# ------------------------------------------------ native-module call records
def _edge_lerp(tab, a, b, r, inv_dr, n_r):
    """The native kernels' table lookup (cuda source/eam_cuda_ext_kernel.cu:9-18):
    floor, clamp to n_r - 2, one lerp, FP32."""
    x = r.astype(np.float32) * np.float32(inv_dr)
    i = np.clip(np.floor(x).astype(np.int64), 0, n_r - 2)
    t = x - i.astype(np.float32)
    return tab[a, b, i] + t * (tab[a, b, i + 1] - tab[a, b, i])


@pytest.mark.parametrize("name,writer", [("legacy_eam_w250_f32", oin.write_fs_w_setfl),
                                         ("legacy_eam_wli250_f32", oin.write_fs_two_element_setfl)])
def test_native_call_records_match_oracle_tables(tmp_path, name, writer):
    """The oracle's FP32 tables equal the reference's bit for bit (one and two
    elements, digests recorded from the reference), and the recorded pass-1 /
    pass-2 inputs give the recorded rho and forces through the native
    kernels' arithmetic restated here (rho 1e-6 relative, forces 5e-6 eV/A)."""
    import hashlib
    g = load(name)
    t = oeam.EAMTables(oeam.parse_eam(writer(str(tmp_path / "pot.eam.fs"))), dtype=torch.float32)
    for key, tab in (("density_table", t.density), ("density_deriv_table", t.density_deriv),
                     ("pair_table", t.pair), ("pair_deriv_table", t.pair_deriv), ("embed_table", t.embed),
                     ("embed_deriv_table", t.embed_deriv)):
        dig = hashlib.sha256(np.ascontiguousarray(tab.numpy().astype(np.float32)).tobytes()).hexdigest()
        assert dig == str(g[key]), key
    D, DD, PD = t.density.numpy(), t.density_deriv.numpy(), t.pair_deriv.numpy()
    types = g["types"]
    for s in range(int(g["evaluations"])):
        r, row, col = g[f"s{s}_d_distances"], g[f"s{s}_d_row"], g[f"s{s}_d_col"]
        inv_dr, n_r = float(g[f"s{s}_d_inv_dr"]), int(g[f"s{s}_d_n_r"])
        a, b = types[row], types[col]
        rho = np.zeros(len(types))
        np.add.at(rho, row, _edge_lerp(D, a, b, r, inv_dr, n_r))
        np.add.at(rho, col, _edge_lerp(D, b, a, r, inv_dr, n_r))
        assert np.max(np.abs(rho - g[f"s{s}_rho"]) / g[f"s{s}_rho"]) < 1e-6
        dF = g[f"s{s}_f_dF"]
        sc = (dF[row] * _edge_lerp(DD, a, b, r, inv_dr, n_r) + dF[col] * _edge_lerp(DD, b, a, r, inv_dr, n_r)
              + _edge_lerp(PD, a, b, r, inv_dr, n_r))
        fv = -sc[:, None] * g[f"s{s}_f_dist_vec"] / (r[:, None] + 1e-8)
        F = np.zeros((len(types), 3))
        np.add.at(F, row, fv)
        np.add.at(F, col, -fv)
        assert np.max(np.abs(F - g[f"s{s}_forces"])) < 5e-6


@pytest.mark.parametrize("mode", ["raw", "fs", "switch"])
def test_native_lj_call_records_match_oracle(mode):
    """The LJ calls the wrapper makes (in-cutoff edges, per-edge FP32 sigma
    and epsilon, smoothing mode) give the recorded FP64 reference energy and
    forces through the oracle's LJ (energy 1e-6 relative, forces 1e-6 eV/A:
    the positions were recorded as the FP32 copies the wrapper passes)."""
    g = load(f"legacy_lj_arcl108_{mode}_f32")
    L = float(g["box_length"])
    pos = g["pos"].astype(np.float64)
    i, j = g["edge_index"]
    rij = pos[i] - pos[j]
    rij -= L * np.round(rij / L)
    assert np.all(np.sqrt((rij ** 2).sum(1)) <= 7.0)
    out = lj_forward(torch.tensor(pos), torch.tensor(i), torch.tensor(j), torch.tensor(g["epsilon"]),
                     torch.tensor(g["sigma"]), OracleBox(np.diag([L, L, L])), 7.0,
                     mode=["raw", "fs", "switch"][int(g["mode"])], rs=float(g["rs"]) or None)
    assert abs(float(out["energy"]) - float(g["energy"])) < 1e-6 * abs(float(g["energy"]))
    assert np.max(np.abs(out["forces"].numpy() - g["forces"])) < 1e-6


def test_sum_of_eam_and_lj_oracle_matches_reference(fsw):
    """The oracle's EAM (FP32 tables) plus its LJ on the same half list give the
    reference's summed forces, energy and virials at FP32 round-off."""
    g = load("sum_w250_eam_lj_f32")
    box = OracleBox(float(g["box"]))
    x = g["x0"].astype(np.float32)
    hl = onb.half_list(x, box, onb.rc2_like_reference(4.4, 0.5, np.float32))
    t32 = oeam.EAMTables(fsw, dtype=torch.float32)
    e = oeam.eam_forward(torch.tensor(x), hl["i"], hl["j"], np.zeros(len(x), np.int64), box, t32)
    n = len(hl["i"])
    lj = lj_forward(torch.tensor(x), hl["i"], hl["j"], torch.full((n,), float(g["epsilon"]), dtype=torch.float32),
                    torch.full((n,), float(g["sigma"]), dtype=torch.float32), box, 4.4)
    F = e["forces"].numpy() + lj["forces"].numpy()
    assert np.max(np.abs(F - g["forces0"])) < 2e-5
    assert abs(float(e["energy"] + lj["energy"]) - float(g["energy0"])) < 2e-6 * abs(float(g["energy0"]))
    assert abs(float(e["virial"] + lj["virial"]) - float(g["virial0"])) < 2e-5 * abs(float(g["virial0"]))
