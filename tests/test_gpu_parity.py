"""GPU parity: the CUDA path (through libsimb200's C ABI) against the oracle
and against golden vectors produced by the reference itself.

Tolerances (stated per test):
  * neighbour pair sets: bit-exact, including the integer image of each pair;
  * EAM forces vs the FP64 oracle: RMSE <= 1e-5 eV/A (the plain-path target),
    energy per atom within 2e-6 eV;
  * LJ FP64 vs the reference's FP64 path: 1e-10 relative;
  * MD trajectories: FP64 LJ NVE/NVT within 1e-8 A after 30 steps (NVT uses
    the same Philox noise as the replayed reference run).
"""
import os

import numpy as np
import pytest
import torch

from oracle import eam as oeam
from oracle import inputs as oin
from oracle import neighbor as onb
from oracle.box import OracleBox
from oracle.philox import langevin_normals

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
DEV = torch.device("cuda")


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


@pytest.fixture(scope="module")
def sb():
    import simulon_b200
    simulon_b200._lib.load()
    return simulon_b200


@pytest.fixture(scope="module")
def fsw_path(tmp_path_factory):
    return oin.write_fs_w_setfl(str(tmp_path_factory.mktemp("pot") / "W_synthetic.eam.fs"))


# ---------------------------------------------------------------- neighbours
NBR = ["nbr_ar108_f64", "nbr_w250_f32", "nbr_wtri432_f32", "nbr_wtri432_f64", "nbr_gas300_orth_f32",
       "nbr_pair2_f64", "nbr_far3_f32"]


@pytest.mark.parametrize("name", NBR)
def test_half_list_matches_reference_bit_exact(sb, name):
    g = load(name)
    pos = torch.tensor(g["pos"], device=DEV)
    dt = pos.dtype
    cutoff = torch.tensor(float(g["cutoff"]), dtype=dt) + torch.tensor(float(g["skin"]), dtype=dt)
    ei, dist, img = sb.find_neighbors_gpu_pbc(pos, cutoff, OracleBox(g["box"]), return_image=True)
    assert np.array_equal(ei[0].cpu().numpy(), g["i"]) and np.array_equal(ei[1].cpu().numpy(), g["j"])
    o = onb.half_list(g["pos"], OracleBox(g["box"]), onb.rc2_like_reference(float(g["cutoff"]), float(g["skin"]),
                                                                           g["pos"].dtype))
    assert np.array_equal(img.cpu().numpy(), o["image"])
    if len(g["i"]):
        np.testing.assert_allclose(dist.cpu().numpy(), g["dist"], rtol=1e-6 if dt == torch.float32 else 1e-14)


@pytest.mark.parametrize("dtype,tri", [(np.float32, False), (np.float64, True), (np.float32, True)])
def test_half_list_large_matches_oracle(sb, dtype, tri):
    if tri:
        x, H = oin.bcc_triclinic(16)
    else:
        x, L = oin.bcc_lattice(20)
        H = np.diag([L, L, L])
    x = oin.jitter(x, 0.08, 21).astype(dtype)
    rc2 = onb.rc2_like_reference(4.4, 0.5, dtype)
    o = onb.half_list(x, OracleBox(H), rc2, mode="cell")
    ei, _, img = sb.neighbor.half_list(torch.tensor(x, device=DEV), rc2, H, return_image=True)
    assert np.array_equal(ei[0].cpu().numpy(), o["i"]) and np.array_equal(ei[1].cpu().numpy(), o["j"])
    assert np.array_equal(img.cpu().numpy(), o["image"])


def test_engine_list_export_matches_oracle(sb):
    x, L = oin.bcc_lattice(12)
    x = oin.jitter(x, 0.1, 22)
    eng = sb.MDEngine(x, np.zeros(len(x), np.int32), [oin.W_MASS], np.diag([L] * 3), 4.4, 0.5, device=DEV)
    ei, dist = eng.half_list(4.9 ** 2)
    o = onb.half_list(x, OracleBox(L), 4.9 ** 2)
    assert np.array_equal(ei[0].cpu().numpy(), o["i"]) and np.array_equal(ei[1].cpu().numpy(), o["j"])
    assert eng.status() == 0
    # slots are a permutation of the atoms and positions round-trip exactly
    assert torch.equal(eng.gather("x").cpu(), torch.tensor(x))


def test_engine_long_rows_match_oracle(sb):
    """The list builder's long forms: FCC Ar within 11.5 A (~174 neighbours
    per row, beyond the 128-entry sorted-row buffer, so rows are written in
    visiting order) in a 2x2x2 cell grid (500 candidates per stencil, two
    register chunks); the engine's export equals the oracle's pair set."""
    x, L = oin.fcc_lattice(5)
    x = oin.jitter(x, 0.05, 41)
    eng = sb.MDEngine(x, np.zeros(len(x), np.int32), [oin.AR_MASS], np.diag([L] * 3), 11.0, 0.5, device=DEV)
    assert list(eng.ncell) == [2, 2, 2] and eng.neighbor_stats()["max"] > 128
    ei, _ = eng.half_list(11.5 ** 2)
    o = onb.half_list(x, OracleBox(L), 11.5 ** 2)
    assert np.array_equal(ei[0].cpu().numpy(), o["i"]) and np.array_equal(ei[1].cpu().numpy(), o["j"])
    assert eng.status() == 0


def test_engine_half_count_row_offsets_in_place_scan(sb):
    """sim_engine_half_count scans its per-row counts in place (counts in
    row_ptr[1:], offsets into row_ptr): for 16,000 atoms the scan crosses
    the 8192-entry tiles; offsets equal the cumulative sum of the oracle's
    per-row pair counts."""
    from simulon_b200 import _lib
    x, L = oin.bcc_lattice(20)
    x = oin.jitter(x, 0.05, 31)
    eng = sb.MDEngine(x, np.zeros(len(x), np.int32), [oin.W_MASS], np.diag([L] * 3), 4.4, 0.5, device=DEV)
    row_ptr = torch.full((eng.n + 1,), -7, device=DEV, dtype=torch.int64)
    _lib.call("sim_engine_half_count", eng.st_ref, 4.9 ** 2, _lib.ptr(row_ptr), eng.stream)
    o = onb.half_list(x, OracleBox(L), 4.9 ** 2)
    want = np.concatenate([[0], np.cumsum(np.bincount(o["i"], minlength=len(x)))])
    assert np.array_equal(row_ptr.cpu().numpy(), want)


@pytest.mark.parametrize("n", [0, 1, 31, 8192, 8193, 100_003])
def test_scan_i64_matches_cumsum(sb, n):
    """sim_scan_i64: out[0] = 0, out[k+1] = in[0] + ... + in[k], exact in int64,
    across the 8192-entry tiles of its one-block loop."""
    from simulon_b200 import _lib
    rng = np.random.default_rng(n)
    counts = rng.integers(0, 1 << 40, size=n, dtype=np.int64)
    src = torch.tensor(counts, device=DEV)
    out = torch.full((n + 1,), -1, dtype=torch.int64, device=DEV)
    _lib.call("sim_scan_i64", _lib.ptr(src), n, _lib.ptr(out), torch.cuda.current_stream().cuda_stream)
    want = np.concatenate([[0], np.cumsum(counts)])
    assert np.array_equal(out.cpu().numpy(), want)


# ---------------------------------------------------------------- EAM
def _eam_engine(sb, fsw_path, x, H, v=None):
    parser = sb.EAMParser(fsw_path)
    tables = sb.EAMDeviceTables(parser, DEV)
    eng = sb.MDEngine(x, np.zeros(len(x), np.int32), [oin.W_MASS], H, parser.cutoff, 0.5, velocities=v, device=DEV)
    return eng, tables, parser


def _oracle_eam64(fsw_path, x, H):
    p = oeam.parse_eam(fsw_path)
    t64 = oeam.EAMTables(p, dtype=torch.float64)
    box = OracleBox(H)
    hl = onb.half_list(np.asarray(x, np.float64), box, 4.9 ** 2)
    return oeam.eam_forward(torch.tensor(x, dtype=torch.float64), hl["i"], hl["j"], np.zeros(len(x), np.int64),
                            box, t64)


@pytest.mark.parametrize("n,tri", [(5, False), (20, False), (8, True)])
def test_eam_forces_vs_fp64_oracle(sb, fsw_path, n, tri):
    if tri:
        x, H = oin.bcc_triclinic(n)
    else:
        x, L = oin.bcc_lattice(n)
        H = np.diag([L] * 3)
    x = oin.jitter(x, 0.06, 30 + n)
    eng, tables, _ = _eam_engine(sb, fsw_path, x, H)
    eng.eam_forces(tables)
    f = eng.gather("f").cpu().numpy()
    e = float(eng.potential_energy())
    o = _oracle_eam64(fsw_path, x, H)
    rmse = float(np.sqrt(((f - o["forces"].numpy()) ** 2).mean()))
    assert rmse <= 1e-5, rmse
    assert abs(e - float(o["energy"])) / len(x) < 2e-6
    red = eng.red_out.cpu().numpy()
    W = o["virial_tensor"].numpy()
    np.testing.assert_allclose(red[3:6], np.diag(W), rtol=2e-5, atol=1e-3)
    np.testing.assert_allclose(red[6:9], [W[0, 1], W[0, 2], W[1, 2]], atol=1e-3)
    np.testing.assert_allclose(red[2], float(o["virial"]), rtol=2e-5, atol=1e-3)
    np.testing.assert_allclose(red[0], float(o["embedding_energy"]), rtol=1e-6)
    assert eng.status() == 0


def test_eam_vs_reference_golden(sb, fsw_path):
    for name in ("eam_w250_jitter_f32", "eam_wtri432_f32"):
        g = load(name)
        eng, tables, _ = _eam_engine(sb, fsw_path, g["pos"].astype(np.float64), g["box"])
        eng.eam_forces(tables)
        f = eng.gather("f").cpu().numpy()
        # the reference path is FP32 throughout; agreement at its round-off
        assert np.sqrt(((f - g["forces"]) ** 2).mean()) < 5e-5
        assert abs(float(eng.potential_energy()) - float(g["energy"])) / len(f) < 5e-6


def test_eam_perfect_lattice_known_answer(sb, fsw_path):
    x, L = oin.bcc_lattice(10)
    eng, tables, _ = _eam_engine(sb, fsw_path, x, np.diag([L] * 3))
    eng.eam_forces(tables)
    _, _, _, e_atom = oin.perfect_bcc_known_answer()
    assert abs(float(eng.potential_energy()) / len(x) - e_atom) < 1e-5
    assert float(eng.gather("f").abs().max()) < 1e-5


@pytest.mark.parametrize("tri", [False, True])
def test_eam_tiled_equals_untiled(sb, fsw_path, tri):
    """Shared-memory neighbour tiles (16-bit tile-local lists) reproduce the
    untiled kernels' forces bit for bit; sums agree to float32 round-off."""
    if tri:
        x, H = oin.bcc_triclinic(14)
    else:
        x, L = oin.bcc_lattice(16)
        H = np.diag([L] * 3)
    x = oin.jitter(x, 0.07, 41)
    parser = sb.EAMParser(fsw_path)
    tables = sb.EAMDeviceTables(parser, DEV)
    out = []
    for tiles in (False, True):
        eng = sb.MDEngine(x, np.zeros(len(x), np.int32), [oin.W_MASS], H, parser.cutoff, 0.5, device=DEV,
                          use_tiles=tiles)
        assert eng.n_tiles > 1 and eng.status() == 0
        eng.eam_forces(tables)
        out.append((eng.gather("f").cpu(), eng.red_out.cpu().numpy()))
    assert torch.equal(out[0][0], out[1][0])
    np.testing.assert_allclose(out[1][1][:9], out[0][1][:9], rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("kind", ["ortho", "tri", "dense"])
def test_eam_cutoff_mask_equals_full_scan(sb, fsw_path, kind):
    """Pass 2 over the in-cutoff slots recorded by pass 1 gives the same forces,
    energies and virial, bit for bit, as pass 2 testing every list slot.
    "dense": BCC compressed to a = 2.75 A, ~34 neighbours inside the cutoff
    and ~47 list entries per row, so rows whose leading run of in-cutoff
    slots fills the mask's low word, and slots of 32 and above, are walked."""
    if kind == "tri":
        x, H = oin.bcc_triclinic(12)
    else:
        x, L = oin.bcc_lattice(14, 2.75) if kind == "dense" else oin.bcc_lattice(14)
        H = np.diag([L] * 3)
    x = oin.jitter(x, 0.09, 43)
    if kind == "dense":   # rows of <= 58 entries: a 64-slot list keeps the mask path
        parser = sb.EAMParser(fsw_path)
        tables = sb.EAMDeviceTables(parser, DEV)
        eng = sb.MDEngine(x, np.zeros(len(x), np.int32), [oin.W_MASS], H, parser.cutoff, 0.5, nbr_cap=64,
                          device=DEV)
        assert eng.neighbor_stats()["max"] > 40 and eng.status() == 0
    else:
        eng, tables, _ = _eam_engine(sb, fsw_path, x, H)
    assert eng.cut_mask is not None
    out = []
    for masked in (True, False):
        if not masked:
            eng.cut_mask = None
            eng._make_struct()
        eng.eam_forces(tables)
        out.append((eng.gather("f").cpu(), eng.red_out.cpu()))
    assert torch.equal(out[0][0], out[1][0]) and torch.equal(out[0][1], out[1][1])


def test_eam_reruns_bitwise_identical(sb, fsw_path):
    x, L = oin.bcc_lattice(16)
    x = oin.jitter(x, 0.07, 40)
    outs = []
    for _ in range(2):
        eng, tables, _ = _eam_engine(sb, fsw_path, x, np.diag([L] * 3))
        eng.eam_forces(tables)
        outs.append((eng.gather("f").cpu(), eng.red_out.cpu()))
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])


# ---------------------------------------------------------------- LJ
def _lj_system(sb, tmp_path, x, L, mode, dtype):
    torch.set_default_dtype(dtype)
    try:
        path = oin.write_xyz(str(tmp_path / "ar.xyz"), x, "Ar")
        mol = sb.AtomFileReader(path, L, 7.0, device=DEV, parameter={"[0 0]": {"epsilon": 0.0104, "sigma": 3.405}},
                                skin_thickness=0.5, is_fs=mode == "fs", is_switch=mode == "switch")
        return mol, sb.LennardJonesForce(mol)
    finally:
        torch.set_default_dtype(torch.float32)


@pytest.mark.parametrize("mode", ["raw", "fs", "switch"])
def test_lj_fp64_matches_reference(sb, tmp_path, mode):
    g = load(f"lj_ar108_{mode}_f64")
    mol, ff = _lj_system(sb, tmp_path, g["pos"], float(g["box"][0, 0]), mode, torch.float64)
    out = ff()
    np.testing.assert_allclose(float(out["energy"]), float(g["energy"]), rtol=1e-11)
    np.testing.assert_allclose(out["forces"].cpu().numpy(), g["forces"], rtol=1e-9, atol=1e-13)
    np.testing.assert_allclose(float(out["virial"]), float(g["virial"]), rtol=1e-11)
    np.testing.assert_allclose(out["virial_tensor"].cpu().numpy(), g["virial_tensor"], rtol=1e-10, atol=1e-13)


@pytest.mark.parametrize("mode", ["raw", "fs", "switch"])
def test_lj_fp32_pairs_match_reference(sb, tmp_path, mode):
    g = load(f"lj_ar108_{mode}_f64")
    mol, ff = _lj_system(sb, tmp_path, g["pos"], float(g["box"][0, 0]), mode, torch.float32)
    out = ff()
    assert abs(float(out["energy"]) - float(g["energy"])) < 2e-6 * abs(float(g["energy"])) + 1e-6
    f = out["forces"].double().cpu().numpy()
    assert np.sqrt(((f - g["forces"]) ** 2).mean()) < 2e-6


@pytest.mark.parametrize("mode,n", [("raw", 6), ("switch", 6), ("raw", 48)])
def test_lj_fused_integrator_equals_separate_kernels(sb, tmp_path, mode, n):
    """FP32 LJ with the integrator in the force pass (second half; second half
    plus the next first half) against the separate force and integrator
    kernels: positions and velocities bit for bit after 40 Langevin steps,
    triggered rebuilds included; energies and virials to FP32 sum order.  At
    n = 48 (442,368 atoms) each thread of the persistent grid takes three
    atoms, so a pass whose first half moved atoms that later iterations still
    gather would show here."""
    from simulon_b200.engine import integrator_params
    x, L = oin.fcc_lattice(n)
    x = oin.jitter(x, 0.05, 91)
    res = []
    for fused in ("separate", "second", "drift"):
        mol, ff = _lj_system(sb, tmp_path, x, L, mode, torch.float32)
        eng = mol.engine
        eng.set_velocities(torch.tensor(oin.maxwell_boltzmann(np.full(len(x), 39.948), 300.0, 92), device=DEV))
        ip = integrator_params(eng, 0.004, langevin=True, temperature=300.0, gamma=10.0, seed=9)
        ff.compute()
        if fused == "drift":
            eng.integrate_first(ip, 0)
            eng.rebuild_if_needed()
            for s in range(40):
                if s < 39:
                    eng.lj_forces_integrate(ff.params, ip, 2)
                    eng.rebuild_if_needed()
                else:
                    eng.lj_forces_integrate(ff.params, ip, 1)
        else:
            for _ in range(40):
                eng.integrate_first(ip, 0)
                eng.rebuild_if_needed()
                if fused == "second":
                    eng.lj_forces_integrate(ff.params, ip, 1)
                else:
                    eng.lj_forces(ff.params, 0)
                    eng.integrate_second(ip, 0)
        torch.cuda.synchronize()
        assert eng.status() == 0
        res.append((eng.gather("x").cpu(), eng.gather("v").cpu(), int(eng.flags[3]), eng.red_out.cpu().numpy(),
                    int(eng.step_ctr[0])))
    assert res[0][2] >= 2     # the load rebuild plus at least one triggered
    for r in res[1:]:
        assert torch.equal(r[0], res[0][0]) and torch.equal(r[1], res[0][1])
        assert r[2] == res[0][2] and r[4] == res[0][4]
        np.testing.assert_allclose(r[3][1:10], res[0][3][1:10], rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("tri", [False, True])
def test_lj_fp32_two_types_matches_fp64(sb, tri):
    """FP32-pair LJ for an Ar/Ne mixture (per type-pair constants read per
    pair) in an orthogonal and a triclinic box, against the FP64 path on the
    same positions: force RMSE < 5e-6 eV/A, energy and virial tensor within
    FP32 round-off."""
    x, L = oin.fcc_lattice(5)
    x = oin.jitter(x, 0.05, 93)
    H = oin.triclinic_box(L) if tri else np.diag([L] * 3)
    if tri:
        x = (x / L) @ H
    sym = ["Ne" if k % 3 == 0 else "Ar" for k in range(len(x))]
    par = {"[0 0]": {"epsilon": 0.00307, "sigma": 2.78}, "[0 1]": {"epsilon": 0.00565, "sigma": 3.09},
           "[1 1]": {"epsilon": 0.0104, "sigma": 3.405}}
    out = []
    for dt in (torch.float32, torch.float64):
        torch.set_default_dtype(dt)
        try:
            mol = sb.AtomFileReader.from_arrays(sym, x, L, 7.0, device=DEV, parameter=par, skin_thickness=0.5,
                                                box_vectors=H if tri else None)
            ff = sb.LennardJonesForce(mol)
        finally:
            torch.set_default_dtype(torch.float32)
        assert mol.engine.n_types == 2 and bool(mol.engine.st.box_orthogonal) == (not tri)
        o = ff()
        out.append((o["forces"].double().cpu().numpy(), float(o["energy"]), o["virial_tensor"].double().cpu().numpy()))
    rmse = float(np.sqrt(((out[0][0] - out[1][0]) ** 2).mean()))
    assert rmse < 5e-6, rmse
    assert abs(out[0][1] - out[1][1]) < 2e-6 * abs(out[1][1]) + 1e-6
    np.testing.assert_allclose(out[0][2], out[1][2], rtol=1e-5, atol=1e-4)


# ---------------------------------------------------------------- MD
@pytest.mark.parametrize("ens", ["nve", "nvt"])
def test_md_lj_fp64_matches_reference_trajectory(sb, tmp_path, ens):
    g = load(f"md_ar108_{ens}_f64")
    torch.set_default_dtype(torch.float64)
    try:
        path = oin.write_xyz(str(tmp_path / "ar.xyz"), g["x0"], "Ar")
        mol = sb.AtomFileReader(path, float(g["box"]), 7.0, device=DEV,
                                parameter={"[0 0]": {"epsilon": 0.0104, "sigma": 3.405}}, skin_thickness=0.5)
        integ = sb.VerletIntegrator(mol, dt=float(g["dt"]), ensemble=ens.upper(),
                                    temperature=(94.4, 94.4) if ens == "nvt" else None,
                                    gamma=10.0 if ens == "nvt" else None, seed=int(g["noise_seed"]))
        mol.atom_velocities = torch.tensor(g["v0"], device=DEV)
        model = sb.BaseModel(sb.SumBackboneInterface([sb.LennardJonesForce(mol)], mol), integ, mol)
        e, k = [], []
        for _ in range(int(g["steps"])):
            out = model()
            e.append(float(out["energy"]))
            k.append(float(out["kinetic_energy"]))
        np.testing.assert_allclose(e, g["energy"], rtol=1e-9)
        np.testing.assert_allclose(k, g["kinetic_energy"], rtol=1e-7 if ens == "nvt" else 1e-9)
        np.testing.assert_allclose(mol.coordinates.cpu().numpy(), g["x"], atol=1e-8)
        np.testing.assert_allclose(mol.atom_velocities.cpu().numpy(), g["v"], atol=1e-7)
    finally:
        torch.set_default_dtype(torch.float32)


@pytest.mark.parametrize("ens", ["nve", "npt"])
def test_md_eam_matches_reference_trajectory(sb, fsw_path, tmp_path, ens):
    g = load(f"md_w250_{ens}_f32")
    path = oin.write_xyz(str(tmp_path / "w.xyz"), g["x0"], "W")
    parser = sb.EAMParser(fsw_path)
    mol = sb.AtomFileReader(path, float(g["box0"]), parser.cutoff, device=DEV, skin_thickness=0.5, is_fs=True)
    integ = sb.VerletIntegrator(mol, dt=float(g["dt"]), ensemble="NPT" if ens == "npt" else "NVE",
                                temperature=(300.0, 300.0) if ens == "npt" else None,
                                gamma=10.0 if ens == "npt" else None, seed=int(g["noise_seed"]))
    mol.atom_velocities = torch.tensor(g["v0"].astype(np.float32), device=DEV)
    baro = sb.BerendsenBarostat(mol, 0.0, float(g["tau_p"])) if ens == "npt" else None
    model = sb.BaseModel(sb.SumBackboneInterface([sb.EAMForceCUDAExt(parser, mol)], mol), integ, mol, barostat=baro)
    e, p = [], []
    for _ in range(int(g["steps"])):
        out = model()
        e.append(float(out["energy"]))
        if baro is not None:
            p.append(float(out["pressure"]))
    # the reference integrates in FP32 here; the device keeps FP64 state
    np.testing.assert_allclose(e, g["energy"], rtol=2e-5)
    if baro is not None:
        np.testing.assert_allclose(p, g["pressure"], rtol=2e-3, atol=100.0)
        np.testing.assert_allclose(mol.engine.box_matrix(), g["box"], rtol=2e-6)
    np.testing.assert_allclose(mol.coordinates.cpu().numpy(), g["x"], atol=5e-4)


def test_npt_runs_equal_per_step_calls(sb, fsw_path):
    """Berendsen NPT: BaseModel.run folds each step's atom scaling into the next
    step's first half (sim_berendsen_scale_first); per-step calls scale
    separately (sim_berendsen).  Same positions, velocities, box and log rows,
    bit for bit, graphed and eager."""
    x, L = oin.bcc_lattice(8)
    x = oin.jitter(x, 0.05, 61)
    v = oin.maxwell_boltzmann(np.full(len(x), oin.W_MASS), 600.0, 62)
    parser = sb.EAMParser(fsw_path)
    res = []
    for mode in ("calls", "graph", "eager"):
        mol = sb.AtomFileReader.from_arrays(["W"] * len(x), x, L, parser.cutoff, device=DEV, skin_thickness=0.5,
                                            is_fs=True)
        integ = sb.VerletIntegrator(mol, dt=0.002, ensemble="NPT", temperature=(600.0, 600.0), gamma=10.0, seed=3)
        mol.atom_velocities = torch.tensor(v, device=DEV)   # after the integrator's own Maxwell-Boltzmann draw
        baro = sb.BerendsenBarostat(mol, 0.0, 1.0)
        model = sb.BaseModel(sb.SumBackboneInterface([sb.EAMForceCUDAExt(parser, mol)], mol), integ, mol,
                             barostat=baro)
        if mode == "calls":
            for _ in range(60):
                model()
        elif mode == "graph":
            model.run(60, graph_steps=20)
        else:
            for _ in range(4):
                model.run(15, graph_steps=20)      # below graph_steps: eager launches
        torch.cuda.synchronize()
        eng = mol.engine
        assert eng.status() == 0
        res.append((eng.gather("x").cpu(), eng.gather("v").cpu(), eng.box_matrix(), eng.log[:60].cpu().numpy(),
                    int(eng.flags[3])))
    assert abs(np.linalg.det(res[0][2]) / L ** 3 - 1.0) > 1e-6      # the box did move
    for r in res[1:]:
        assert torch.equal(r[0], res[0][0]) and torch.equal(r[1], res[0][1])
        np.testing.assert_array_equal(r[2], res[0][2])
        np.testing.assert_array_equal(r[3], res[0][3])
        assert r[4] == res[0][4]


def _lib_red_slots():
    from simulon_b200 import _lib
    return _lib.RED_SLOTS


def test_eam_drift_fused_equals_separate_at_scale(sb, fsw_path):
    """BCC W 2*64^3 = 524,288 atoms, where each thread of the persistent pass 2
    takes three or four atoms: 30 Langevin steps with the next first half
    fused into pass 2 (sim_eam_step_drift) against separate force, second-half
    and first-half kernels, positions and velocities bit for bit (pass 2
    gathers pass 1's copy of the positions, so atoms that its epilogue has
    moved are never seen by the same pass)."""
    from simulon_b200.engine import integrator_params
    x, L = oin.bcc_lattice(64)
    x = oin.jitter(x, 0.05, 52)
    v = oin.maxwell_boltzmann(np.full(len(x), oin.W_MASS), 600.0, 53)
    res = []
    for fused in (False, True):
        eng, tables, _ = _eam_engine(sb, fsw_path, x, np.diag([L] * 3), v)
        integ = integrator_params(eng, 0.002, langevin=True, temperature=600.0, gamma=10.0, seed=7)
        eng.eam_forces(tables)
        eng.integrate_first(integ, 0)
        eng.rebuild_if_needed()
        for s in range(30):
            if fused and s < 29:
                eng.eam_step_drift(tables, integ)
                continue
            eng.eam_forces(tables)
            eng.integrate_second(integ, 0)
            if s < 29:
                eng.integrate_first(integ, 0)
                eng.rebuild_if_needed()
        torch.cuda.synchronize()
        assert eng.status() == 0
        res.append((eng.gather("x").cpu(), eng.gather("v").cpu(), int(eng.flags[3])))
    assert torch.equal(res[0][0], res[1][0]) and torch.equal(res[0][1], res[1][1])
    assert res[0][2] == res[1][2]


def test_graph_run_matches_eager_steps(sb, fsw_path):
    x, L = oin.bcc_lattice(10)
    x = oin.jitter(x, 0.05, 50)
    v = oin.maxwell_boltzmann(np.full(len(x), oin.W_MASS), 600.0, 51)
    res = []
    from simulon_b200.engine import integrator_params
    # (graph?, conditional IF-node rebuild?, second half fused into EAM pass 2?);
    # fused == "drift": the next step's first half is fused in as well;
    # fused == "sf": standalone forces, then sim_integrate_second_first;
    # fused == "step": sim_eam_step_drift (log row and rebuild decision in pass 2)
    modes = [(False, False, False), (True, False, False), (True, True, False), (True, True, True), (False, True, True),
             (False, True, "drift"), (True, True, "drift"), (False, True, "sf"), (True, True, "sf"),
             (False, True, "step"), (True, True, "step")]
    for use_graph, cond, fused in modes:
        eng, tables, parser = _eam_engine(sb, fsw_path, x, np.diag([L] * 3), v)
        # an NVT integrator exercises the noise and triggers rebuilds
        integ = integrator_params(eng, 0.002, langevin=True, temperature=600.0, gamma=10.0, seed=7)
        eng.eam_forces(tables)

        def drift_steps(k):
            eng.integrate_first(integ, 0)
            eng.rebuild_if_needed()
            for s in range(k):
                if s < k - 1 and fused == "step":
                    eng.eam_step_drift(tables, integ)
                elif s < k - 1:
                    if fused == "sf":
                        eng.eam_forces(tables)
                        eng.integrate_second_first(integ, 0)
                    else:
                        eng.eam_forces_integrate_drift(tables, integ)
                    eng.log_step(after_drift=True)
                    eng.rebuild_if_needed()
                elif fused == "sf":
                    eng.eam_forces(tables)
                    eng.integrate_second(integ, 0)
                    eng.log_step()
                else:
                    eng.eam_forces_integrate(tables, integ)
                    eng.log_step()

        def step():
            eng.integrate_first(integ, 0)
            if cond:
                eng.rebuild_if_needed()
            else:
                eng.rebuild(True)
            if fused:
                eng.eam_forces_integrate(tables, integ)
            else:
                eng.eam_forces(tables)
                eng.integrate_second(integ, 0)
        steps = 60
        if use_graph:
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=s):
                if fused in ("drift", "sf", "step"):
                    drift_steps(20)
                else:
                    for _ in range(20):
                        step()
                        eng.log_step()
            torch.cuda.current_stream().wait_stream(s)
            for _ in range(steps // 20):
                g.replay()
        elif fused in ("drift", "sf", "step"):
            for _ in range(steps // 20):
                drift_steps(20)
        else:
            for _ in range(steps):
                step()
                eng.log_step()
        torch.cuda.synchronize()
        res.append((eng.gather("x").cpu(), eng.gather("v").cpu(), int(eng.flags[3].item()),
                    eng.red_out.cpu().numpy(), eng.log[:steps, :_lib_red_slots()].cpu().numpy(),
                    eng.step_ctr.cpu().numpy(), eng.log[:steps].cpu().numpy()))
    for r in res[1:]:
        assert torch.equal(res[0][0], r[0]) and torch.equal(res[0][1], r[1])
        assert r[2] == res[0][2]
        assert r[5][0] == res[0][5][0] == steps - 1
        # per-step log rows: energies and virial agree to FP32 partial-sum order
        np.testing.assert_allclose(r[4][:, :9], res[0][4][:, :9], rtol=1e-6, atol=1e-9)
        np.testing.assert_allclose(r[3][9], res[0][3][9], rtol=1e-6)   # kinetic energy (FP32 per-thread partials)
    assert res[0][2] >= 2      # the load rebuild plus at least one triggered
    # the step entry point runs the drift path's kernels: whole log rows
    # (reductions, extra columns, status) equal bit for bit, eager and graphed
    drift = res[modes.index((True, True, "drift"))][6]
    for m in ((False, True, "step"), (True, True, "step")):
        np.testing.assert_array_equal(res[modes.index(m)][6], drift)


def test_langevin_noise_matches_oracle_philox(sb, fsw_path):
    """One NVT step from rest with zero forces isolates the noise: v = xi * rff."""
    x, L = oin.bcc_lattice(6)
    eng, tables, parser = _eam_engine(sb, fsw_path, x, np.diag([L] * 3))
    from simulon_b200.engine import integrator_params
    integ = integrator_params(eng, 0.002, langevin=True, temperature=300.0, gamma=10.0, seed=123456789)
    eng.f32.zero_()
    eng.integrate_first(integ, 0)
    eng.integrate_second(integ, 0)
    v = eng.gather("v").cpu().numpy()
    z = langevin_normals(len(x), 0, 123456789)
    rff = integ.keep[0].cpu().numpy()[0]
    np.testing.assert_allclose(v, z * rff, rtol=1e-6, atol=1e-12)


def test_neighbor_overflow_is_detected_and_grown(sb, fsw_path):
    x, L = oin.bcc_lattice(8)
    eng = sb.MDEngine(x, np.zeros(len(x), np.int32), [oin.W_MASS], np.diag([L] * 3), 4.4, 0.5, device=DEV, nbr_cap=8)
    assert eng.nbr_cap >= 26 and eng.status() & sb._lib.SIM_STATUS_OVERFLOW == 0
    assert eng.neighbor_stats()["max"] == 26


# ------------------------------------------------ Maxwell-Boltzmann velocities
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_maxwell_boltzmann_velocities_match_reference_formula(sb, dtype):
    """AtomFileReader.set_maxwell_boltzmann_velocity against the reference's
    formula (io_utils/reader.py:319-339) restated here with the same seeded
    torch generator: bit-equal velocities; centre-of-mass momentum zero to
    round-off; the per-species kinetic temperature within 5% of the target
    for 54,000 atoms of two masses (6,000 of the lighter one)."""
    old = torch.get_default_dtype()
    torch.set_default_dtype(dtype)
    try:
        coords, L = oin.bcc_lattice(30)       # 54,000 sites, every ninth one a lighter species
        symbols = ["Ar" if k % 9 == 0 else "W" for k in range(len(coords))]
        mol = sb.AtomFileReader.from_arrays(symbols, coords, L, 4.4, device=DEV, skin_thickness=0.5)
        T = 523.0
        torch.manual_seed(1234)
        mol.set_maxwell_boltzmann_velocity(T)
        v = mol.atom_velocities
        # the reference's formula, same generator state
        torch.manual_seed(1234)
        m_internal = (mol.atom_mass * 1.036427e-4).unsqueeze(-1)
        sigma = torch.sqrt(8.617333262e-5 * T / m_internal)
        ref = torch.randn((mol.atom_count, 3), device=DEV, dtype=dtype) * sigma
        ref = ref - (ref * m_internal).sum(dim=0) / m_internal.sum()
    finally:
        torch.set_default_dtype(old)
    assert v.dtype == dtype and torch.equal(v, ref)
    m = m_internal.double()
    p = (v.double() * m).sum(0)
    assert float(p.abs().max()) < (1e-9 if dtype == torch.float64 else 1e-4) * float((v.double().abs() * m).sum())
    light = torch.tensor([s == "Ar" for s in symbols], device=DEV)
    for sel in (light, ~light):
        ke = 0.5 * float((m[sel] * v[sel].double() ** 2).sum())
        t_kin = 2.0 * ke / (3.0 * int(sel.sum())) / 8.617333262e-5
        assert abs(t_kin / T - 1.0) < 0.05, t_kin


def test_update_coordinates_from_pinned_host_rows(sb, fsw_path):
    """update_coordinates(x, velocities=v) from pinned float32 host rows (the
    velocities cross on a side stream while the cell sort and list build run)
    reads back the same rows, and 10 MD steps from it are bit-equal to the
    same steps after a load of the same rows from device tensors."""
    coords, L = oin.bcc_lattice(8)
    rng = np.random.default_rng(11)
    x = np.minimum(np.mod(oin.jitter(coords, 0.08, 5) + 0.3 * L, L), L - 1e-3)[rng.permutation(len(coords))]
    v = rng.normal(0.0, 0.01, x.shape)
    xh = torch.tensor(x, dtype=torch.float32).pin_memory()
    vh = torch.tensor(v, dtype=torch.float32).pin_memory()
    parser = sb.EAMParser(fsw_path)
    states = []
    for host in (True, False):
        mol = sb.AtomFileReader.from_arrays(["W"] * len(x), coords, L, parser.cutoff, device=DEV, skin_thickness=0.5,
                                            is_fs=True)
        model = sb.BaseModel(sb.SumBackboneInterface([sb.EAMForceCUDAExt(parser, mol)], mol),
                             sb.VerletIntegrator(mol, dt=0.002, ensemble="NVE"), mol)
        model.run(3, graph_steps=3)
        if host:
            mol.update_coordinates(xh, velocities=vh)
        else:
            mol.update_coordinates(xh.to(DEV), velocities=vh.to(DEV))
        assert torch.equal(mol.coordinates.cpu(), xh) and torch.equal(mol.atom_velocities.cpu(), vh)
        model.run(10, graph_steps=5)
        states.append((mol.engine.gather("x").cpu(), mol.engine.gather("v").cpu()))
    assert torch.equal(states[0][0], states[1][0]) and torch.equal(states[0][1], states[1][1])


# ------------------------------------------------ sum of force fields
def test_sum_of_eam_and_lj_matches_reference(sb, fsw_path, tmp_path):
    """SumBackboneInterface([EAM, LJ]) (core/md_model.py:19-52): the LJ pass
    adds its forces, energy and virials to the EAM pass's on the device
    (sim_lj_forces_add).  One evaluation against the reference's summed
    outputs (forces 5e-5 eV/A, energy 2e-6 relative, virials 1e-5 relative),
    then 10 NVE steps through BaseModel (energies 2e-5 relative, positions
    5e-4 A; the reference integrates in FP32, the device in FP64)."""
    g = load("sum_w250_eam_lj_f32")
    path = oin.write_xyz(str(tmp_path / "w.xyz"), g["x0"], "W")
    parser = sb.EAMParser(fsw_path)
    params = {"[0 0]": {"epsilon": float(g["epsilon"]), "sigma": float(g["sigma"])}}
    mol = sb.AtomFileReader(path, float(g["box"]), parser.cutoff, device=DEV, skin_thickness=0.5,
                            parameter=params)
    bone = sb.SumBackboneInterface([sb.EAMForceCUDAExt(parser, mol), sb.LennardJonesForce(mol)], mol)
    out = bone()
    assert np.max(np.abs(out["forces"].cpu().numpy() - g["forces0"])) < 5e-5
    assert abs(float(out["energy"]) - float(g["energy0"])) < 2e-6 * abs(float(g["energy0"]))
    assert abs(float(out["virial"]) - float(g["virial0"])) < 1e-5 * abs(float(g["virial0"]))
    np.testing.assert_allclose(out["virial_tensor"].cpu().numpy(), g["virial_tensor0"], rtol=1e-5,
                               atol=1e-5 * float(np.abs(g["virial_tensor0"]).max()))
    integ = sb.VerletIntegrator(mol, dt=float(g["dt"]), ensemble="NVE")
    mol.atom_velocities = torch.tensor(g["v0"].astype(np.float32), device=DEV)
    model = sb.BaseModel(bone, integ, mol)
    e = [float(model()["energy"]) for _ in range(int(g["steps"]))]
    np.testing.assert_allclose(e, g["energy"], rtol=2e-5)
    np.testing.assert_allclose(mol.coordinates.cpu().numpy(), g["x"], atol=5e-4)
    assert mol.engine.status() == 0
