"""Tensile-workflow callers of the force path on the GPU: the device
UniaxialTensileLoader and AnisotropicNPTBarostat against the reference's own
run (tests/golden/mech_ar108_*_f64.npz, written by running the unmodified
reference; the oracle's restatement is pinned to the same vectors by
tests/test_oracle_golden.py).  LJ argon 108 atoms, FP64 forces, NVE: energies
and axis pressures to 1e-8 relative, box to 1e-12, strain rates to 1e-7,
final wrapped positions to 1e-8 A and velocities to 1e-7 A/ps.  Also: the
cell-grid guard reports a box that shrank below the list cutoff per cell, and
MDEngine.regrid repairs it.  The graph variants capture the whole run
(loader steps included, UniaxialTensileLoader.run) and compare the final
state."""
import json

import numpy as np
import pytest
import torch

from oracle import inputs as oin

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")


@pytest.fixture(scope="module")
def fsw_path(tmp_path_factory):
    return oin.write_fs_w_setfl(str(tmp_path_factory.mktemp("pot") / "W_synthetic.eam.fs"))


@pytest.fixture(scope="module")
def sb():
    import simulon_b200
    simulon_b200._lib.load()
    return simulon_b200


def _golden(name):
    import os
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    with np.load(os.path.join(here, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("name", ["tensile", "aniso"])
@pytest.mark.parametrize("graph", [False, True])
def test_tensile_and_aniso_npt_match_reference(sb, tmp_path, name, graph):
    from simulon_b200.barostat import AnisotropicNPTBarostat
    from simulon_b200.mechanics import UniaxialTensileLoader
    g = _golden(f"mech_ar108_{name}_f64")
    load_kw = json.loads(str(g["load"]))
    baro_kw = json.loads(str(g["baro"]))
    torch.set_default_dtype(torch.float64)
    try:
        path = oin.write_xyz(str(tmp_path / "ar.xyz"), g["x0"], "Ar")
        mol = sb.AtomFileReader(path, float(g["box0"]), 7.0, device=DEV,
                                parameter={"[0 0]": {"epsilon": 0.0104, "sigma": 3.405}}, skin_thickness=0.5)
        integ = sb.VerletIntegrator(mol, dt=float(g["dt"]), ensemble="NVE")
        mol.atom_velocities = torch.tensor(g["v0"], device=DEV)
        baro = AnisotropicNPTBarostat(mol, temperature_k=94.4, tau_p=0.2, gamma_p=2.0, compressibility_bar_inv=3.2e-5,
                                      pressure_tolerance_bar=25.0, **baro_kw)
        model = sb.BaseModel(sb.SumBackboneInterface([sb.LennardJonesForce(mol)], mol), integ, mol, barostat=baro)
        loader = UniaxialTensileLoader(mol, **load_kw) if load_kw else None
        E, P, H, eta, strain = [], [], [], [], []
        for s in range(int(g["steps"])):
            if graph:     # whole run as CUDA graphs (loader and MD steps captured together): no per-step record
                if loader is None:
                    model.run(int(g["steps"]), graph_steps=5)
                else:
                    last = loader.run(model, int(g["steps"]), float(g["dt"]), graph_steps=5)
                    np.testing.assert_allclose(float(last), g["strain"][-1], rtol=1e-12)
                break
            strain.append(loader.step(float(g["dt"])) if loader else 0.0)
            out = model()
            E.append(float(out["energy"]))
            P.append(out["pressure"].cpu().numpy().copy())
            H.append(mol.engine.box_matrix())
            eta.append(baro.eta_dot.cpu().numpy().copy())
        if E:
            np.testing.assert_allclose(E, g["energy"], rtol=1e-9)
            np.testing.assert_allclose(np.array(P), g["pressure"], rtol=1e-8, atol=1e-6)
            np.testing.assert_allclose(np.array(H), g["H"], rtol=1e-12, atol=1e-12)
            np.testing.assert_allclose(np.array(eta), g["eta_dot"], rtol=1e-7, atol=1e-12)
            np.testing.assert_allclose(strain, g["strain"], rtol=1e-12)
        else:
            np.testing.assert_allclose(mol.engine.box_matrix(), g["H"][-1], rtol=1e-12, atol=1e-12)
            np.testing.assert_allclose(baro.eta_dot.cpu().numpy(), g["eta_dot"][-1], rtol=1e-7, atol=1e-12)
        np.testing.assert_allclose(mol.coordinates.cpu().numpy(), g["x"], atol=1e-8)
        np.testing.assert_allclose(mol.atom_velocities.cpu().numpy(), g["v"], atol=1e-7)
        assert mol.engine.status() == 0
    finally:
        torch.set_default_dtype(torch.float32)


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_fused_tensile_steps_equal_per_step_calls(sb, tmp_path, fsw_path, precision):
    """loader.run (CUDA graphs; the barostat's atom scaling of step s, the
    loader's update and the first half of step s+1 in one pass,
    sim_box_scale_after_first) against the reference-shaped loop
    loader.step(dt); model() with separate launches: positions, velocities,
    box, strain rates and step-log rows bit for bit.  LJ argon with FP64 forces
    and EAM tungsten with FP32 forces."""
    from simulon_b200.barostat import AnisotropicNPTBarostat
    from simulon_b200.mechanics import UniaxialTensileLoader
    old = torch.get_default_dtype()
    res = []
    for mode in ("calls", "run"):
        if precision == "f64":
            torch.set_default_dtype(torch.float64)
            x, L = oin.fcc_lattice(3)
            x = oin.jitter(x, 0.05, 0)
            v = oin.maxwell_boltzmann(np.full(len(x), oin.AR_MASS), 94.4, 1)
            mol = sb.AtomFileReader.from_arrays(["Ar"] * len(x), x, L, 7.0, device=DEV, skin_thickness=0.5,
                                                parameter={"[0 0]": {"epsilon": 0.0104, "sigma": 3.405}})
            ff = sb.LennardJonesForce(mol)
            T = 94.4
        else:
            x, L = oin.bcc_lattice(8)
            x = oin.jitter(x, 0.05, 71)
            v = oin.maxwell_boltzmann(np.full(len(x), oin.W_MASS), 300.0, 72)
            parser = sb.EAMParser(fsw_path)
            mol = sb.AtomFileReader.from_arrays(["W"] * len(x), x, L, parser.cutoff, device=DEV, skin_thickness=0.5,
                                                is_fs=True)
            ff = sb.EAMForceCUDAExt(parser, mol)
            T = 300.0
        try:
            integ = sb.VerletIntegrator(mol, dt=0.002, ensemble="NVE")
            mol.atom_velocities = torch.tensor(v, device=DEV)
            baro = AnisotropicNPTBarostat(mol, [0.0, 0.0, 0.0], temperature_k=T, control_axes=(False, True, True),
                                          compressibility_bar_inv=3.2e-5)
            model = sb.BaseModel(sb.SumBackboneInterface([ff], mol), integ, mol, barostat=baro)
            loader = UniaxialTensileLoader(mol, axis=0, strain_rate=2.0)
            if mode == "calls":
                for _ in range(12):
                    loader.step(0.002)
                    model()
            else:
                loader.run(model, 12, 0.002, graph_steps=5)
            torch.cuda.synchronize()
            eng = mol.engine
            res.append((eng.gather("x").cpu().numpy(), eng.gather("v").cpu().numpy(), eng.box_matrix(),
                        baro.eta_dot.cpu().numpy(), model.step_log(0, 12).cpu().numpy(), float(loader.state[12])))
            assert eng.status() == 0
        finally:
            torch.set_default_dtype(old)
    a, b = res
    for k in range(5):
        np.testing.assert_array_equal(a[k], b[k])
    assert a[5] == b[5]


def test_cell_guard_and_regrid(sb, tmp_path):
    """A loader that contracts the lateral axes (Poisson) below the grid's
    rc + skin per cell: the rebuild reports SIM_STATUS_CELLS unless the loader
    regrids, and after the regrid the list equals a fresh engine's list."""
    from simulon_b200 import _lib
    from simulon_b200.mechanics import UniaxialTensileLoader
    x, L = oin.bcc_lattice(12)                      # 37.98 A: 7 cells of 5.43 A at rc + skin = 4.9 A
    x = oin.jitter(x, 0.03, 5)
    eng = sb.MDEngine(x, np.zeros(len(x), np.int32), [oin.W_MASS], np.diag([L] * 3), 4.4, 0.5, device=DEV)
    assert list(eng.ncell) == [7, 7, 7]
    # shrink y and z by 12 % directly: the next rebuild must flag the grid
    work = torch.zeros(_lib.BOXSCALE_WORK, dtype=torch.float64, device=DEV)
    s = _lib.SimBoxScale()
    s.scale[:] = [1.0, 0.88, 0.88]
    s.vel_scale[:] = [1.0, 1.0, 1.0]
    s.reset_reference = 1
    import ctypes
    _lib.call("sim_box_scale", eng.st_ref, ctypes.byref(s), _lib.ptr(work), eng.stream)
    eng.rebuild(only_if_flagged=False)
    assert eng.status() & _lib.SIM_STATUS_CELLS
    assert not eng.cells_valid()
    assert eng.regrid()
    assert eng.status() == 0 and eng.cells_valid()
    assert list(eng.ncell) == [7, 6, 6]
    ref = sb.MDEngine(eng.gather("x").cpu().numpy(), np.zeros(len(x), np.int32), [oin.W_MASS], eng.box_matrix(),
                      4.4, 0.5, device=DEV)
    a, _ = eng.half_list(4.9 ** 2)
    b, _ = ref.half_list(4.9 ** 2)
    pa = set(zip(a[0].tolist(), a[1].tolist()))
    pb = set(zip(b[0].tolist(), b[1].tolist()))
    assert pa == pb and len(pa) > 0
    # the loader regrids by itself
    eng2 = sb.MDEngine(x, np.zeros(len(x), np.int32), [oin.W_MASS], np.diag([L] * 3), 4.4, 0.5, device=DEV)

    class Mol:
        engine = eng2
    loader = UniaxialTensileLoader(Mol(), axis=0, strain_rate=50.0, lateral_mode="poisson", poisson_ratio=0.3,
                                   max_lateral_scale_step=0.05)
    for _ in range(10):
        loader.step(0.002)
    assert loader.regrids >= 1 and eng2.cells_valid() and eng2.status() == 0


def test_indenter_backbone_matches_reference(sb, tmp_path):
    """LJ (FP64) + SphericalIndenterForce as a second backbone, centre moved
    every step: energies, virial (trace and upper triangle of the reference's
    F (x) x tensor), force on the indenter, contacts and the final state."""
    from simulon_b200.mechanics import SphericalIndenterForce
    g = _golden("ind_ar108_f64")
    torch.set_default_dtype(torch.float64)
    try:
        path = oin.write_xyz(str(tmp_path / "ar.xyz"), g["x0"], "Ar")
        mol = sb.AtomFileReader(path, float(g["box0"]), 7.0, device=DEV,
                                parameter={"[0 0]": {"epsilon": 0.0104, "sigma": 3.405}}, skin_thickness=0.5)
        integ = sb.VerletIntegrator(mol, dt=float(g["dt"]), ensemble="NVE")
        mol.atom_velocities = torch.tensor(g["v0"], device=DEV)
        ind = SphericalIndenterForce(mol, radius=float(g["radius"]), stiffness=float(g["stiffness"]),
                                     center=g["center"][0])
        model = sb.BaseModel(sb.SumBackboneInterface([sb.LennardJonesForce(mol), ind], mol), integ, mol)
        E, V, W, Fi, n, Ei = [], [], [], [], [], []
        for s in range(int(g["steps"])):
            ind.set_center(g["center"][s])
            out = model()
            E.append(float(out["energy"]))
            V.append(float(out["virial"]))
            W.append(out["virial_tensor"].cpu().numpy())
            Fi.append(ind.force_on_indenter.cpu().numpy().copy())
            Ei.append(float(ind.last_energy))
            n.append(ind.contact_atoms)
        np.testing.assert_allclose(E, g["energy"], rtol=1e-9)
        np.testing.assert_allclose(V, g["virial"], rtol=1e-9, atol=1e-12)
        iu = np.triu_indices(3)
        np.testing.assert_allclose(np.array(W)[:, iu[0], iu[1]], g["virial_tensor"][:, iu[0], iu[1]], rtol=1e-8,
                                   atol=1e-12)
        np.testing.assert_allclose(np.array(Fi), g["force_on_indenter"], rtol=1e-8, atol=1e-13)
        np.testing.assert_allclose(Ei, g["indenter_energy"], rtol=1e-8, atol=1e-15)
        assert n == list(g["contact_atoms"])
        np.testing.assert_allclose(mol.coordinates.cpu().numpy(), g["x"], atol=1e-8)
        np.testing.assert_allclose(mol.atom_velocities.cpu().numpy(), g["v"], atol=1e-7)
        assert mol.engine.status() == 0
    finally:
        torch.set_default_dtype(torch.float32)


def test_indenter_alone_and_with_eam_in_graphs(sb, tmp_path):
    """The indenter as the only backbone (forces against the FP64
    restatement), and EAM + indenter stepped eagerly and through CUDA graphs
    with the centre changed between replays (the indenter inside EAM pass 2)
    and by the separate kernels: identical states."""
    from oracle.integrator import indenter
    from simulon_b200.mechanics import SphericalIndenterForce
    x, L = oin.bcc_lattice(6)
    x = oin.jitter(x, 0.05, 9)
    c = np.array([0.5 * L, 0.5 * L, float(x[:, 2].max()) + 1.5])
    eng = sb.MDEngine(x, np.zeros(len(x), np.int32), [oin.W_MASS], np.diag([L] * 3), 4.4, 0.5, device=DEV)

    class Mol:
        engine = eng
        device = DEV
        dtype = torch.float64
    ind = SphericalIndenterForce(Mol(), radius=3.0, stiffness=1.0, center=c)
    ind.compute()
    o = indenter(torch.tensor(x), c, 3.0, 1.0)
    np.testing.assert_allclose(eng.gather("f").cpu().numpy(), o["forces"].numpy(), rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(float(eng.potential_energy()), float(o["energy"]), rtol=1e-12)
    assert ind.contact_atoms == o["contact_atoms"] > 0
    from oracle import inputs as oi
    pot = oi.write_fs_w_setfl(str(tmp_path / "W.eam.fs"))
    parser = sb.EAMParser(pot)
    res = []
    # eager model steps and graph runs (both with the indenter inside EAM pass
    # 2), and the separate kernels: force field, indenter, integrator halves
    for mode in ("eager", "graph", "separate"):
        p = oi.write_xyz(str(tmp_path / f"w_{mode}.xyz"), x, "W")
        mol = sb.AtomFileReader(p, L, parser.cutoff, device=DEV, skin_thickness=0.5, is_fs=True)
        mol.atom_velocities = torch.tensor(oi.maxwell_boltzmann(np.full(len(x), oi.W_MASS), 300.0, 4), device=DEV)
        integ = sb.VerletIntegrator(mol, dt=0.002, ensemble="NVE")
        ind = SphericalIndenterForce(mol, radius=3.0, stiffness=1.0, center=c)
        ff = sb.EAMForceCUDAExt(parser, mol)
        model = sb.BaseModel(sb.SumBackboneInterface([ff, ind], mol), integ, mol)
        eng = mol.engine
        if mode == "separate":
            model.sum_bone.compute()
        for chunk in range(4):
            ind.set_center(c - np.array([0.0, 0.0, 0.1 * chunk]))
            if mode == "graph":
                model.run(5, graph_steps=5)
            elif mode == "eager":
                for _ in range(5):
                    model()
            else:
                for _ in range(5):
                    eng.integrate_first(integ.params, 0)
                    eng.rebuild_if_needed()
                    eng.eam_forces(ff.tables)
                    ind.add_to_engine(0)
                    eng.integrate_second(integ.params, 0)
                    eng.log_step()
        torch.cuda.synchronize()
        res.append((mol.coordinates.cpu(), mol.atom_velocities.cpu(), ind.out.cpu(), eng.red_out.cpu()))
        assert eng.status() == 0
    assert torch.equal(res[0][0], res[1][0]) and torch.equal(res[0][1], res[1][1])
    assert torch.equal(res[0][2], res[1][2]) and res[0][2][4] > 0
    assert torch.equal(res[0][0], res[2][0]) and torch.equal(res[0][1], res[2][1])
    np.testing.assert_allclose(res[0][2].numpy(), res[2][2].numpy(), rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(res[0][3].numpy()[:10], res[2][3].numpy()[:10], rtol=1e-6, atol=1e-6)
