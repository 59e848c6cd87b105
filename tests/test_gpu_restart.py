"""Checkpoint/restart (io_utils/restart.py layout) and the simulator's output
files (md_simulation.py formats) on the device state."""
import os

import numpy as np
import pytest
import torch

from oracle import inputs as oin

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")


@pytest.fixture(scope="module")
def sb():
    import simulon_b200
    simulon_b200._lib.load()
    return simulon_b200


def _lj_model(sb, tmp_path, x, L, v, seed=3):
    path = oin.write_xyz(str(tmp_path / "ar.xyz"), x, "Ar")
    mol = sb.AtomFileReader(path, L, 7.0, device=DEV, parameter={"[0 0]": {"epsilon": 0.0104, "sigma": 3.405}},
                            skin_thickness=0.5)
    integ = sb.VerletIntegrator(mol, dt=0.002, ensemble="NVT", temperature=(94.4, 94.4), gamma=10.0, seed=seed)
    mol.atom_velocities = torch.tensor(v, device=DEV)
    return sb.BaseModel(sb.SumBackboneInterface([sb.LennardJonesForce(mol)], mol), integ, mol), mol


def test_restart_continues_the_run(sb, tmp_path):
    """10 Langevin steps, checkpoint, 10 more; a fresh model restored from the
    checkpoint runs the same 10 steps (same Philox noise) to the same state."""
    from simulon_b200.restart import load_checkpoint, save_checkpoint
    torch.set_default_dtype(torch.float64)
    try:
        x, L = oin.fcc_lattice(3)
        x = oin.jitter(x, 0.05, 0)
        v = oin.maxwell_boltzmann(np.full(len(x), oin.AR_MASS), 94.4, 1)
        model, mol = _lj_model(sb, tmp_path, x, L, v)
        for _ in range(10):
            model()
        ck = str(tmp_path / "restart.pt")
        save_checkpoint(model, 9, ck)
        for _ in range(10):
            model()
        xa, va = mol.coordinates.cpu().numpy(), mol.atom_velocities.cpu().numpy()
        ckpt = torch.load(ck, map_location="cpu", weights_only=True)
        for k in ("step", "coordinates", "velocities", "box_H", "rng_cpu", "rng_cuda", "force_cache",
                  "energy_cache", "virial_cache"):
            assert k in ckpt, k
        assert ckpt["coordinates"].shape == (108, 3) and ckpt["coordinates"].dtype == torch.float64
        model2, mol2 = _lj_model(sb, tmp_path, oin.jitter(x, 0.3, 9), L, np.zeros_like(v))
        assert load_checkpoint(model2, ck) == 10
        for _ in range(10):
            model2()
        np.testing.assert_allclose(mol2.coordinates.cpu().numpy(), xa, atol=1e-9)
        np.testing.assert_allclose(mol2.atom_velocities.cpu().numpy(), va, atol=1e-8)
    finally:
        torch.set_default_dtype(torch.float32)


def test_restart_reads_box_length_layout(sb, tmp_path):
    """A checkpoint in the reference's layout for a molecular without a Box
    (key 'box_length' instead of 'box_H', io_utils/restart.py:55-58) restores
    a cubic box of that side along with the positions."""
    from simulon_b200.restart import load_checkpoint, save_checkpoint
    torch.set_default_dtype(torch.float64)
    try:
        x, L = oin.fcc_lattice(3)
        x = oin.jitter(x, 0.05, 0)
        v = oin.maxwell_boltzmann(np.full(len(x), oin.AR_MASS), 94.4, 1)
        model, mol = _lj_model(sb, tmp_path, x, L, v)
        model()
        ck = str(tmp_path / "restart.pt")
        save_checkpoint(model, 0, ck)
        ckpt = torch.load(ck, map_location="cpu", weights_only=True)
        del ckpt["box_H"]
        ckpt["box_length"] = 1.02 * L
        torch.save(ckpt, ck)
        model2, mol2 = _lj_model(sb, tmp_path, x, L, np.zeros_like(v))
        assert load_checkpoint(model2, ck) == 1
        np.testing.assert_allclose(model2.engine.box_matrix(), np.diag([1.02 * L] * 3), rtol=1e-14, atol=0)
        np.testing.assert_array_equal(mol2.coordinates.cpu().numpy(), ckpt["coordinates"].numpy())
        model2()
        assert model2.engine.status() == 0
    finally:
        torch.set_default_dtype(torch.float32)


def test_simulator_output_files(sb, tmp_path):
    """traj.xyz every 5 steps, energies.csv every step, forces every 10, over
    a 20-step graph-captured run: contents equal the device log and state."""
    x, L = oin.bcc_lattice(5)
    x = oin.jitter(x, 0.05, 3)
    pot = oin.write_fs_w_setfl(str(tmp_path / "W.eam.fs"))
    parser = sb.EAMParser(pot)
    mol = sb.AtomFileReader(oin.write_xyz(str(tmp_path / "w.xyz"), x, "W"), L, parser.cutoff, device=DEV,
                            skin_thickness=0.5, is_fs=True)
    mol.atom_velocities = torch.tensor(oin.maxwell_boltzmann(np.full(len(x), oin.W_MASS), 300.0, 4), device=DEV)
    integ = sb.VerletIntegrator(mol, dt=0.002, ensemble="NVE")
    model = sb.BaseModel(sb.SumBackboneInterface([sb.EAMForceCUDAExt(parser, mol)], mol), integ, mol)
    out = tmp_path / "out"
    sim = sb.MDSimulator(model, 20, print_interval=10, store_outputs=False, verbose=False, output_dir=str(out),
                         traj_interval=5, write_energies=True, write_forces=True, forces_interval=10)
    sim.run()
    lines = open(out / "traj.xyz").read().splitlines()
    assert len(lines) == 4 * (250 + 2)
    assert lines[1].startswith("Step 5, Energy = ") and lines[-251].startswith("Step 20, Energy = ")
    last = np.array([[float(t) for t in ln.split()[1:]] for ln in lines[-250:]])
    np.testing.assert_allclose(last, mol.coordinates.cpu().numpy(), atol=1e-6)
    rows = np.loadtxt(out / "energies.csv", delimiter=",", skiprows=1)
    assert rows.shape == (20, 5) and list(rows[:, 0]) == list(range(1, 21))
    log = model.step_log(model.steps_done - 20, 20).cpu().numpy()
    np.testing.assert_allclose(rows[:, 1], log[:, 0] + log[:, 1], rtol=1e-8)
    np.testing.assert_allclose(rows[:, 2], log[:, 9], rtol=1e-8)
    assert abs(float(lines[-251].split("=")[1]) - (log[-1, 0] + log[-1, 1])) < 1e-5
    for s in (10, 20):
        f = torch.load(str(out / "forces" / f"forces_{s:06d}.pt"), weights_only=True)
        assert f.shape == (250, 3)
    f20 = torch.load(str(out / "forces" / "forces_000020.pt"), weights_only=True)
    np.testing.assert_allclose(f20.numpy(), mol.engine.gather("f").cpu().numpy(), rtol=1e-6, atol=1e-7)
