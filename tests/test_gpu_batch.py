"""Batched replicas on the GPU (C ABI group 3) against the single-system
engine run on each replica alone.

Tolerances: forces and trajectories bit for bit (same kernels' arithmetic,
same list order); per-replica energies and virials within 1e-6 relative
or 1e-5 eV absolute (FP32 partial sums grouped differently; off-diagonal
virial terms cancel to near zero); grip atoms exactly at their prescribed
positions with zero velocity.
"""
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


@pytest.fixture(scope="module")
def fsw(sb, tmp_path_factory):
    path = oin.write_fs_w_setfl(str(tmp_path_factory.mktemp("pot") / "W_synthetic.eam.fs"))
    parser = sb.EAMParser(path)
    return parser, sb.EAMDeviceTables(parser, DEV)


def _replicas(sb, tri=False):
    from simulon_b200.batch import Replica
    reps = []
    for k, n in enumerate((5, 7, 6)):
        if tri and k == 1:
            x, H = oin.bcc_triclinic(n)
        else:
            x, L = oin.bcc_lattice(n)
            H = np.diag([L, L, L])
        x = oin.jitter(x, 0.06, 70 + k)
        v = oin.maxwell_boltzmann(np.full(len(x), oin.W_MASS), 400.0 + 300 * k, 80 + k)
        reps.append(Replica(positions=x, H=H, velocities=v, temperature=300.0 + 200 * k))
    return reps


def _single(sb, rp, parser, velocities=None):
    return sb.MDEngine(rp.positions, np.zeros(len(rp.positions), np.int32), [oin.W_MASS], rp.H, parser.cutoff,
                       0.5, velocities=velocities, device=DEV)


@pytest.mark.parametrize("tri", [False, True])
def test_batch_forces_match_single_engines(sb, fsw, tri):
    from simulon_b200.batch import BatchedEngine
    parser, tables = fsw
    reps = _replicas(sb, tri)
    be = BatchedEngine(reps, oin.W_MASS, parser.cutoff, 0.5, device=DEV)
    assert be.status() == 0
    be.eam_forces(tables)
    f = be.gather("f").cpu()
    x = be.gather("x").cpu()
    for k, rp in enumerate(reps):
        eng = _single(sb, rp, parser)
        eng.eam_forces(tables)
        sl = be.replica_slice(k)
        assert torch.equal(x[sl], eng.gather("x").cpu())
        assert torch.equal(f[sl], eng.gather("f").cpu()), k
        red = eng.red_out.cpu().numpy()
        np.testing.assert_allclose(be.rep_red[k].cpu().numpy()[:9], red[:9], rtol=1e-6, atol=1e-5)
    assert (be.rebuild_counts() == 1).all()


def _single_drift_run(eng, tables, integ, k):
    eng.integrate_first(integ, 0)
    eng.rebuild_if_needed()
    for s in range(k):
        if s < k - 1:
            eng.eam_forces_integrate_drift(tables, integ)
            eng.rebuild_if_needed()
        else:
            eng.eam_forces_integrate(tables, integ)


def test_batch_nve_trajectory_matches_single_engines_at_scale(sb, fsw):
    """A 351,232-atom replica (each thread of the persistent batched passes
    takes two or three atoms) next to a 250-atom one: 30 NVE steps in
    graphs of 10, positions and velocities bit for bit against the single
    engine, so no pass of the batch sees atoms that its own epilogue moved."""
    from simulon_b200.batch import BatchedEngine, Replica
    from simulon_b200.engine import integrator_params
    parser, tables = fsw
    reps = []
    for k, n in enumerate((56, 5)):
        x, L = oin.bcc_lattice(n)
        x = oin.jitter(x, 0.06, 170 + k)
        v = oin.maxwell_boltzmann(np.full(len(x), oin.W_MASS), 600.0, 180 + k)
        reps.append(Replica(positions=x, H=np.diag([L] * 3), velocities=v, temperature=600.0))
    be = BatchedEngine(reps, oin.W_MASS, parser.cutoff, 0.5, device=DEV)
    integ = be.integrator(0.002, langevin=False)
    be.run(tables, integ, 30, graph_steps=10)
    torch.cuda.synchronize()
    assert be.status() == 0
    xb, vb = be.gather("x").cpu(), be.gather("v").cpu()
    for k, rp in enumerate(reps):
        eng = _single(sb, rp, parser, rp.velocities)
        ip = integrator_params(eng, 0.002)
        eng.eam_forces(tables)
        for _ in range(3):
            _single_drift_run(eng, tables, ip, 10)
        sl = be.replica_slice(k)
        assert torch.equal(xb[sl], eng.gather("x").cpu()), k
        assert torch.equal(vb[sl], eng.gather("v").cpu()), k


def test_batch_nve_trajectory_matches_single_engines(sb, fsw):
    from simulon_b200.batch import BatchedEngine
    from simulon_b200.engine import integrator_params
    parser, tables = fsw
    reps = _replicas(sb)
    be = BatchedEngine(reps, oin.W_MASS, parser.cutoff, 0.5, device=DEV)
    integ = be.integrator(0.002, langevin=False)
    be.run(tables, integ, 60, graph_steps=20)
    torch.cuda.synchronize()
    assert be.status() == 0
    xb, vb = be.gather("x").cpu(), be.gather("v").cpu()
    assert int(be.step_ctr[0]) == 59
    for k, rp in enumerate(reps):
        eng = _single(sb, rp, parser, rp.velocities)
        ip = integrator_params(eng, 0.002)
        eng.eam_forces(tables)
        for _ in range(3):
            _single_drift_run(eng, tables, ip, 20)
        sl = be.replica_slice(k)
        assert torch.equal(xb[sl], eng.gather("x").cpu()), k
        assert torch.equal(vb[sl], eng.gather("v").cpu()), k
        assert int(be.rep_rebuilds[k]) == int(eng.flags[3])
        red = eng.red_out.cpu().numpy()
        np.testing.assert_allclose(be.rep_red[k].cpu().numpy()[:10], red[:10], rtol=1e-6, atol=1e-5)
        np.testing.assert_allclose(be.log[59 % be.log_capacity, k].cpu().numpy()[:10], red[:10], rtol=1e-6,
                                   atol=1e-5)


def test_batch_rebuilds_only_moving_replicas(sb, fsw):
    from simulon_b200.batch import BatchedEngine, Replica
    parser, tables = fsw
    xc, Lc = oin.bcc_lattice(6)                      # perfect lattice at rest
    xh, Lh = oin.bcc_lattice(6)
    vh = oin.maxwell_boltzmann(np.full(len(xh), oin.W_MASS), 3000.0, 91)
    reps = [Replica(positions=xc, H=np.diag([Lc] * 3), temperature=0.0),
            Replica(positions=xh, H=np.diag([Lh] * 3), velocities=vh, temperature=3000.0)]
    be = BatchedEngine(reps, oin.W_MASS, parser.cutoff, 0.5, device=DEV)
    integ = be.integrator(0.002, gamma=10.0, langevin=True, seed=3)
    be.run(tables, integ, 100, graph_steps=20)
    torch.cuda.synchronize()
    counts = be.rebuild_counts()
    assert counts[0] == 1 and counts[1] >= 2, counts
    x = be.gather("x").cpu().numpy()
    assert np.abs(x[be.replica_slice(0)] - xc).max() < 1e-4
    T = be.temperature().cpu().numpy()
    assert T[0] < 1e-6 and T[1] > 300.0


def test_batch_small_rebuild_rows_equal_full_rebuild(sb, fsw):
    """A rebuild of few atoms (they fit in one wave of the list kernel's warps)
    builds one row per warp; a rebuild of every replica builds the rows of a
    cell with one warp.  From the same positions both give the same slots and
    the same rows, bit for bit."""
    from simulon_b200.batch import BatchedEngine, Replica
    parser, tables = fsw
    reps = []
    for k, n in enumerate((7, 7, 7, 7, 5)):
        x, L = oin.bcc_lattice(n)
        x = oin.jitter(x, 0.06, 120 + k)
        v = oin.maxwell_boltzmann(np.full(len(x), oin.W_MASS), 600.0, 130 + k)
        reps.append(Replica(positions=x, H=np.diag([L] * 3), velocities=v, temperature=600.0))
    be = BatchedEngine(reps, oin.W_MASS, parser.cutoff, 0.5, device=DEV)
    be.run(tables, be.integrator(0.002, langevin=False), 20, graph_steps=20)   # off the loaded lattice
    torch.cuda.synchronize()
    small = len(reps) - 1
    o, ns = int(be.plan.off[small]), int(be.plan.n_slots[small])
    n_warps = 4 * min(-(-int(be.plan.n_cell_entries) // 4), 148 * 64)
    assert ns <= n_warps < sum(int(s) for s in be.plan.n_slots)   # one warp per row; a full rebuild per cell
    before = be.rebuild_counts().copy()
    be.rep_flags.zero_()
    be.rep_flags[small] = 1
    be.rebuild(only_flagged=True)
    torch.cuda.synchronize()
    assert (be.rebuild_counts() - before).tolist() == [0] * small + [1]
    orig1, n1, rows1 = be.orig[o:o + ns].clone(), be.nnbr[o:o + ns].clone(), be.nbr[:, o:o + ns].clone()
    be.rebuild(only_flagged=False)
    torch.cuda.synchronize()
    assert be.status() == 0
    assert torch.equal(be.orig[o:o + ns], orig1)
    assert torch.equal(be.nnbr[o:o + ns], n1) and int(n1.max()) > 0
    filled = torch.arange(rows1.shape[0], device=DEV)[:, None] < n1[None, :].long()
    assert torch.equal(be.nbr[:, o:o + ns][filled], rows1[filled])


def test_batch_grips_follow_the_opening(sb, fsw):
    from simulon_b200.batch import BatchedEngine, crack_slab
    parser, tables = fsw
    rate = 2e-3
    reps = [crack_slab(2000, temperature=300.0, grip_rate=rate, seed=5),
            crack_slab(3500, temperature=900.0, grip_rate=rate, seed=6)]
    be = BatchedEngine(reps, oin.W_MASS, parser.cutoff, 0.5, device=DEV)
    integ = be.integrator(0.001, gamma=10.0, langevin=True, seed=9)
    steps = 40
    be.run(tables, integ, steps, graph_steps=20)
    torch.cuda.synchronize()
    assert be.status() == 0
    x, v = be.gather("x").cpu().numpy(), be.gather("v").cpu().numpy()
    last = steps - 1
    for k, rp in enumerate(reps):
        sl = be.replica_slice(k)
        g = rp.grip
        shift = 0.5 * rate * (last + 1)
        lo, hi = g == 1, g == 2
        assert lo.sum() > 0 and hi.sum() > 0
        want = rp.positions.copy()
        want[lo, 1] -= shift
        want[hi, 1] += shift
        np.testing.assert_allclose(x[sl][lo | hi], want[lo | hi], rtol=0, atol=1e-12)
        assert np.all(v[sl][lo | hi] == 0.0)
        assert np.abs(v[sl][g == 0]).max() > 0.0


def test_batch_crack_run_matches_reference_grip_loop(sb, fsw):
    """Two crack slabs with grips in one batch against the reference's own
    grip loop (run_scripts/w_crack.py:384-394,456-471 with its pure-PyTorch
    EAM, VerletIntegrator and BaseModel; recorded by make_golden.py,
    group crack_md): NVE, dt 1 fs, opening 2e-3 A per step, 20 steps.  The
    reference lets grip atoms take the first half-kick and drift of a step
    and puts them back around each model() call, so during a force
    evaluation they sit up to F dt^2 / 2m (~3e-5 A) from where the batched
    engine holds them; with the reference integrating in FP32, free atoms
    agree within 5e-4 A and 5e-3 A/ps, grip atoms within 1e-5 A (FP32
    rounding of their prescribed positions), potential energies within 2e-5
    relative at every step."""
    from simulon_b200.batch import BatchedEngine, Replica
    parser, tables = fsw
    gold = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    gs = [dict(np.load(os.path.join(gold, f"crack_md_w{n}.npz"))) for n in (1200, 2000)]
    reps = [Replica(positions=g["x0"], H=g["H"], velocities=g["v0"], temperature=float(g["T"]), grip=g["grip"],
                    grip_axis=1, grip_rate=float(g["rate"])) for g in gs]
    be = BatchedEngine(reps, oin.W_MASS, parser.cutoff, 0.5, device=DEV)
    integ = be.integrator(float(gs[0]["dt"]), langevin=False)
    epot = []
    for _ in range(int(gs[0]["steps"])):
        be.run(tables, integ, 1, graph_steps=1)
        epot.append(be.potential_energy().cpu().numpy())
    assert be.status() == 0
    epot = np.array(epot)
    x, v = be.gather("x").cpu().numpy(), be.gather("v").cpu().numpy()
    for k, g in enumerate(gs):
        sl = be.replica_slice(k)
        free, held = g["grip"] == 0, g["grip"] != 0
        np.testing.assert_allclose(epot[:, k], g["epot"], rtol=2e-5)
        np.testing.assert_allclose(x[sl][free], g["x"][free], rtol=0, atol=5e-4)
        np.testing.assert_allclose(v[sl][free], g["v"][free], rtol=0, atol=5e-3)
        np.testing.assert_allclose(x[sl][held], g["x"][held], rtol=0, atol=1e-5)
        assert np.all(v[sl][held] == 0.0) and np.all(g["v"][held] == 0.0)
