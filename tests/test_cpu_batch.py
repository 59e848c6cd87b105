"""Host-side logic of the batched form, on CPU: slot/cell layout, the
longest-processing-time partition of replicas over ranks, the crack-slab
geometry (precrack, grips), and the end-of-run gather of per-replica results
across ranks over gloo (world size 2, no GPU)."""
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from simulon_b200.batch import crack_slab, crack_sweep, gather_replica_table, partition_replicas, plan_batch


def test_plan_batch_layout():
    sizes = [1, 31, 32, 33, 2000, 250]
    boxes = [np.diag([20.0 + k, 21.0, 22.0]) for k in range(len(sizes))]
    p = plan_batch(sizes, boxes, 4.9)
    assert np.all(p.off % 32 == 0) and np.all(p.n_slots % 32 == 0) and np.all(p.n_slots >= p.n)
    assert np.all(p.n_slots - p.n < 32)
    assert np.all(np.diff(p.off) == p.n_slots[:-1])
    assert p.total_slots == p.off[-1] + p.n_slots[-1] and p.n_pad % 128 == 0 and p.n_pad >= p.total_slots
    assert list(p.first) == list(np.cumsum([0] + sizes[:-1]))
    assert np.all(np.diff(p.cell_off) == p.n_cells[:-1] + 1)
    assert p.n_cell_entries == int((p.n_cells + 1).sum())
    with pytest.raises(ValueError):
        plan_batch([5, 0], boxes[:2], 4.9)


def test_partition_replicas_lpt():
    rng = np.random.default_rng(4)
    sizes = np.exp(rng.uniform(np.log(2000), np.log(250000), 48)).astype(int)
    for ranks in (1, 2, 3, 8):
        parts = partition_replicas(sizes, ranks)
        assert sorted(i for p in parts for i in p) == list(range(48))
        loads = [int(sizes[p].sum()) for p in parts]
        # LPT guarantee: no rank exceeds the mean load by more than the largest replica
        assert max(loads) <= sizes.sum() / ranks + sizes.max()
        assert all(p == sorted(p) for p in parts)
    assert partition_replicas([5, 4, 3], 5)[3:] == [[], []]


def test_crack_slab_geometry():
    r = crack_slab(2000, temperature=600.0, grip_rate=1e-4, seed=2)
    a = 3.165
    nx, ny, nz = r.meta["cells"]
    assert r.meta["removed"] > 0 and len(r.positions) == 2 * nx * ny * nz - r.meta["removed"]
    H = np.asarray(r.H)
    assert H[1, 1] > ny * a + 10.0                      # vacuum gap: open along y
    y = r.positions[:, 1]
    for code, layers in ((1, np.unique(np.round(y[r.grip == 1], 6))), (2, np.unique(np.round(y[r.grip == 2], 6)))):
        assert len(layers) == 3, (code, layers)
    assert np.all(r.velocities[r.grip != 0] == 0.0)
    free = r.grip == 0
    assert np.abs(r.velocities[free].mean(axis=0)).max() < 1e-12
    # no atom within 1.5 A of the crack plane over the central quarter of x
    xc = 0.5 * (r.positions[:, 0].min() + r.positions[:, 0].max())
    yc = 0.5 * (y.min() + y.max())
    plane = y[np.argmin(np.abs(y - yc))]
    gap = (np.abs(r.positions[:, 0] - xc) <= nx * a / 8.0) & (np.abs(y - plane) <= 1.5)
    assert not gap.any()


def test_crack_sweep_sizes_and_temperatures():
    reps = crack_sweep(12, n_min=2000, n_max=40000, seed=1)
    n = np.array([len(r.positions) for r in reps])
    assert n.min() > 1000 and n.max() < 60000
    assert np.allclose([r.temperature for r in reps], np.linspace(50.0, 1200.0, 12))


def _gather_worker(rank, world, port, sizes, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = partition_replicas(sizes, world)[rank]
        rows = torch.tensor([[k, 10.0 * k + rank, sizes[k]] for k in mine], dtype=torch.float64).reshape(-1, 3)
        table = gather_replica_table(mine, rows, len(sizes))
        torch.save(table, os.path.join(out_dir, f"table{rank}.pt"))
    finally:
        dist.destroy_process_group()


def test_gather_replica_table_over_gloo(tmp_path):
    sizes = [9000, 2000, 150000, 40000, 3000, 70000, 12000]
    port = 29500 + (os.getpid() % 1000)
    mp.spawn(_gather_worker, args=(2, port, sizes, str(tmp_path)), nprocs=2, join=True)
    parts = partition_replicas(sizes, 2)
    owner = {k: r for r, p in enumerate(parts) for k in p}
    for rank in range(2):
        t = torch.load(tmp_path / f"table{rank}.pt")
        assert t.shape == (len(sizes), 3)
        for k in range(len(sizes)):
            assert t[k, 0] == k and t[k, 1] == 10.0 * k + owner[k] and t[k, 2] == sizes[k]
