"""Batched replicas: many independent EAM systems advanced together.

The reference runs a parameter sweep (temperatures, crack slabs) as one
``BaseModel`` loop per system (run_scripts/w_crack.py:433-440).  Here every
replica lives in one set of device arrays (C ABI group 3 of
include/simb200.h): replica k owns a slot range whose start and length are
multiples of 32, has its own box, cell grid, neighbour-list rebuild flag,
Langevin temperature and optional grips, and each kernel launch covers all
replicas.  A step is four launches plus a conditional rebuild of only the
replicas whose atoms moved more than skin/2, captured in CUDA graphs.

Replicas shard across GPUs without any per-step exchange:
``partition_replicas`` assigns them to ranks by longest-processing-time
bin packing and ``gather_replica_table`` collects per-replica results at the
end of a run.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._lib import SimBatch, SimRep
from .engine import KB_EV, MASS_TO_INTERNAL, DeviceStruct, cell_grid, estimate_capacity, make_box, morton_rank

SLOT_ALIGN = 32


@dataclass
class Replica:
    """One independent system.  positions/velocities [n,3] (A, A/ps); H rows
    are the box vectors; grip [n] 0 free, 1 lower grip, 2 upper grip."""
    positions: np.ndarray
    H: np.ndarray
    velocities: np.ndarray | None = None
    temperature: float = 0.0
    grip: np.ndarray | None = None
    grip_axis: int = -1
    grip_rate: float = 0.0          # total opening per step (A)
    meta: dict = field(default_factory=dict)


@dataclass
class BatchPlan:
    """Slot and cell layout of a batch (host-side bookkeeping, no device)."""
    n: np.ndarray            # atoms per replica
    n_slots: np.ndarray      # n rounded up to SLOT_ALIGN
    off: np.ndarray          # first slot
    first: np.ndarray        # first original index
    ncell: np.ndarray        # [R,3]
    n_cells: np.ndarray
    cell_off: np.ndarray     # first cell entry (each replica has n_cells + 1 entries)
    total_slots: int
    n_pad: int
    n_cell_entries: int


def plan_batch(sizes, boxes, list_cutoff: float) -> BatchPlan:
    sizes = np.asarray(sizes, dtype=np.int64)
    if len(sizes) == 0 or np.any(sizes < 1):
        raise ValueError("every replica needs at least one atom")
    n_slots = ((sizes + SLOT_ALIGN - 1) // SLOT_ALIGN) * SLOT_ALIGN
    off = np.concatenate([[0], np.cumsum(n_slots)[:-1]]).astype(np.int64)
    first = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    ncell = np.stack([cell_grid(H, list_cutoff, int(n)) for H, n in zip(boxes, sizes)]).astype(np.int32)
    n_cells = ncell.prod(axis=1).astype(np.int64)
    cell_off = np.concatenate([[0], np.cumsum(n_cells + 1)[:-1]]).astype(np.int64)
    total = int(n_slots.sum())
    n_pad = ((total + 127) // 128) * 128
    return BatchPlan(sizes, n_slots, off, first, ncell, n_cells, cell_off, total, n_pad, int((n_cells + 1).sum()))


def partition_replicas(sizes, n_ranks: int) -> list[list[int]]:
    """Longest-processing-time bin packing of replicas (by atom count) onto
    ranks; each rank's list keeps the replicas' original order."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    load = [0] * n_ranks
    parts: list[list[int]] = [[] for _ in range(n_ranks)]
    for k in sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i)):
        r = min(range(n_ranks), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += int(sizes[k])
    return [sorted(p) for p in parts]


def gather_replica_table(local_ids, local_rows: torch.Tensor, n_total: int, group=None) -> torch.Tensor:
    """End-of-run collection over torch.distributed: every rank contributes the
    rows of its replicas; returns the [n_total, cols] table on every rank."""
    import torch.distributed as dist
    rows = local_rows.detach().to("cpu", torch.float64)
    cols = rows.shape[1]
    out = torch.zeros(n_total, cols, dtype=torch.float64)
    if not (dist.is_available() and dist.is_initialized()):
        out[list(local_ids)] = rows
        return out
    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, (list(local_ids), rows), group=group)
    for ids, r in parts:
        if len(ids):
            out[ids] = r
    return out


class BatchedEngine:
    """Device state of a batch of single-element EAM replicas."""

    def __init__(self, replicas: list[Replica], mass_amu: float, cutoff: float, skin: float, *, device=None,
                 nbr_cap: int | None = None, log_capacity: int = 1024):
        self.lib = _lib.load()
        self.device = torch.device(device or "cuda")
        if self.device.type != "cuda":
            raise RuntimeError("BatchedEngine runs on CUDA devices only (no CPU fallback)")
        self.replicas = list(replicas)
        R = len(self.replicas)
        self.n_rep = R
        self.cutoff, self.skin = float(cutoff), float(skin)
        self.x_rc = self.cutoff + self.skin
        boxes = [np.asarray(r.H, np.float64).reshape(3, 3) for r in self.replicas]
        for k, H in enumerate(boxes):
            if np.any(np.diag(H) <= 0):
                raise ValueError(f"replica {k}: box diagonal must be positive")
        sizes = [len(r.positions) for r in self.replicas]
        self.plan = plan = plan_batch(sizes, boxes, self.x_rc)
        self.n_atoms = int(plan.n.sum())
        self.nbr_cap = int(nbr_cap or max(estimate_capacity(int(n), H, self.x_rc) for n, H in zip(sizes, boxes)))
        dev, P = self.device, plan.n_pad
        f64 = dict(device=dev, dtype=torch.float64)
        i32 = dict(device=dev, dtype=torch.int32)
        self.mass_internal = float(mass_amu) * MASS_TO_INTERNAL
        # slot arrays
        self.x = torch.zeros(3, P, **f64)
        self.v = torch.zeros(3, P, **f64)
        self.f32 = torch.zeros(P, 4, device=dev, dtype=torch.float32)
        self.posq = torch.zeros(P, 4, **i32)
        self.xref = torch.zeros(3, P, **i32)
        self.orig = torch.zeros(P, **i32)
        self.posfp = torch.zeros(P, 4, **i32)
        self.nbr = torch.zeros(self.nbr_cap, P, **i32)
        self.nnbr = torch.zeros(P, **i32)
        self.cut_mask = torch.zeros(P, device=dev, dtype=torch.int64) if self.nbr_cap <= 64 else None
        self.cell_of = torch.zeros(P, **i32)
        self.cell_count = torch.zeros(plan.n_cell_entries, **i32)
        self.cell_start = torch.zeros(plan.n_cell_entries, **i32)
        ranks = np.zeros(2 * plan.n_cell_entries, np.int32)
        cell_rep = np.zeros(plan.n_cell_entries, np.int32)
        for k in range(R):
            r, lin = morton_rank(plan.ncell[k])
            c0, nc = int(plan.cell_off[k]), int(plan.n_cells[k])
            ranks[2 * c0:2 * c0 + nc] = r
            ranks[2 * c0 + nc:2 * c0 + 2 * nc] = lin
            cell_rep[c0:c0 + nc + 1] = k
        self.cell_rank = torch.from_numpy(ranks).to(dev)
        self.cell_rep = torch.from_numpy(cell_rep).to(dev)
        self.perm = torch.zeros(P, **i32)
        self.x_alt = torch.zeros(3, P, **f64)
        self.v_alt = torch.zeros(3, P, **f64)
        self.f32_alt = torch.zeros(P, 4, device=dev, dtype=torch.float32)
        self.orig_alt = torch.zeros(P, **i32)
        self.mass = torch.tensor([self.mass_internal], **f64)
        self.inv_mass = 1.0 / self.mass
        self.flags = torch.zeros(8, **i32)
        self.partials = torch.zeros(16, **f64)
        self.red_counter = torch.zeros(4, **i32)
        self.red_out = torch.zeros(_lib.RED_SLOTS, **f64)
        slot_rep = np.full(P, -R, np.int32)          # slots past the last replica: its padding
        for k in range(R):
            o, ns, n = int(plan.off[k]), int(plan.n_slots[k]), int(plan.n[k])
            slot_rep[o:o + n] = k
            slot_rep[o + n:o + ns] = -1 - k
        self.slot_rep = torch.from_numpy(slot_rep).to(dev)
        self.rep_flags = torch.zeros(R, **i32)
        self.rep_rebuilds = torch.zeros(R, **i32)
        self.work = torch.zeros(3 * (R + 1), **i32)
        grip = np.zeros(self.n_atoms, np.int8)
        gref = np.zeros((3, P), np.float64)
        for k, rp in enumerate(self.replicas):
            a0 = int(plan.first[k])
            if rp.grip is not None:
                grip[a0:a0 + len(rp.positions)] = np.asarray(rp.grip, np.int8)
            gref[:, a0:a0 + len(rp.positions)] = np.asarray(rp.positions, np.float64).T
        self.grip = torch.from_numpy(grip).to(dev)
        self.gref = torch.from_numpy(gref).to(dev)
        self.temperatures = np.array([float(r.temperature) for r in self.replicas])
        self.rep_rff = torch.zeros(R, **f64)
        self.chunk_red = torch.zeros(P // SLOT_ALIGN + _lib.SIM_BATCH_RED_SPLIT * R, _lib.RED_SLOTS, **f64)
        self.rep_red = torch.zeros(R, _lib.RED_SLOTS, **f64)
        self.step_ctr = torch.full((2,), -1, device=dev, dtype=torch.int64)
        self.log_capacity = int(log_capacity)
        self.log = torch.zeros(self.log_capacity, R, _lib.RED_SLOTS, **f64)
        reps = (SimRep * R)()
        self.box_orthogonal = True
        for k, rp in enumerate(self.replicas):
            s = reps[k]
            s.box = make_box(boxes[k])
            self.box_orthogonal &= bool(s.box.orthogonal)
            s.off, s.first = int(plan.off[k]), int(plan.first[k])
            s.n, s.n_slots = int(plan.n[k]), int(plan.n_slots[k])
            s.ncell[:] = [int(v) for v in plan.ncell[k]]
            s.n_cells, s.cell_off = int(plan.n_cells[k]), int(plan.cell_off[k])
            s.grip_axis = int(rp.grip_axis) if rp.grip is not None else -1
            s.grip_rate = float(rp.grip_rate)
        self.rep_dev = torch.frombuffer(bytearray(bytes(reps)), dtype=torch.uint8).to(dev)
        self._make_struct()
        xs = np.concatenate([np.asarray(r.positions, np.float64) for r in self.replicas])
        vs = np.concatenate([np.zeros((len(r.positions), 3)) if r.velocities is None
                             else np.asarray(r.velocities, np.float64) for r in self.replicas])
        self.types = torch.zeros(self.n_atoms, **i32)
        xs_d, vs_d = torch.from_numpy(xs).to(dev), torch.from_numpy(vs).to(dev)   # alive until the load ran
        _lib.call("sim_batch_load", self.ref, _lib.ptr(xs_d), _lib.ptr(vs_d), _lib.ptr(self.types), self.stream)
        torch.cuda.synchronize(dev)
        del xs_d, vs_d
        self.forces_valid = False
        self._graphs = {}
        self.check_capacity()

    # ---- struct plumbing -------------------------------------------------
    def _make_struct(self):
        b = SimBatch()
        e = b.e
        plan = self.plan
        e.n, e.n_pad, e.n_types, e.nbr_cap = plan.total_slots, plan.n_pad, 1, self.nbr_cap
        e.x_rc = self.x_rc
        e.skin_half2 = (self.skin / 2.0) ** 2
        p = _lib.ptr
        e.box = p(self.rep_dev)            # replica 0's box; the batch kernels use each replica's
        for name in ("x", "v", "f32", "posq", "xref", "orig", "posfp", "nbr", "nnbr", "cell_of", "cell_count",
                     "cell_start", "cell_rank", "perm", "x_alt", "v_alt", "f32_alt", "orig_alt", "inv_mass", "mass",
                     "flags", "partials", "red_counter", "red_out", "cut_mask"):
            setattr(e, name, p(getattr(self, name)))
        e.n_blocks_max = 1
        e.box_orthogonal = int(self.box_orthogonal)
        b.rep = p(self.rep_dev)
        b.n_rep, b.n_cell_entries = self.n_rep, plan.n_cell_entries
        for name in ("slot_rep", "cell_rep", "rep_flags", "rep_rebuilds", "work", "grip", "gref", "rep_rff",
                     "chunk_red", "rep_red"):
            setattr(b, name, p(getattr(self, name)))
        self.st = b
        self.ref = ctypes.byref(b)

    @property
    def stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def check_capacity(self):
        """Grow the list if a rebuild overflowed it (synchronises)."""
        for _ in range(3):
            flags = self.flags.cpu()
            if not int(flags[1]) & _lib.SIM_STATUS_OVERFLOW:
                return
            self.nbr_cap = int(math.ceil((int(flags[2]) * 1.15 + 8) / 8.0) * 8)
            self.nbr = torch.zeros(self.nbr_cap, self.plan.n_pad, device=self.device, dtype=torch.int32)
            self.cut_mask = (torch.zeros(self.plan.n_pad, device=self.device, dtype=torch.int64)
                             if self.nbr_cap <= 64 else None)
            self._graphs = {}
            self.flags.zero_()
            self._make_struct()
            _lib.call("sim_batch_rebuild", self.ref, 0, self.stream)
        raise _lib.SimError("neighbour list overflow persists after growing the capacity")

    # ---- primitives ------------------------------------------------------
    def rebuild(self, only_flagged: bool = True):
        _lib.call("sim_batch_rebuild", self.ref, int(only_flagged), self.stream)

    def eam_forces(self, tables):
        """Pass 1 + pass 2 (forces, energies, virials) for every replica, no integration."""
        _lib.call("sim_batch_eam_density", self.ref, tables.ref, self.stream)
        _lib.call("sim_batch_eam_force", self.ref, tables.ref, None, 0, self.stream)
        _lib.call("sim_batch_reduce", self.ref, None, None, 0, self.stream)
        self.forces_valid = True

    def integrator(self, dt: float, *, gamma: float = 0.0, langevin: bool = True, seed: int = 0) -> DeviceStruct:
        """SimIntegrator with per-replica Langevin amplitudes from each replica's
        temperature (integrator.py:45-88 per replica)."""
        s = _lib.SimIntegrator()
        s.dt = float(dt)
        s.langevin = int(langevin)
        if langevin:
            g = torch.tensor(float(gamma), dtype=torch.float64)
            s.damp = float(torch.exp(-g * dt))
            T = torch.tensor(self.temperatures, dtype=torch.float64)
            rff = torch.sqrt(KB_EV * T / self.mass_internal * (1.0 - torch.exp(-2.0 * g * dt)))
            self.rep_rff.copy_(rff.to(self.device))
        else:
            s.damp = 1.0
        s.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        s.step_ctr = _lib.ptr(self.step_ctr)
        return DeviceStruct(s, [])

    def _launch_steps(self, tables, integ, k: int):
        _lib.call("sim_batch_first_half", self.ref, integ.ref, self.stream)
        _lib.call("sim_batch_rebuild_if_needed", self.ref, self.stream)
        for s in range(k):
            _lib.call("sim_batched_step", self.ref, tables.ref, integ.ref, int(s == k - 1), _lib.ptr(self.log),
                      self.log_capacity, self.stream)

    def run(self, tables, integ, n_steps: int, graph_steps: int = 20):
        """Advance every replica n_steps (CUDA graphs of graph_steps steps, no host sync)."""
        if not self.forces_valid:
            self.eam_forces(tables)
        full, rest = divmod(int(n_steps), int(graph_steps))
        if full:
            key = (int(graph_steps), id(tables), id(integ))
            if key not in self._graphs:
                s = torch.cuda.Stream(self.device)
                s.wait_stream(torch.cuda.current_stream(self.device))
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=s):
                    self._launch_steps(tables, integ, int(graph_steps))
                torch.cuda.current_stream(self.device).wait_stream(s)
                self._graphs[key] = g
            for _ in range(full):
                self._graphs[key].replay()
        if rest:
            self._launch_steps(tables, integ, rest)

    # ---- results ---------------------------------------------------------
    def gather(self, which: str) -> torch.Tensor:
        """[atoms, 3] FP64 in original order (replica after replica): x, v or f."""
        out = torch.zeros(self.n_atoms, 3, device=self.device, dtype=torch.float64)
        if which == "f":
            _lib.call("sim_batch_gather_f32", self.ref, _lib.ptr(self.f32), _lib.ptr(out), self.stream)
        else:
            src = {"x": self.x, "v": self.v}[which]
            _lib.call("sim_batch_gather_f64", self.ref, _lib.ptr(src), _lib.ptr(out), self.stream)
        return out

    def replica_slice(self, k: int) -> slice:
        a = int(self.plan.first[k])
        return slice(a, a + int(self.plan.n[k]))

    def potential_energy(self) -> torch.Tensor:
        return self.rep_red[:, _lib.RED_EPOT_EMBED] + self.rep_red[:, _lib.RED_EPOT_PAIR]

    def kinetic_energy(self) -> torch.Tensor:
        return self.rep_red[:, _lib.RED_KE]

    def temperature(self) -> torch.Tensor:
        """2 K / (3 N kB) per replica, N counting every atom (integrator.py:116-124)."""
        n = torch.tensor(self.plan.n, dtype=torch.float64, device=self.device)
        return 2.0 * self.kinetic_energy() / (3.0 * n * KB_EV)

    def status(self) -> int:
        return int(self.flags[1].item())

    def rebuild_counts(self) -> np.ndarray:
        return self.rep_rebuilds.cpu().numpy()


# ---------------------------------------------------------------------------
# crack-slab replicas (run_scripts/w_crack.py:297-392 geometry)

def crack_slab(n_target: int, a: float = 3.165, *, vacuum: float = 15.0, crack_gap: float = 3.0,
               grip_layers: int = 3, temperature: float = 300.0, grip_rate: float = 1e-4, seed: int = 0) -> Replica:
    """BCC slab with cube axes along x, y, z: periodic in x and z, open in y (a
    vacuum gap added to the box), a centre through-thickness precrack made by
    deleting the atoms within crack_gap/2 of the atomic plane nearest the
    centre over a segment of length L_x/4 (w_crack.py:309-320), and grips of
    grip_layers atomic layers at the bottom and top (w_crack.py:346-353)."""
    nz = max(4, int(round((n_target / 8.0) ** (1.0 / 3.0))))
    nx = ny = 2 * nz
    base = np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.5]])
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    cells = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], axis=1).astype(np.float64)
    x = ((cells[:, None, :] + base[None, :, :]).reshape(-1, 3)) * a
    Lx, Ly, Lz = nx * a, ny * a, nz * a
    H = np.diag([Lx, Ly + vacuum, Lz])
    xc = 0.5 * (x[:, 0].min() + x[:, 0].max())
    yc_mid = 0.5 * (x[:, 1].min() + x[:, 1].max())
    y_plane = x[np.argmin(np.abs(x[:, 1] - yc_mid)), 1]
    crack = (np.abs(x[:, 1] - y_plane) <= 0.5 * crack_gap) & (np.abs(x[:, 0] - xc) <= Lx / 8.0)
    x = x[~crack]
    y0, y1 = x[:, 1].min(), x[:, 1].max()
    thick = (grip_layers - 0.5) * 0.5 * a
    grip = np.zeros(len(x), np.int8)
    grip[x[:, 1] <= y0 + thick] = 1
    grip[x[:, 1] >= y1 - thick] = 2
    rng = np.random.default_rng(seed)
    m = 183.84 * MASS_TO_INTERNAL
    v = rng.normal(0.0, math.sqrt(KB_EV * temperature / m), size=x.shape)
    v[grip != 0] = 0.0
    free = grip == 0
    v[free] -= v[free].mean(axis=0)
    return Replica(positions=x, H=H, velocities=v, temperature=temperature, grip=grip, grip_axis=1,
                   grip_rate=grip_rate, meta={"cells": (nx, ny, nz), "removed": int(crack.sum()),
                                              "crack_plane_y": float(y_plane), "crack_half_length": Lx / 8.0})


def crack_sweep(n_replicas: int = 48, n_min: int = 2000, n_max: int = 250000, t_min: float = 50.0,
                t_max: float = 1200.0, seed: int = 0, **kw) -> list[Replica]:
    """Replica sizes log-uniform in [n_min, n_max] (seeded), temperatures evenly
    spaced from t_min to t_max."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(n_min), math.log(n_max), size=n_replicas))
    temps = np.linspace(t_min, t_max, n_replicas)
    return [crack_slab(int(s), temperature=float(T), seed=seed + 1 + k, **kw)
            for k, (s, T) in enumerate(zip(sizes, temps))]


# ---------------------------------------------------------------------------
# crack observables (w_crack.py:113-188) on the device

def select_mouth_groups(vx, vy, x_center: float, y_center: float, crack_half_length: float):
    """Atoms at the crack mouth above and below the crack plane, in windows
    growing until both groups are non-empty (w_crack.py:125-133)."""
    mouth_x = x_center + crack_half_length
    for xw in (0.8, 1.2, 1.8, 2.5):
        for yw in (0.8, 1.2, 1.8, 2.5):
            near = np.abs(vx - mouth_x) <= xw
            upper = near & (vy > y_center) & ((vy - y_center) <= yw)
            lower = near & (vy < y_center) & ((y_center - vy) <= yw)
            if upper.any() and lower.any():
                return upper, lower
    raise ValueError("failed to find crack-mouth atoms; increase replicas or crack size")


class CrackObserver:
    """Per-replica crack-mouth opening, crack length and projected stress of a
    BatchedEngine, computed on the device (``sim_batch_crack_observe``) from
    the current positions and the last reduction, so a sweep needs no host
    round trip per step (the reference's script computes them on the host,
    w_crack.py:113-188, 474-496).  Set-up as the reference's: the lattice
    axes are the normalised box rows 0 and 1; the crack-axis range and centre
    and the mouth groups come from the reference positions (default: the
    engine's current ones), the opening is measured from their initial
    value.  Replicas without crack metadata (``crack_plane_y``,
    ``crack_half_length``) report only the stress."""

    COLUMNS = ("stress_bar", "native_stress_yy_bar", "cmod_A", "signed_cmod_A", "crack_length_A",
               "crack_extension_A", "open_bins", "reserved")

    def __init__(self, batch: "BatchedEngine", threshold: float = 1.0, bins: int = 160, reference_positions=None):
        self.batch = batch
        dev = batch.device
        x = (batch.gather("x") if reference_positions is None else torch.as_tensor(reference_positions))
        x = x.to(torch.float64).cpu().numpy()
        R = batch.n_rep
        table = (_lib.SimCrack * R)()
        mouth = np.zeros(batch.n_atoms, np.int8)
        off = 0
        self.initial_cmod = np.zeros(R)
        for k, rep in enumerate(batch.replicas):
            c = table[k]
            H = np.asarray(rep.H, np.float64)
            xu = H[0] / max(np.linalg.norm(H[0]), 1e-12)
            yu = H[1] / max(np.linalg.norm(H[1]), 1e-12)
            c.x_unit[:], c.y_unit[:] = xu.tolist(), yu.tolist()
            if "crack_plane_y" not in rep.meta or "crack_half_length" not in rep.meta:
                c.bins = 0
                continue
            sl = batch.replica_slice(k)
            xs = x[sl]
            vx, vy = xs @ xu, xs @ yu
            c.x_min, c.x_max = float(vx.min()), float(vx.max())
            c.x_center = 0.5 * (c.x_min + c.x_max)
            c.y_plane = float(rep.meta["crack_plane_y"])
            c.half_length = float(rep.meta["crack_half_length"])
            c.threshold = float(threshold)
            up, lo = select_mouth_groups(vx, vy, c.x_center, c.y_plane, c.half_length)
            c.initial_cmod = float(vy[up].mean() - vy[lo].mean())
            self.initial_cmod[k] = c.initial_cmod
            c.n_upper, c.n_lower = int(up.sum()), int(lo.sum())
            first = sl.start
            mouth[first + np.nonzero(up)[0]] = 1
            mouth[first + np.nonzero(lo)[0]] = 2
            c.bins = int(max(8, bins))
            c.bin_off = off
            off += c.bins
        self.total_bins = off
        raw = bytes(table)
        self.table = torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(dev)
        self.mouth = torch.from_numpy(mouth).to(dev)
        self.bins = torch.zeros(max(1, 2 * off), dtype=torch.int64, device=dev)
        self.sums = torch.zeros(2 * R, dtype=torch.float64, device=dev)
        self.out = torch.zeros(R, _lib.SIM_CRACK_OUT, dtype=torch.float64, device=dev)

    def observe(self) -> torch.Tensor:
        """[n_rep, 8] device tensor, columns ``COLUMNS`` (no synchronisation)."""
        b = self.batch
        _lib.call("sim_batch_crack_observe", b.ref, _lib.ptr(self.table), _lib.ptr(self.mouth), int(self.total_bins),
                  _lib.ptr(self.bins), _lib.ptr(self.sums), _lib.ptr(self.out), b.stream)
        return self.out
