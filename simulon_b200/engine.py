"""Device-resident MD state and the step primitives of libsimb200.

``MDEngine`` owns every device buffer the C ABI needs (the library allocates
nothing).  Atoms live in cell order ("slots"); the per-atom arrays are padded
to a multiple of 128.  Positions and velocities are FP64 structure-of-arrays;
the pair kernels gather 16-byte fixed-point fractional positions (posq) and
walk a full Verlet list in ELL layout.  All launches go to PyTorch's current
stream, so a step can be captured in a CUDA graph.

The cell grid is fixed when the engine is created: cells are at least
(rc + skin) wide perpendicular to each face and visited in Morton order, so
the neighbours of a slot are nearby slots and pair gathers hit L1/L2.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib

MASS_TO_INTERNAL = 10.0 / (6.02214076e23 * 1.60218e-19)   # amu -> eV ps^2 / A^2 (integrator.py:61-64)
KB_EV = 8.617333262e-5                                      # integrator.py:41
LOG_EXTRA = 2                                               # pressure (bar), mu
TILE = 1024                 # atoms per neighbour tile (SIM_TILE)
HALO_CAP_MAX = 4096         # largest halo the tiled kernels accept


def make_box(H) -> _lib.SimBox:
    """SimBox from a [3,3] matrix with rows = lattice vectors (core/box.py:39-57)."""
    H = np.asarray(H, dtype=np.float64).reshape(3, 3)
    b = _lib.SimBox()
    Hi = np.linalg.inv(H)
    off = H - np.diag(np.diag(H))
    b.H[:] = H.ravel().tolist()
    b.Hinv[:] = Hi.ravel().tolist()
    b.Hf[:] = H.astype(np.float32).ravel().tolist()
    b.orthogonal = int(np.allclose(off, 0.0, atol=1e-8))
    return b


def box_from_struct(b: _lib.SimBox) -> np.ndarray:
    return np.array(b.H[:], dtype=np.float64).reshape(3, 3)


def perpendicular_widths(H) -> np.ndarray:
    H = np.asarray(H, dtype=np.float64)
    V = abs(np.linalg.det(H))
    a, b, c = H
    return np.array([V / np.linalg.norm(np.cross(b, c)), V / np.linalg.norm(np.cross(c, a)),
                     V / np.linalg.norm(np.cross(a, b))])


def cell_grid(H, rc: float, n_atoms: int) -> np.ndarray:
    """Cells per axis: each at least rc wide (with a 1e-6 margin), total <= max(4N, 27)."""
    n = np.maximum(np.floor(perpendicular_widths(H) / (rc * (1.0 + 1e-6))), 1).astype(np.int64)
    limit = max(4 * n_atoms, 27)
    while n.prod() > limit:
        k = int(np.argmax(n))
        n[k] = max(1, n[k] // 2)
    return n.astype(np.int32)


def morton_rank(ncell) -> tuple[np.ndarray, np.ndarray]:
    """(rank of each linear cell, linear cell of each rank) for a Z-order walk."""
    nx, ny, nz = (int(v) for v in ncell)
    cz, cy, cx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    cx, cy, cz = (a.ravel().astype(np.uint64) for a in (cx, cy, cz))

    def spread(v):
        v = v & np.uint64(0x1FFFFF)
        v = (v | (v << np.uint64(32))) & np.uint64(0x1F00000000FFFF)
        v = (v | (v << np.uint64(16))) & np.uint64(0x1F0000FF0000FF)
        v = (v | (v << np.uint64(8))) & np.uint64(0x100F00F00F00F00F)
        v = (v | (v << np.uint64(4))) & np.uint64(0x10C30C30C30C30C3)
        v = (v | (v << np.uint64(2))) & np.uint64(0x1249249249249249)
        return v
    code = spread(cx) | (spread(cy) << np.uint64(1)) | (spread(cz) << np.uint64(2))
    lin_of_rank = np.argsort(code, kind="stable").astype(np.int32)
    rank_of_lin = np.empty_like(lin_of_rank)
    rank_of_lin[lin_of_rank] = np.arange(len(lin_of_rank), dtype=np.int32)
    return rank_of_lin, lin_of_rank


def estimate_capacity(n_atoms: int, H, rc: float) -> int:
    dens = n_atoms / abs(np.linalg.det(np.asarray(H, np.float64)))
    est = 4.0 / 3.0 * math.pi * rc ** 3 * dens
    cap = int(math.ceil((est * 1.35 + 16) / 8.0) * 8)
    return max(8, min(cap, ((n_atoms + 7) // 8) * 8))


class MDEngine:
    """Device state + C-ABI calls for one system.

    positions/velocities: [N,3] (any float dtype, any device), original atom order.
    types: [N] ints (element ids 0..n_types-1); masses_amu: [n_types].
    """

    def __init__(self, positions, types, masses_amu, H, cutoff: float, skin: float, *, velocities=None,
                 device=None, nbr_cap: int | None = None, fp64_forces: bool = False, log_capacity: int = 4096,
                 use_tiles: bool = False, halo_cap: int = 3072):
        self.lib = _lib.load()
        self.device = torch.device(device or "cuda")
        if self.device.type != "cuda":
            raise RuntimeError("MDEngine runs on CUDA devices only (no CPU fallback)")
        pos = torch.as_tensor(positions).to(self.device, torch.float64).contiguous()
        n = int(pos.shape[0])
        if n < 1:
            raise ValueError("engine needs at least one atom")
        self.n = n
        self.n_pad = ((n + 127) // 128) * 128
        self.cutoff = float(cutoff)
        self.skin = float(skin)
        self.x_rc = self.cutoff + self.skin
        self.H0 = np.asarray(H, dtype=np.float64).reshape(3, 3)
        self.box = make_box(self.H0)
        self.ncell = cell_grid(self.H0, self.x_rc, n)
        self.n_cells = int(np.prod(self.ncell))
        masses = np.asarray(masses_amu, dtype=np.float64).reshape(-1)
        self.n_types = len(masses)
        self.fp64_forces = bool(fp64_forces)
        self.nbr_cap = int(nbr_cap or estimate_capacity(n, self.H0, self.x_rc))
        dev, P = self.device, self.n_pad
        f64 = dict(device=dev, dtype=torch.float64)
        i32 = dict(device=dev, dtype=torch.int32)
        self.box_dev = torch.frombuffer(bytearray(bytes(self.box)), dtype=torch.uint8).to(dev)
        self.x = torch.zeros(3, P, **f64)
        self.v = torch.zeros(3, P, **f64)
        self.f32 = torch.zeros(P, 4, device=dev, dtype=torch.float32)
        self.f64 = torch.zeros(3, P, **f64) if self.fp64_forces else None
        self.posq = torch.zeros(P, 4, **i32)
        self.xref = torch.zeros(3, P, **i32)
        self.orig = torch.zeros(P, **i32)
        self.posfp = torch.zeros(P, 4, **i32)
        self.n_tiles = (n + TILE - 1) // TILE
        self.halo_cap = int(halo_cap)
        self.use_tiles = bool(use_tiles)
        self._alloc_lists()
        self.nnbr = torch.zeros(P, **i32)
        self.cell_of = torch.zeros(P, **i32)
        self.cell_count = torch.zeros(self.n_cells + 1, **i32)
        self.cell_start = torch.zeros(self.n_cells + 1, **i32)
        r, lin = morton_rank(self.ncell)
        self.cell_rank = torch.from_numpy(np.concatenate([r, lin])).to(dev)
        self.perm = torch.zeros(P, **i32)
        self.x_alt = torch.zeros(3, P, **f64)
        self.v_alt = torch.zeros(3, P, **f64)
        self.f32_alt = torch.zeros(P, 4, device=dev, dtype=torch.float32)
        self.f64_alt = torch.zeros(3, P, **f64) if self.fp64_forces else None
        self.orig_alt = torch.zeros(P, **i32)
        m_int = masses * MASS_TO_INTERNAL
        self.mass_amu = torch.tensor(masses, **f64)
        self.mass = torch.tensor(m_int, **f64)
        self.inv_mass = torch.tensor(1.0 / m_int, **f64)
        self.flags = torch.zeros(8, **i32)
        self.n_blocks_max = (P + 127) // 128
        self.partials = torch.zeros(self.n_blocks_max, _lib.RED_SLOTS, **f64)
        self.red_counter = torch.zeros(4, **i32)
        self.red_out = torch.zeros(_lib.RED_SLOTS, **f64)
        # [0] current step index (advanced by the first half-step), [1] index of
        # the step whose second half ran in a drift-fused force pass (step log)
        self.step_ctr = torch.full((2,), -1, device=dev, dtype=torch.int64)
        self.log_capacity = int(log_capacity)
        self.log = torch.zeros(self.log_capacity, _lib.RED_SLOTS + LOG_EXTRA + 1, **f64)
        self.extra = torch.zeros(LOG_EXTRA, **f64)
        self.types = torch.as_tensor(types).to(dev, torch.int32).contiguous()
        if self.types.shape[0] != n:
            raise ValueError("types must have one entry per atom")
        if int(self.types.min()) < 0 or int(self.types.max()) >= self.n_types:
            raise ValueError(f"atom types must lie in [0, {self.n_types})")
        self.rebuilds_host = 0
        # launch shapes (SimEngine.launch; 0 = built-in): EAM pass-1 / pass-2
        # threads per block, MLP descriptor / force threads per atom
        self.launch = [0, 0, 0, 0]
        # bumped whenever device buffers are reallocated: CUDA graphs captured
        # before then hold stale pointers
        self.generation = 0
        self._make_struct()
        vel = None if velocities is None else torch.as_tensor(velocities).to(dev, torch.float64).contiguous()
        self.load(pos, vel)

    # ---- struct plumbing -------------------------------------------------
    def _make_struct(self):
        s = _lib.SimEngine()
        s.n, s.n_pad, s.n_types, s.nbr_cap = self.n, self.n_pad, self.n_types, self.nbr_cap
        s.ncell[:] = [int(v) for v in self.ncell]
        s.n_cells = self.n_cells
        s.x_rc = self.x_rc
        s.skin_half2 = (self.skin / 2.0) ** 2
        p = _lib.ptr
        s.box = p(self.box_dev)
        for name in ("x", "v", "f32", "f64", "posq", "xref", "orig", "posfp", "nbr", "nnbr", "cell_of",
                     "cell_count", "cell_start", "cell_rank", "perm", "x_alt", "v_alt", "f32_alt", "f64_alt",
                     "orig_alt", "inv_mass", "mass", "flags", "partials", "red_counter", "red_out"):
            setattr(s, name, p(getattr(self, name)))
        s.n_blocks_max = self.n_blocks_max
        s.box_orthogonal = int(self.box.orthogonal)
        s.n_tiles, s.halo_cap = self.n_tiles, self.halo_cap
        s.halo, s.halo_n, s.nbr16 = _lib.ptr(self.halo), _lib.ptr(self.halo_n), _lib.ptr(self.nbr16)
        s.cut_mask = _lib.ptr(self.cut_mask)
        s.launch[:] = list(self.launch)
        self.st = s
        self.st_ref = ctypes.byref(s)

    @property
    def stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def set_launch(self, eam_density_threads: int | None = None, eam_force_threads: int | None = None,
                   mlp_desc_group: int | None = None, mlp_force_group: int | None = None):
        """Launch shapes of the EAM and MLP kernels (0 = built-in); see
        simulon_b200.autotune for measuring them.  Graphs captured before the
        change keep the shapes they were captured with."""
        for k, v in enumerate((eam_density_threads, eam_force_threads, mlp_desc_group, mlp_force_group)):
            if v is not None:
                self.launch[k] = int(v)
        self.st.launch[:] = list(self.launch)

    # ---- state in/out ------------------------------------------------------
    def load(self, positions, velocities=None):
        """Load original-order rows, sort into cells and build the list.  The
        copies from pinned host rows are asynchronous; the capacity check at
        the end synchronises, so they have landed when this returns.  Host
        velocities cross on a side stream while the cell sort and the list
        build run on the positions, and are scattered into the sorted slots
        afterwards (the same slots' values as loading them together)."""
        pos = torch.as_tensor(positions).to(self.device, torch.float64, non_blocking=True).contiguous()
        vel = None if velocities is None else torch.as_tensor(velocities)
        late_v = vel is not None and vel.device.type == "cpu"
        if late_v:
            main = torch.cuda.current_stream(self.device)
            side = self._copy_stream()
            side.wait_stream(main)
            with torch.cuda.stream(side):
                vel = vel.to(self.device, torch.float64, non_blocking=True).contiguous()
            vel.record_stream(main)
            ready = side.record_event()
        elif vel is not None:
            vel = vel.to(self.device, torch.float64).contiguous()
        _lib.call("sim_engine_load", self.st_ref, _lib.ptr(pos), _lib.ptr(None if late_v else vel),
                  _lib.ptr(self.types), self.stream)
        if late_v:
            main.wait_event(ready)
            _lib.call("sim_scatter_original_f64", self.st_ref, _lib.ptr(vel), _lib.ptr(self.v), self.stream)
        self.rebuilds_host += 1
        self.forces_valid = False
        self.ensure_capacity()

    def _copy_stream(self):
        if getattr(self, "_side_stream", None) is None:
            self._side_stream = torch.cuda.Stream(self.device)
        return self._side_stream

    def _alloc_lists(self):
        dev, P = self.device, self.n_pad
        self.nbr = torch.zeros(self.nbr_cap, P, device=dev, dtype=torch.int32)
        # in-cutoff slot mask written by EAM pass 1 (one 64-bit word per atom)
        self.cut_mask = torch.zeros(P, device=dev, dtype=torch.int64) if self.nbr_cap <= 64 else None
        if self.use_tiles:
            self.nbr16 = torch.zeros(self.nbr_cap, P, device=dev, dtype=torch.int16)
            self.halo = torch.zeros(self.n_tiles, self.halo_cap, device=dev, dtype=torch.int32)
            self.halo_n = torch.zeros(self.n_tiles, device=dev, dtype=torch.int32)
        else:
            self.nbr16 = self.halo = self.halo_n = None

    def ensure_capacity(self) -> bool:
        """Grow the neighbour list or the tile halos if the last rebuild overflowed
        them (synchronises).  True if anything grew."""
        grew = False
        for _ in range(3):
            flags = self.flags.cpu()
            bits = int(flags[1])
            if not bits & (_lib.SIM_STATUS_OVERFLOW | _lib.SIM_STATUS_HALO):
                return grew
            if bits & _lib.SIM_STATUS_OVERFLOW:
                self.nbr_cap = int(math.ceil((int(flags[2]) * 1.15 + 8) / 8.0) * 8)
            if bits & _lib.SIM_STATUS_HALO:
                want = int(math.ceil(int(flags[4]) * 1.2 / 256.0) * 256)
                if want <= HALO_CAP_MAX:
                    self.halo_cap = max(self.halo_cap, want)
                else:
                    self.use_tiles = False          # fall back to the untiled kernels
            self._alloc_lists()
            self.flags.zero_()
            self._make_struct()
            self.generation += 1
            _lib.call("sim_rebuild", self.st_ref, 0, self.stream)
            grew = True
        raise _lib.SimError("neighbour list / halo overflow persists after growing the capacity")

    def gather(self, which: str) -> torch.Tensor:
        """[N,3] float64 in the original atom order: 'x', 'v', 'f' (forces)."""
        out = torch.empty(self.n, 3, device=self.device, dtype=torch.float64)
        if which == "f":
            if self.fp64_forces and self._last_force_precision == 1:
                _lib.call("sim_gather_original_f64", self.st_ref, _lib.ptr(self.f64), _lib.ptr(out), self.stream)
            else:
                _lib.call("sim_gather_original_f32", self.st_ref, _lib.ptr(self.f32), _lib.ptr(out), self.stream)
        else:
            src = {"x": self.x, "v": self.v}[which]
            _lib.call("sim_gather_original_f64", self.st_ref, _lib.ptr(src), _lib.ptr(out), self.stream)
        return out

    _last_force_precision = 0

    def scatter(self, which: str, rows):
        """Write original-order rows into the slot arrays ('x' or 'v')."""
        rows = torch.as_tensor(rows).to(self.device, torch.float64).contiguous()
        dst = {"x": self.x, "v": self.v}[which]
        _lib.call("sim_scatter_original_f64", self.st_ref, _lib.ptr(rows), _lib.ptr(dst), self.stream)

    def set_positions(self, rows, velocities=None):
        """New coordinates (and, if given, velocities): reload (re-sorts cells,
        rebuilds the list, resets the skin reference)."""
        self.load(rows, self.gather("v") if velocities is None else velocities)

    def set_velocities(self, rows):
        self.scatter("v", rows)

    def box_matrix(self) -> np.ndarray:
        raw = self.box_dev.cpu().numpy().tobytes()
        return box_from_struct(_lib.SimBox.from_buffer_copy(raw))

    def cells_valid(self, H=None) -> bool:
        """Whether every axis of the cell grid with 3 or more cells is still at
        least rc + skin wide per cell for box H (default: the device box)."""
        H = self.box_matrix() if H is None else np.asarray(H, np.float64)
        w = perpendicular_widths(H)
        return all(int(n) < 3 or w[k] / int(n) >= self.x_rc for k, n in enumerate(self.ncell))

    def regrid(self, margin: float = 0.0) -> bool:
        """Cell grid for the current device box (after a barostat or a loader
        shrank cells below rc + skin, SIM_STATUS_CELLS, or to within ``margin``
        of it) and a full reload: the list is rebuilt on the new grid.  Cells
        are chosen at least (rc + skin)(1 + margin) wide.  Synchronises; True
        if the grid changed."""
        H = self.box_matrix()
        nc = cell_grid(H, self.x_rc * (1.0 + float(margin)), self.n)
        if np.array_equal(nc, self.ncell) and self.cells_valid(H):
            return False
        x, v = self.gather("x"), self.gather("v")
        self.ncell = nc
        self.n_cells = int(np.prod(nc))
        i32 = dict(device=self.device, dtype=torch.int32)
        self.cell_count = torch.zeros(self.n_cells + 1, **i32)
        self.cell_start = torch.zeros(self.n_cells + 1, **i32)
        r, lin = morton_rank(nc)
        self.cell_rank = torch.from_numpy(np.concatenate([r, lin])).to(self.device)
        self._make_struct()
        self.generation += 1
        self.load(x, v)
        return True

    def set_box(self, H):
        self.box = make_box(H)
        self.box_dev.copy_(torch.frombuffer(bytearray(bytes(self.box)), dtype=torch.uint8))
        self.st.box_orthogonal = int(self.box.orthogonal)

    # ---- step primitives ---------------------------------------------------
    def rebuild(self, only_if_flagged: bool = True):
        _lib.call("sim_rebuild", self.st_ref, int(only_if_flagged), self.stream)

    def rebuild_if_needed(self):
        """Conditional rebuild (an IF node when captured in a CUDA graph)."""
        _lib.call("sim_rebuild_if_needed", self.st_ref, self.stream)

    def eam_forces_integrate(self, tables, integ):
        """EAM pass 1, then pass 2 with the second half-step fused into it."""
        _lib.call("sim_eam_density", self.st_ref, tables.ref, self.stream)
        _lib.call("sim_eam_force_integrate", self.st_ref, tables.ref, integ.ref, self.stream)
        self._last_force_precision = 0
        self.forces_valid = True

    def eam_forces_integrate_drift(self, tables, integ):
        """EAM pass 1, then pass 2 with this step's second half and the next
        step's first half fused into it (needs the untiled kernels)."""
        _lib.call("sim_eam_density", self.st_ref, tables.ref, self.stream)
        _lib.call("sim_eam_force_integrate_drift", self.st_ref, tables.ref, integ.ref, self.stream)
        self._last_force_precision = 0
        self.forces_valid = True

    def eam_forces_integrate_indenter(self, tables, integ, indenter_ref, mode: int):
        """EAM pass 1, then pass 2 with a spherical indenter's force added before
        the integrator epilogue: mode 1 the second half-step, mode 2 also the
        next step's first half."""
        _lib.call("sim_eam_density", self.st_ref, tables.ref, self.stream)
        _lib.call("sim_eam_force_integrate_indenter", self.st_ref, tables.ref, integ.ref, indenter_ref, int(mode),
                  self.stream)
        self._last_force_precision = 0
        self.forces_valid = True

    def eam_step_drift_indenter(self, tables, integ, indenter_ref):
        """eam_forces_integrate_indenter (mode 2) + log_step(after_drift=True)
        + rebuild_if_needed, with the log row and the rebuild decision made by
        pass 2's last block."""
        _lib.call("sim_eam_step_drift_indenter", self.st_ref, tables.ref, integ.ref, indenter_ref, _lib.ptr(self.extra),
                  LOG_EXTRA, _lib.ptr(self.log), self.log_capacity, self.stream)
        self._last_force_precision = 0
        self.forces_valid = True

    def eam_step_drift(self, tables, integ):
        """eam_forces_integrate_drift + log_step(after_drift=True) +
        rebuild_if_needed, with the log row and the rebuild decision made by
        pass 2's last block (no separate log or condition kernel)."""
        _lib.call("sim_eam_step_drift", self.st_ref, tables.ref, integ.ref, _lib.ptr(self.extra), LOG_EXTRA,
                  _lib.ptr(self.log), self.log_capacity, self.stream)
        self._last_force_precision = 0
        self.forces_valid = True

    def eam_forces(self, tables):
        _lib.call("sim_eam_forces", self.st_ref, tables.ref, self.stream)
        self._last_force_precision = 0
        self.forces_valid = True

    def lj_forces(self, params, precision: int):
        _lib.call("sim_lj_forces", self.st_ref, params.ref, int(precision), self.stream)
        self._last_force_precision = int(precision)
        self.forces_valid = True

    def lj_forces_integrate(self, params, integ, mode: int):
        """FP32-pair LJ forces with the integrator's second half (mode 1), and
        also the next step's first half (mode 2), in the same pass."""
        _lib.call("sim_lj_forces_integrate", self.st_ref, params.ref, integ.ref, int(mode), self.stream)
        self._last_force_precision = 0
        self.forces_valid = True

    def integrate_first(self, integ, precision: int):
        _lib.call("sim_integrate_first", self.st_ref, integ.ref, int(precision), self.stream)

    def integrate_second(self, integ, precision: int):
        _lib.call("sim_integrate_second", self.st_ref, integ.ref, int(precision), self.stream)

    def integrate_second_first(self, integ, precision: int):
        """Second half of this step and first half of the next with the same forces."""
        _lib.call("sim_integrate_second_first", self.st_ref, integ.ref, int(precision), self.stream)

    def berendsen(self, params):
        _lib.call("sim_berendsen", self.st_ref, params.ref, _lib.ptr(self.extra), self.stream)

    def berendsen_mu(self, params):
        """The Berendsen controller alone (pressure, mu, box scaled); the atoms
        follow in berendsen_scale_first at the next step."""
        _lib.call("sim_berendsen_mu", self.st_ref, params.ref, _lib.ptr(self.extra), self.stream)

    def berendsen_scale_first(self, params, integ, precision: int):
        """The atoms' part of the last berendsen_mu and this step's first half in one pass."""
        _lib.call("sim_berendsen_scale_first", self.st_ref, params.ref, _lib.ptr(self.extra), integ.ref,
                  int(precision), self.stream)

    def log_step(self, after_drift: bool = False):
        """Record this step's reductions in the device log (after_drift: the step
        was finished by eam_forces_integrate_drift, whose index is step_ctr[1])."""
        ctr = self.step_ctr[1:] if after_drift else self.step_ctr
        _lib.call("sim_log_step", self.st_ref, _lib.ptr(ctr), _lib.ptr(self.extra), LOG_EXTRA,
                  _lib.ptr(self.log), self.log_capacity, self.stream)

    # ---- reductions (device tensors, no sync) ----------------------------
    def potential_energy(self) -> torch.Tensor:
        return self.red_out[_lib.RED_EPOT_EMBED] + self.red_out[_lib.RED_EPOT_PAIR]

    def virial_tensor(self) -> torch.Tensor:
        w = self.red_out[_lib.RED_W]
        return torch.stack([torch.stack([w[0], w[3], w[4]]), torch.stack([w[3], w[1], w[5]]),
                            torch.stack([w[4], w[5], w[2]])])

    def kinetic_tensor(self) -> torch.Tensor:
        k = self.red_out[_lib.RED_K]
        return torch.stack([torch.stack([k[0], k[3], k[4]]), torch.stack([k[3], k[1], k[5]]),
                            torch.stack([k[4], k[5], k[2]])])

    def status(self) -> int:
        """Device status bits (synchronises)."""
        return int(self.flags[1].item())

    def neighbor_stats(self):
        nn = self.nnbr[: self.n].float()
        return dict(mean=float(nn.mean()), max=int(nn.max()), cap=self.nbr_cap)

    def half_list(self, rc2: float | None = None):
        """The engine's Verlet list as the reference's half list (i<j by original
        index, sorted), filtered in FP64 at the current positions."""
        rc2 = self.x_rc ** 2 if rc2 is None else float(rc2)
        row_ptr = torch.zeros(self.n + 1, device=self.device, dtype=torch.int64)
        _lib.call("sim_engine_half_count", self.st_ref, rc2, _lib.ptr(row_ptr), self.stream)
        E = int(row_ptr[-1].item())
        ei = torch.empty(E, device=self.device, dtype=torch.int64)
        ej = torch.empty(E, device=self.device, dtype=torch.int64)
        dist = torch.empty(E, device=self.device, dtype=torch.float64)
        if E:
            _lib.call("sim_engine_half_fill", self.st_ref, rc2, _lib.ptr(row_ptr), _lib.ptr(ei), _lib.ptr(ej),
                      _lib.ptr(dist), self.stream)
        return torch.stack([ei, ej]), dist


class DeviceStruct:
    """Keeps a ctypes struct and the tensors it points into alive together."""

    def __init__(self, struct, keep):
        self.struct = struct
        self.keep = keep
        self.ref = ctypes.byref(struct)


def integrator_params(engine: MDEngine, dt: float, *, langevin: bool = False, temperature: float = 0.0,
                      gamma: float = 0.0, seed: int = 0) -> DeviceStruct:
    """SimIntegrator for VerletIntegrator semantics (integrator.py:45-88)."""
    s = _lib.SimIntegrator()
    s.dt = float(dt)
    s.langevin = int(langevin)
    keep = []
    if langevin:
        g = torch.tensor(float(gamma), dtype=torch.float64)
        T = torch.tensor(float(temperature), dtype=torch.float64)
        s.damp = float(torch.exp(-g * dt))
        rff = torch.sqrt((KB_EV * T) / engine.mass.cpu() * (1.0 - torch.exp(-2.0 * g * dt))).to(engine.device)
        keep.append(rff)
        s.rff = _lib.ptr(rff)
    else:
        s.damp = 1.0
    s.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    s.step_ctr = _lib.ptr(engine.step_ctr)
    return DeviceStruct(s, keep)


def berendsen_params(dt: float, target_bar: float, tau: float, kappa: float = 4.57e-5, mu_max: float = 0.05,
                     coordinate_scale_power: int = 2, reset_reference: bool = True) -> DeviceStruct:
    """SimBerendsen for BerendsenBarostat semantics (barostat.py:21-68)."""
    s = _lib.SimBerendsen()
    s.target_bar, s.tau, s.kappa, s.mu_max, s.dt = float(target_bar), float(tau), float(kappa), float(mu_max), float(dt)
    s.coordinate_scale_power = int(coordinate_scale_power)
    s.reset_reference = int(reset_reference)
    return DeviceStruct(s, [])
