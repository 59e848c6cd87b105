"""System state with the interface of io_utils/reader.py (AtomFileReader).

The atoms' positions, velocities, forces and Verlet list live on the device
inside an ``MDEngine`` (cell order, FP64 state).  The reference attributes
(``coordinates``, ``atom_velocities``, ``graph_data.pos/edge_index/edge_attr``,
``pair_params``) are materialised in the caller's atom order and dtype when
read, and writing them uploads into the engine.
"""
from __future__ import annotations

import time

import numpy as np
import torch

from .box import Box
from .engine import MDEngine

# element masses in amu (core/element_info.py:5-27, plus common EAM metals)
ELEMENT_MASS = {"H": 1.008, "He": 4.003, "Li": 6.940, "Be": 9.012, "B": 10.810, "C": 12.011, "N": 14.007,
                "O": 15.999, "F": 18.998, "Ne": 20.180, "Na": 22.990, "Mg": 24.305, "Al": 26.982,
                "Si": 28.085, "P": 30.974, "S": 32.060, "Cl": 35.450, "Ar": 39.948, "Fe": 55.845,
                "Ni": 58.693, "Cu": 63.546, "Mo": 95.95, "Ta": 180.948, "W": 183.84, "Re": 186.207,
                "Pt": 195.084, "Au": 196.967}


def _mass(symbol: str) -> float:
    if symbol not in ELEMENT_MASS:
        raise KeyError(f"no mass for element {symbol!r}")
    return ELEMENT_MASS[symbol]


class _GraphData:
    """graph_data view: pos / edge_index / edge_attr materialised on demand."""

    def __init__(self, owner):
        self._owner = owner

    @property
    def pos(self):
        return self._owner.coordinates

    @property
    def edge_index(self):
        return self._owner._half_list()[0]

    @property
    def edge_attr(self):
        return self._owner._half_list()[1]

    @property
    def element_edge_0(self):
        return self._owner.element_ids[self.edge_index[0]]

    @property
    def element_edge_1(self):
        return self._owner.element_ids[self.edge_index[1]]

    @property
    def index_pairs(self):
        ei = self.edge_index
        return torch.stack([self._owner.element_ids[ei[0]], self._owner.element_ids[ei[1]]], dim=1)

    def get(self, key, default=None):
        return getattr(self, key, default)


class AtomFileReader:
    def __init__(self, filename, box_length, cutoff, device=None, parameter=None, skin_thickness=5.0,
                 is_mlp=False, is_fs=False, is_switch=False, switch_ratio: float = 0.9, box_vectors=None,
                 nbr_capacity: int | None = None):
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        if self.device.type != "cuda":
            raise RuntimeError("simulon_b200 runs on CUDA devices only")
        self.dtype = torch.get_default_dtype()
        self.box = Box(box_vectors if box_vectors is not None else box_length, device=self.device)
        self.box_length_cpu = box_length
        self.box_length = self.box.diag[0] if self.box.is_orthogonal else torch.tensor(
            box_length, device=self.device, dtype=torch.float64)
        self.cutoff = torch.tensor(cutoff, device=self.device)
        self.parameter = parameter
        self.is_mlp, self.is_fs, self.is_switch = is_mlp, is_fs, is_switch
        self.switch_ratio = float(switch_ratio)
        self.atom_types, coords, self._masses = self._load_input(filename)
        self.atom_count = len(self.atom_types)
        ids = {}
        self.element_to_id = [ids.setdefault(a, len(ids)) for a in self.atom_types]
        self.elements = list(ids)
        self.element_ids = torch.tensor(self.element_to_id, device=self.device)
        self.atom_mass = torch.tensor(self._masses, device=self.device)
        self.skin_thickness = torch.tensor(skin_thickness, device=self.device)
        self.verlet_cutoff = self.cutoff + self.skin_thickness
        # coordinates enter in the default dtype, as the reference stores them (reader.py:279)
        coords = torch.as_tensor(np.asarray(coords, dtype=np.float64)).to(self.dtype).to(torch.float64)
        type_mass = [_mass(e) for e in self.elements]
        self.engine = MDEngine(coords, self.element_ids, type_mass, self.box.H.cpu().numpy(),
                               float(self.cutoff), float(self.skin_thickness), device=self.device,
                               nbr_cap=nbr_capacity, fp64_forces=self.dtype == torch.float64)
        self.graph_data = _GraphData(self)
        self.last_positions = None
        self.needs_update = False
        self.profile = {"neighbor_time": 0.0, "neighbor_builds": 0, "effective_edges_last": 0}

    @classmethod
    def from_arrays(cls, symbols, coords, box_length, cutoff, **kw):
        """Same as the file constructor, from in-memory symbols and [N,3] coordinates."""
        obj = cls.__new__(cls)
        obj._arrays = (list(symbols), np.asarray(coords, dtype=np.float64))
        cls.__init__(obj, None, box_length, cutoff, **kw)
        return obj

    # ---- file input (reader.py:256-279) ----------------------------------
    def _load_input(self, filename):
        if filename is None:
            symbols, coords = self._arrays
            return symbols, coords, [_mass(s) for s in symbols]
        return self.read_file(filename)

    @staticmethod
    def read_file(filename):
        with open(filename) as fh:
            lines = fh.readlines()
        if not lines:
            raise ValueError(f"Error: The file {filename} is empty.")
        skip = 1 if str(filename).lower().endswith(".xyz") else 0
        try:
            n = int(lines[0].strip())
            types, coords, masses = [], [], []
            for line in lines[1 + skip:]:
                parts = line.split()
                if len(parts) >= 4:
                    types.append(parts[0])
                    coords.append([float(parts[1]), float(parts[2]), float(parts[3])])
                    masses.append(_mass(parts[0]))
        except Exception as e:
            raise ValueError(f"Error: {e}")
        if len(types) != n:
            raise ValueError(f"Error: header says {n} atoms, found {len(types)}")
        return types, coords, masses

    # ---- state views -----------------------------------------------------
    @property
    def coordinates(self) -> torch.Tensor:
        return self.engine.gather("x").to(self.dtype)

    @coordinates.setter
    def coordinates(self, value):
        self.engine.set_positions(value)

    @property
    def atom_velocities(self) -> torch.Tensor:
        return self.engine.gather("v").to(self.dtype)

    @atom_velocities.setter
    def atom_velocities(self, value):
        self.engine.set_velocities(value)

    def update_velocities(self, velocities):
        self.engine.set_velocities(velocities)

    def update_coordinates(self, coordinates, velocities=None):
        """Replace the coordinates (re-sorts, rebuilds the list, resets the skin
        reference); ``velocities`` (beyond the reference's signature) replaces
        the velocities in the same load."""
        self.engine.set_positions(coordinates, velocities)

    def update_neighbor_list(self):
        t0 = time.perf_counter()
        self.engine.rebuild(only_if_flagged=False)
        torch.cuda.synchronize(self.device)
        self.profile["neighbor_time"] += time.perf_counter() - t0

    def _half_list(self):
        return self.engine.half_list(float(self.verlet_cutoff) ** 2)

    def get_cutoff_mask(self):
        return self.graph_data.edge_attr <= self.cutoff

    def effective_edge_count(self) -> int:
        return int(self.get_cutoff_mask().sum().item())

    def initial_parameters(self):
        """Per-edge LJ parameters in dictionary order, float32 (reader.py:165-210)."""
        ei = self.graph_data.edge_index
        first = next(iter(self.parameter.values()))
        pairs = torch.stack([self.element_ids[ei[0]], self.element_ids[ei[1]]], 1).cpu().numpy()
        out = []
        for key in first:
            vals = [self.parameter[str(np.array(p))][key] for p in pairs]
            out.append(torch.tensor(vals, dtype=torch.float32, device=self.device))
        return out

    @property
    def pair_params(self):
        return self.initial_parameters()

    # ---- velocities (reader.py:292-339) ----------------------------------
    def set_maxwell_boltzmann_velocity(self, temperature):
        """v ~ N(0, kB T / m) per component from torch's generator on this
        device, centre-of-mass momentum removed; the operations and their
        order are those of reader.py:319-339, so a seeded draw gives the
        reference's velocities bit for bit."""
        kB_eV = 8.617333262e-5
        MASS_CONV = 1.036427e-4
        m_internal = (self.atom_mass * MASS_CONV).unsqueeze(-1)
        sigma = torch.sqrt(kB_eV * temperature / m_internal)
        v = torch.randn((self.atom_count, 3), device=self.device, dtype=self.dtype) * sigma
        total_p = (v * m_internal).sum(dim=0)
        total_m = m_internal.sum()
        v = v - total_p / total_m
        self.engine.set_velocities(v)

    def create_velocity_gaussian(self, temperature, seed):
        torch.manual_seed(seed)
        sigma = torch.sqrt((8.617333262e-5 * temperature * 1.60218e-20) / self.atom_mass.to(self.dtype))
        v = torch.randn((self.atom_count, 3), device=self.device, dtype=self.dtype) * sigma.view(-1, 1)
        m = self.atom_mass.to(self.dtype).view(-1, 1)
        v -= (v * m).sum(0) / m.sum()
        self.engine.set_velocities(v)

    def get_atom_num(self):
        return self.atom_count

    def get_atom_type_array(self):
        return self.atom_types

    def get_atom_coordinates(self):
        return self.coordinates

    def get_atom_mass(self):
        return self.atom_mass
