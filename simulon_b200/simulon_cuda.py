"""Drop-in for the reference's native module ``simulon_cuda``.

Same five functions and argument meanings as the pybind module of
cuda source/ops.cpp:47-53, backed by libsimb200.so:

* lj_energy_force_cuda(pos f32[N,3], edge_index i64[2,E], sigma f32[E],
  epsilon f32[E], box_length) -> [energy f32[1], forces f32[N,3]]
  (cuda source/lj_energy_force.cpp:10-20; smoothing mode from
  configure_lj_smoothing, ops.cpp:43-45, kept as host state here instead of
  device globals);
* neighbor_search_cuda(positions f32[N,3], cutoff, box_length) ->
  [edge_index i64[2,E], dist f32[E]] (neighbor_search_kernel.cu:73-138) --
  here via the exact half-list builder: no 500-neighbour truncation, no
  O(N^2) loop, no device-wide synchronisation;
* density_pass(...) / force_pass(...) accumulate in place into caller
  buffers (eam_cuda_ext.cpp:30-60); *_cuda aliases are provided because the
  reference's EAMForceCUDAExt looks for either name (eam_force_cu.py:424-430).

Put ``simulon_b200`` on the path and ``import simulon_b200.simulon_cuda as
simulon_cuda`` (or register it under that name with
``simulon_b200.install_simulon_cuda()``) so the reference wrappers pick it up.
"""
from __future__ import annotations

import torch

from . import _lib
from .neighbor import half_list

_SMOOTHING = {"mode": 0, "rc": 0.0, "rs": 0.0}


def _need_cuda(*ts):
    for t in ts:
        if not (torch.is_tensor(t) and t.is_cuda):
            raise RuntimeError("simulon_cuda: arguments must be CUDA tensors")


def configure_lj_smoothing(mode: int, rc: float, rs: float):
    if int(mode) not in (0, 1, 2):
        raise ValueError("mode must be 0 (raw), 1 (force shift) or 2 (switch)")
    _SMOOTHING.update(mode=int(mode), rc=float(rc), rs=float(rs))


def lj_energy_force_cuda(pos, edge_index, sigma, epsilon, box_length):
    _need_cuda(pos, edge_index, sigma, epsilon)
    pos = pos.contiguous().float()
    n = pos.shape[0]
    forces = torch.zeros(n, 3, device=pos.device, dtype=torch.float32)
    energy = torch.zeros(1, device=pos.device, dtype=torch.float32)
    ei = edge_index.contiguous().long()
    st = torch.cuda.current_stream(pos.device).cuda_stream
    _lib.call("sim_legacy_lj_energy_force", _lib.ptr(pos), _lib.ptr(ei[0]), _lib.ptr(ei[1]), int(ei.shape[1]),
              _lib.ptr(sigma.contiguous().float()), _lib.ptr(epsilon.contiguous().float()), float(box_length),
              _SMOOTHING["mode"], _SMOOTHING["rc"], _SMOOTHING["rs"], _lib.ptr(forces), _lib.ptr(energy), st)
    return [energy, forces]


def neighbor_search_cuda(positions, cutoff, box_length):
    _need_cuda(positions)
    L = float(box_length)
    import numpy as np
    rc2 = float(torch.tensor(float(cutoff) ** 2, dtype=torch.float64).float())
    ei, dist = half_list(positions.contiguous().float(), rc2, np.diag([L, L, L]))
    return [ei, dist]


def density_pass(distances, row_index, col_index, atom_types, density_table, inv_dr, n_r, rho_out):
    _need_cuda(distances, row_index, col_index, atom_types, density_table, rho_out)
    E = int(density_table.shape[0]) if density_table.dim() == 3 else 1
    _lib.call("sim_legacy_density_pass", _lib.ptr(distances.contiguous()), _lib.ptr(row_index.contiguous()),
              _lib.ptr(col_index.contiguous()), _lib.ptr(atom_types.contiguous()), int(distances.numel()),
              _lib.ptr(density_table.contiguous()), E, float(inv_dr), int(n_r), _lib.ptr(rho_out),
              torch.cuda.current_stream(distances.device).cuda_stream)


def force_pass(distances, dist_vec, row_index, col_index, atom_types, density_deriv_table, pair_deriv_table,
               dF_drho, inv_dr, n_r, forces_out):
    _need_cuda(distances, dist_vec, row_index, col_index, atom_types, density_deriv_table, pair_deriv_table,
               dF_drho, forces_out)
    E = int(density_deriv_table.shape[0]) if density_deriv_table.dim() == 3 else 1
    _lib.call("sim_legacy_force_pass", _lib.ptr(distances.contiguous()), _lib.ptr(dist_vec.contiguous()),
              _lib.ptr(row_index.contiguous()), _lib.ptr(col_index.contiguous()), _lib.ptr(atom_types.contiguous()),
              int(distances.numel()), _lib.ptr(density_deriv_table.contiguous()),
              _lib.ptr(pair_deriv_table.contiguous()), _lib.ptr(dF_drho.contiguous()), E, float(inv_dr), int(n_r),
              _lib.ptr(forces_out), torch.cuda.current_stream(distances.device).cuda_stream)


density_pass_cuda = density_pass
force_pass_cuda = force_pass
