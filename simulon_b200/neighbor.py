"""Half Verlet list on the device: drop-in for find_neighbors_gpu_pbc.

``find_neighbors_gpu_pbc(positions, cutoff, box)`` returns
``(edge_index int64 [2,E], dist [E])`` with the contract of
core/neighbor_search/gpu_kdtree.py:56-155 as consumed by
io_utils/reader.py:477-484: pairs i<j with |min_image(x_i - x_j)|^2 < rc^2,
sorted by (i, j).  The membership test runs in the dtype of ``positions``
with the reference's exact operation order (orthogonal: r - d*round(r/d);
triclinic: fma-chained products with H^-1 and H; d^2 = (x^2 + y^2) + z^2), so
the pair set is bit-identical to the reference's.  Unlike the reference's
CUDA branch it handles any box (orthorhombic and triclinic), never truncates
rows, and is O(N) through a cell grid instead of O(N^2).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .engine import make_box, perpendicular_widths


def _box_matrix(box, device) -> np.ndarray:
    if hasattr(box, "H"):
        return torch.as_tensor(box.H).detach().double().cpu().numpy()
    L = float(box)
    return np.diag([L, L, L])


def reference_rc2(cutoff, dtype: torch.dtype) -> float:
    """rc^2 as the reference compares it: cutoff*cutoff in the cutoff's own
    dtype (a tensor in the reference, reader.py:50,77-78), then cast to the
    coordinate dtype for the comparison."""
    if torch.is_tensor(cutoff):
        rc2 = (cutoff * cutoff).to(dtype)
        return float(rc2)
    return float(torch.tensor(float(cutoff) * float(cutoff), dtype=torch.float64).to(dtype))


def half_list(positions: torch.Tensor, rc2: float, H, return_image: bool = False):
    """Core call: (edge_index [2,E] int64, dist [E] in positions' dtype[, image int32 [E,3]])."""
    if not positions.is_cuda:
        raise RuntimeError("positions must be a CUDA tensor")
    if positions.dtype not in (torch.float32, torch.float64):
        raise TypeError("positions must be float32 or float64")
    pos = positions.contiguous()
    dev = pos.device
    n = int(pos.shape[0])
    code = 0 if pos.dtype == torch.float32 else 1
    box = make_box(H)
    rc = float(np.sqrt(rc2))
    nc = np.maximum(np.floor(perpendicular_widths(H) / (rc * (1.0 + 1e-6))), 1).astype(np.int64)
    while nc.prod() > max(4 * n, 27):
        k = int(np.argmax(nc))
        nc[k] = max(1, nc[k] // 2)
    ncell = nc.astype(np.int32)
    n_cells = int(ncell.prod())
    i32 = dict(device=dev, dtype=torch.int32)
    cell_of = torch.empty(max(n, 1), **i32)
    cell_count = torch.zeros(n_cells + 1, **i32)
    cell_start = torch.empty(n_cells + 1, **i32)
    sorted_idx = torch.empty(max(n, 1), **i32)
    row_ptr = torch.zeros(n + 1, device=dev, dtype=torch.int64)
    st = torch.cuda.current_stream(dev).cuda_stream
    nc_c = (ctypes.c_int32 * 3)(*[int(v) for v in ncell])
    _lib.call("sim_half_list_count", _lib.ptr(pos), code, n, ctypes.byref(box), rc2, nc_c, _lib.ptr(cell_of),
              _lib.ptr(cell_count), _lib.ptr(cell_start), _lib.ptr(sorted_idx), _lib.ptr(row_ptr), st)
    E = int(row_ptr[-1].item())
    ei = torch.empty(E, device=dev, dtype=torch.int64)
    ej = torch.empty(E, device=dev, dtype=torch.int64)
    dist = torch.empty(E, device=dev, dtype=pos.dtype)
    img = torch.empty(E, 3, **i32) if return_image else None
    if E:
        _lib.call("sim_half_list_fill", _lib.ptr(pos), code, n, ctypes.byref(box), rc2, nc_c, _lib.ptr(cell_start),
                  _lib.ptr(sorted_idx), _lib.ptr(cell_of), _lib.ptr(row_ptr), _lib.ptr(ei), _lib.ptr(ej),
                  _lib.ptr(img), _lib.ptr(dist), st)
    out = (torch.stack([ei, ej]), dist)
    return out + (img,) if return_image else out


def find_neighbors_gpu_pbc(positions, cutoff, box, batch_size=None, return_image: bool = False):
    """Drop-in for gpu_kdtree.find_neighbors_gpu_pbc (batch_size is accepted and unused)."""
    H = _box_matrix(box, positions.device)
    return half_list(positions, reference_rc2(cutoff, positions.dtype), H, return_image=return_image)


find_neighbors_gpu_pbc_pytorch = find_neighbors_gpu_pbc
