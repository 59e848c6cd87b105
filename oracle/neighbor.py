"""Oracle half Verlet list (TEST INFRASTRUCTURE ONLY).

Python wrapper over ``neighbor_ref.c`` -- the C restatement of
core/neighbor_search/gpu_kdtree.py:90-155 followed by io_utils/reader.py:477-484
(keep i<j, recompute distances with the box's minimum image).

``half_list`` returns the pair set sorted by (i, j) together with the integer
image of each pair and its squared distance in the coordinate dtype.  The
brute-force mode is the literal restatement; the cell mode enumerates the same
candidates through a 27-cell stencil (cells at least rc wide, >= 3 per axis)
and is checked against the brute force in the tests before it is used at
sizes where O(N^2) is infeasible.

``rc2_like_reference`` reproduces how the reference forms rc^2: the Verlet
cutoff is a torch tensor (cutoff + skin, in the default dtype;
reader.py:50,77-78) and ``rc2 = cutoff*cutoff`` is formed in that dtype
(gpu_kdtree.py:99) before the comparison in the coordinate dtype.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from .box import OracleBox

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "neighbor_ref.c")
_LIB_DIR = os.path.join(_HERE, "_build")
_LIB = os.path.join(_LIB_DIR, "libneighbor_ref.so")
_lib = None


def build() -> str:
    """Compile the C restatement (gcc, contraction off so only explicit fma fuses)."""
    os.makedirs(_LIB_DIR, exist_ok=True)
    if (not os.path.exists(_LIB)) or os.path.getmtime(_LIB) < os.path.getmtime(_SRC):
        tmp = _LIB + f".{os.getpid()}.tmp"
        subprocess.check_call(["gcc", "-O2", "-shared", "-fPIC", "-ffp-contract=off",
                               "-fno-fast-math", _SRC, "-o", tmp, "-lm"])
        os.replace(tmp, _LIB)
    return _LIB


def _load():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(build())
        for suf, ct in (("f64", ctypes.c_double), ("f32", ctypes.c_float)):
            fn = getattr(lib, f"oracle_half_list_{suf}")
            fn.restype = ctypes.c_int64
            fn.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                           ctypes.c_int, ct, ctypes.c_int, ctypes.c_void_p,
                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                           ctypes.c_int64]
        _lib = lib
    return _lib


def rc2_like_reference(cutoff: float, skin: float, dtype) -> float:
    """rc^2 exactly as the reference forms it from tensor(cutoff) + tensor(skin)."""
    npd = np.float32 if np.dtype(dtype) == np.float32 else np.float64
    rc = npd(npd(cutoff) + npd(skin))
    return float(npd(rc * rc))


def cell_grid(box: OracleBox, rc: float):
    """Cells per axis for the stencil mode, or None when any axis has < 3 cells."""
    w = box.perpendicular_widths()
    n = np.floor(w / (rc * 1.0001)).astype(np.int64)
    if (n < 3).any():
        return None
    return n.astype(np.int32)


def half_list(pos: np.ndarray, box: OracleBox, rc2: float, mode: str = "auto"):
    """Half list (i<j, d^2 < rc2) in the dtype of ``pos`` (float32 or float64).

    Returns dict(i, j int64 [E], image int32 [E,3], d2 [E] in pos dtype).
    """
    lib = _load()
    pos = np.ascontiguousarray(pos)
    if pos.dtype not in (np.float32, np.float64):
        raise TypeError("positions must be float32 or float64")
    suf = "f32" if pos.dtype == np.float32 else "f64"
    H = np.ascontiguousarray(box.H.numpy(), dtype=np.float64)
    Hi = np.ascontiguousarray(box.H_inv.numpy(), dtype=np.float64)
    rc = float(np.sqrt(rc2))
    grid = cell_grid(box, rc) if mode in ("auto", "cell") else None
    if mode == "cell" and grid is None:
        raise ValueError("box too small for the cell stencil (need >= 3 cells per axis)")
    cell_mode = 1 if grid is not None else 0
    ncell = grid if grid is not None else np.ones(3, np.int32)
    n = pos.shape[0]
    fn = getattr(lib, f"oracle_half_list_{suf}")
    cap = max(16, int(n) * 32)          # grown (and the search rerun) when a row set needs more
    while True:
        oi = np.empty(cap, np.int64)
        oj = np.empty(cap, np.int64)
        oimg = np.empty((cap, 3), np.int32)
        od2 = np.empty(cap, pos.dtype)
        got = fn(pos.ctypes.data, n, H.ctypes.data, Hi.ctypes.data,
                 int(box.is_orthogonal), rc2, cell_mode, ncell.ctypes.data,
                 oi.ctypes.data, oj.ctypes.data, oimg.ctypes.data, od2.ctypes.data, cap)
        if got >= 0:
            return dict(i=oi[:got].copy(), j=oj[:got].copy(), image=oimg[:got].copy(),
                        d2=od2[:got].copy())
        cap = -got


def edge_distances(pos, i, j, box: OracleBox):
    """reader.py:364-376: |minimum_image(pos_i - pos_j)| in the coordinate dtype."""
    import torch
    p = torch.as_tensor(pos)
    rij = box.minimum_image(p[torch.as_tensor(i)] - p[torch.as_tensor(j)])
    return torch.norm(rij, dim=1).numpy()
