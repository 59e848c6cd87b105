"""Launch-shape autotuning (C ABI group 5) with a per-machine cache.

The kernels' launch shapes (threads per block of the two EAM passes,
threads per atom of the MLP descriptor and force kernels) live in
``SimEngine.launch``.  ``tune_eam`` / ``tune_mlp`` time every candidate on the
engine's current state with CUDA events (``sim_autotune_eam`` /
``sim_autotune_mlp``), store the fastest in the engine and cache the result
per (GPU, kernel family, atom count, mean list length) in a JSON file, so a
second run on the same machine and system size only reads the cache.

No counterpart in the reference, whose kernels have fixed launch shapes.
"""
from __future__ import annotations

import json
import os

import torch

from . import _lib

EAM_DENSITY_THREADS = (128, 256, 512)
EAM_FORCE_THREADS = (256, 512, 1024)
MLP_GROUPS = (4, 8)


def cache_path() -> str:
    """SIMB200_TUNE_CACHE, else ~/.cache/simulon_b200/launch_shapes.json."""
    env = os.environ.get("SIMB200_TUNE_CACHE")
    if env:
        return env
    return os.path.join(os.path.expanduser("~"), ".cache", "simulon_b200", "launch_shapes.json")


def _load(path):
    try:
        with open(path) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _store(path, key, value):
    data = _load(path)
    data[key] = value
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as fh:
        json.dump(data, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def cache_key(engine, family: str) -> str:
    """(GPU name, kernel family, atom count, mean list length rounded)."""
    nbar = float(engine.nnbr[:engine.n].float().mean())
    return f"{torch.cuda.get_device_name(engine.device)}|{family}|{engine.n}|{round(nbar)}"


def tune_eam(engine, tables, reps: int = 10, use_cache: bool = True, path: str | None = None) -> dict:
    """Pick and set the EAM pass-1 and pass-2 threads per block."""
    path = path or cache_path()
    key = cache_key(engine, "eam")
    hit = _load(path).get(key) if use_cache else None
    if hit is None:
        ms = torch.zeros(6, dtype=torch.float32)
        best = torch.zeros(2, dtype=torch.int32)
        _lib.call("sim_autotune_eam", engine.st_ref, tables.ref, int(reps), ms.data_ptr(), best.data_ptr(),
                  engine.stream)
        hit = {"density_threads": int(best[0]), "force_threads": int(best[1]),
               "ms": {f"density_{t}": float(v) for t, v in zip(EAM_DENSITY_THREADS, ms[:3])}
               | {f"force_{t}": float(v) for t, v in zip(EAM_FORCE_THREADS, ms[3:])}}
        if use_cache:
            _store(path, key, hit)
    engine.set_launch(eam_density_threads=hit["density_threads"], eam_force_threads=hit["force_threads"])
    return hit


def tune_mlp(engine, reps: int = 10, use_cache: bool = True, path: str | None = None, dEdG=None) -> dict:
    """Pick and set the MLP descriptor and force kernels' threads per atom
    (times them with dEdG, default a constant [n, 16] array)."""
    path = path or cache_path()
    key = cache_key(engine, "mlp")
    hit = _load(path).get(key) if use_cache else None
    if hit is None:
        dev = engine.device
        G = torch.zeros(engine.n_pad, 16, device=dev, dtype=torch.float32)
        d = dEdG if dEdG is not None else torch.full((engine.n, 16), 0.01, device=dev, dtype=torch.float32)
        ms = torch.zeros(4, dtype=torch.float32)
        best = torch.zeros(2, dtype=torch.int32)
        _lib.call("sim_autotune_mlp", engine.st_ref, _lib.ptr(d), _lib.ptr(G), int(reps), ms.data_ptr(),
                  best.data_ptr(), engine.stream)
        hit = {"desc_group": int(best[0]), "force_group": int(best[1]),
               "ms": {f"desc_{g}": float(v) for g, v in zip(MLP_GROUPS, ms[:2])}
               | {f"force_{g}": float(v) for g, v in zip(MLP_GROUPS, ms[2:])}}
        if use_cache:
            _store(path, key, hit)
    engine.set_launch(mlp_desc_group=hit["desc_group"], mlp_force_group=hit["force_group"])
    return hit
