"""Host logic of the launch-shape autotuner (simulon_b200/autotune.py): cache
keys, the JSON cache and how results reach SimEngine.launch, with the C ABI
calls replaced by a fake that writes timings through the pointers."""
import ctypes

import numpy as np
import torch

from simulon_b200 import autotune


class FakeEngine:
    def __init__(self, n=1000, nbar=26.2):
        self.n = n
        self.n_pad = ((n + 127) // 128) * 128
        self.nnbr = torch.full((self.n_pad,), int(round(nbar)), dtype=torch.int32)
        self.device = torch.device("cpu")
        self.st_ref = None
        self.stream = 0
        self.launch = [0, 0, 0, 0]

    def set_launch(self, eam_density_threads=None, eam_force_threads=None, mlp_desc_group=None,
                   mlp_force_group=None):
        for k, v in enumerate((eam_density_threads, eam_force_threads, mlp_desc_group, mlp_force_group)):
            if v is not None:
                self.launch[k] = int(v)


def _fake_call(calls):
    def call(name, *args):
        calls.append(name)
        if name == "sim_autotune_eam":
            ms_p, best_p = args[3], args[4]
            ms = (ctypes.c_float * 6).from_address(ms_p)
            ms[:] = [0.30, 0.20, 0.25, 0.5, 0.4, 0.45]
            best = (ctypes.c_int32 * 2).from_address(best_p)
            best[:] = [256, 512]
        elif name == "sim_autotune_mlp":
            ms_p, best_p = args[4], args[5]
            ms = (ctypes.c_float * 4).from_address(ms_p)
            ms[:] = [0.4, 0.3, 0.6, 0.7]
            best = (ctypes.c_int32 * 2).from_address(best_p)
            best[:] = [8, 4]
        return 0
    return call


def test_tune_caches_and_applies(tmp_path, monkeypatch):
    calls = []
    monkeypatch.setattr(autotune._lib, "call", _fake_call(calls))
    monkeypatch.setattr(autotune._lib, "ptr", lambda t: t.data_ptr())
    monkeypatch.setattr(torch.cuda, "get_device_name", lambda dev=None: "FakeGPU")

    class Tables:
        ref = None
    path = str(tmp_path / "shapes.json")
    eng = FakeEngine()
    hit = autotune.tune_eam(eng, Tables(), path=path)
    assert hit["density_threads"] == 256 and hit["force_threads"] == 512
    assert eng.launch[:2] == [256, 512]
    assert abs(hit["ms"]["density_256"] - 0.2) < 1e-6
    hit = autotune.tune_mlp(eng, path=path)
    assert eng.launch[2:] == [8, 4]
    assert calls == ["sim_autotune_eam", "sim_autotune_mlp"]
    # a second engine of the same size reads the cache: no further timing calls
    eng2 = FakeEngine()
    autotune.tune_eam(eng2, Tables(), path=path)
    autotune.tune_mlp(eng2, path=path)
    assert calls == ["sim_autotune_eam", "sim_autotune_mlp"]
    assert eng2.launch == [256, 512, 8, 4]
    # another size is a new key
    autotune.tune_eam(FakeEngine(n=2000), Tables(), path=path)
    assert calls[-1] == "sim_autotune_eam" and len(calls) == 3
    keys = sorted(__import__("json").load(open(path)))
    assert keys == ["FakeGPU|eam|1000|26", "FakeGPU|eam|2000|26", "FakeGPU|mlp|1000|26"]


def test_cache_path_from_environment(monkeypatch, tmp_path):
    monkeypatch.setenv("SIMB200_TUNE_CACHE", str(tmp_path / "x.json"))
    assert autotune.cache_path() == str(tmp_path / "x.json")
    assert autotune._load(str(tmp_path / "missing.json")) == {}
    (tmp_path / "bad.json").write_text("{not json")
    assert autotune._load(str(tmp_path / "bad.json")) == {}
    np.testing.assert_equal(autotune.EAM_FORCE_THREADS, (256, 512, 1024))
