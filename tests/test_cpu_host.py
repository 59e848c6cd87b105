"""CPU-only checks: the C-ABI library loads and exports every declared entry
point, the ctypes struct layouts match the C ones, and the host-side logic
(cell grid, Morton order, rc^2 formation, EAM file parsing and table
construction, LJ constants) agrees with the oracle.  No GPU compute calls."""
import ctypes
import os
import re

import numpy as np
import pytest
import torch

from oracle import eam as oeam
from oracle import inputs as oin
from oracle import neighbor as onb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    from simulon_b200 import build, _lib
    build.build()
    return _lib.load()


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "simb200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int64_t|int|const char\*)\s+(sim_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol(lib):
    from simulon_b200 import _lib
    names = declared_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, f"{name} not bound in simulon_b200._lib"


def test_struct_layouts_match(lib):
    from simulon_b200 import _lib
    out = np.zeros(len(_lib.STRUCTS), np.int64)
    assert lib.sim_struct_sizes(out.ctypes.data, len(_lib.STRUCTS)) == 0
    assert list(out) == [ctypes.sizeof(s) for s in _lib.STRUCTS]
    assert lib.sim_version() == 1


def test_argument_errors_are_reported_without_gpu(lib):
    from simulon_b200 import _lib
    assert lib.sim_rebuild(None, 0, None) == _lib.SIM_ERR_ARG
    assert lib.sim_legacy_density_pass(None, None, None, None, 0, None, 1, 1.0, 1, None, None) == _lib.SIM_ERR_ARG
    assert lib.sim_legacy_density_pass(None, None, None, None, 0, None, 1, 1.0, 8, None, None) == _lib.SIM_OK
    # the fused step, LJ and Berendsen entry points check their arguments before any device work
    assert lib.sim_eam_step_drift(None, None, None, None, 0, None, 0, None) == _lib.SIM_ERR_ARG
    assert lib.sim_lj_forces_integrate(None, None, None, 1, None) == _lib.SIM_ERR_ARG
    assert lib.sim_berendsen_mu(None, None, None, None) == _lib.SIM_ERR_ARG
    assert lib.sim_berendsen_scale_first(None, None, None, None, 0, None) == _lib.SIM_ERR_ARG
    assert lib.sim_eam_force_integrate_indenter(None, None, None, None, 1, None) == _lib.SIM_ERR_ARG
    assert lib.sim_eam_step_drift_indenter(None, None, None, None, None, 0, None, 0, None) == _lib.SIM_ERR_ARG
    assert lib.sim_scan_i64(None, 5, None, None) == _lib.SIM_ERR_ARG
    assert lib.sim_scan_i64(None, -1, None, None) == _lib.SIM_ERR_ARG
    e, p, ip = _lib.SimEngine(), _lib.SimLJParams(), _lib.SimIntegrator()
    e.n = 10
    for mode in (0, 3):   # only 1 (second half) and 2 (with the next first half)
        assert lib.sim_lj_forces_integrate(ctypes.byref(e), ctypes.byref(p), ctypes.byref(ip), mode, None) == \
            _lib.SIM_ERR_ARG
    # the summed-LJ and loader-bookkeeping entry points
    assert lib.sim_lj_forces_add(None, None, None) == _lib.SIM_ERR_ARG
    assert lib.sim_lj_forces_add(ctypes.byref(_lib.SimEngine()), ctypes.byref(p), None) == _lib.SIM_ERR_ARG
    chk = _lib.SimLoaderCheck()
    assert lib.sim_loader_check(None, ctypes.byref(chk), None, None) == _lib.SIM_ERR_ARG
    for axis, strain, margin in ((3, 0.01, 0.01), (-1, 0.01, 0.01), (0, -1.0, 0.01), (0, 0.01, -0.5)):
        chk.axis, chk.rebuild_strain, chk.regrid_margin = axis, strain, margin
        assert lib.sim_loader_check(ctypes.byref(e), ctypes.byref(chk), ctypes.c_void_p(16), None) == \
            _lib.SIM_ERR_ARG
    # the fused tensile pieces
    assert lib.sim_aniso_control(None, None, None, None) == _lib.SIM_ERR_ARG
    bs = _lib.SimBoxScale()
    bs.scale[:] = [1.0, 1.0, 1.0]
    bs.vel_scale[:] = [1.0, 0.0, 1.0]     # a non-positive factor
    assert lib.sim_box_scale_after_first(ctypes.byref(e), ctypes.c_void_p(16), 1, ctypes.byref(bs),
                                         ctypes.c_void_p(16), ctypes.byref(ip), 0, None) == _lib.SIM_ERR_ARG
    assert lib.sim_box_scale_after_first(None, None, 1, None, None, None, 0, None) == _lib.SIM_ERR_ARG
    # the linked tensile step: a missing piece, a bad loader scale or a bad loader check, before any launch
    an = _lib.SimAniso()
    assert lib.sim_tensile_link(None, None, None, None, None, 0, None, 0, None, None, None, 0, None, None,
                                None) == _lib.SIM_ERR_ARG
    assert lib.sim_tensile_link(ctypes.byref(e), ctypes.byref(an), ctypes.c_void_p(16), None, None, 0,
                                ctypes.c_void_p(16), 8, ctypes.byref(bs), ctypes.c_void_p(16), ctypes.byref(ip), 0,
                                ctypes.byref(chk), ctypes.c_void_p(16), None) == _lib.SIM_ERR_ARG
    # EAM tables of 2^22 rows or more are refused (the kernels' row truncation is exact below that)
    tb = _lib.SimEAMTables()
    for name in ("density", "density_deriv", "pair", "pair_deriv", "embed", "embed_deriv", "rho_min", "inv_drho",
                 "rho_clamp_hi", "dens_vd", "deriv_vd", "pair_vd"):
        setattr(tb, name, 16)
    tb.n_types, tb.n_r, tb.n_rho = 1, 1 << 22, 100
    e.n_types, e.posfp = 1, 16
    assert lib.sim_eam_density(ctypes.byref(e), ctypes.byref(tb), None) == _lib.SIM_ERR_ARG
    assert lib.sim_eam_atom_energy(ctypes.byref(e), ctypes.byref(tb), ctypes.c_void_p(16), None) == _lib.SIM_ERR_ARG
    with pytest.raises(_lib.SimError):
        _lib.check(_lib.SIM_ERR_ARG, "probe")


def test_xyz_rows_match_python_formatting(lib):
    """The trajectory row formatter (host code of the library) against
    Python's f"{v:.6f}": random magnitudes, exact ties (ties to even),
    signed zeros, tiny and subnormal values, large values and non-finite ones."""
    rng = np.random.default_rng(5)
    edge = [0.0, -0.0, 0.0078125, -0.0078125, 0.0234375, 1.0000005, 2.5e-7, -2.5e-7, 4.9999995e-7, 123456.0000005,
            1e-300, -1e-300, 5e-324, 1.5, 2.0 ** 39 + 0.1, 2.0 ** 40 + 0.5, 1e15, -1e15, float("inf"),
            float("-inf"), float("nan"), -float("nan"), 999999.9999995, -0.0000005]
    vals = np.concatenate([rng.normal(0, 50, 3000), rng.uniform(-1e6, 1e6, 600), rng.normal(0, 1e-5, 600),
                           np.ldexp(rng.integers(-2 ** 20, 2 ** 20, 600).astype(np.float64), -20), edge])
    vals = np.concatenate([vals, np.zeros((-len(vals)) % 3)])
    xyz = np.ascontiguousarray(vals.reshape(-1, 3))
    types = (np.arange(len(xyz)) % 2).astype(np.int32)
    syms = (ctypes.c_char_p * 2)(b"W", b"Ar")
    buf = np.empty(len(xyz) * 220, np.uint8)
    nb = lib.sim_format_xyz_rows(xyz.ctypes.data, types.ctypes.data, len(xyz), syms, 2, buf.ctypes.data, buf.size)
    want = "".join(f"{('W', 'Ar')[t]} {x:.6f} {y:.6f} {z:.6f}\n" for t, (x, y, z) in zip(types, xyz.tolist()))
    assert nb == len(want.encode()) and bytes(buf[:nb]).decode() == want
    assert lib.sim_format_xyz_rows(xyz.ctypes.data, None, len(xyz), syms, 2, buf.ctypes.data, 100) == -1


def test_cell_grid_and_morton_order():
    from simulon_b200.engine import cell_grid, morton_rank, estimate_capacity, perpendicular_widths
    L = 80 * 3.165
    nc = cell_grid(np.diag([L] * 3), 4.9, 1_024_000)
    assert list(nc) == [51, 51, 51]
    H = oin.triclinic_box(L)
    w = perpendicular_widths(H)
    assert np.all(w / cell_grid(H, 4.9, 1_024_000) >= 4.9)
    r, lin = morton_rank(np.array([5, 6, 7]))
    assert sorted(r.tolist()) == list(range(210)) and np.array_equal(r[lin], np.arange(210))
    # consecutive ranks are spatial neighbours most of the time
    cx, cy, cz = lin % 5, (lin // 5) % 6, lin // 30
    steps = np.abs(np.diff(cx)) + np.abs(np.diff(cy)) + np.abs(np.diff(cz))
    assert np.mean(steps == 1) > 0.5
    assert estimate_capacity(16000, np.diag([63.3] * 3), 4.9) >= 32
    assert list(cell_grid(np.diag([15.78] * 3), 7.5, 108)) == [2, 2, 2]


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_reference_rc2(dtype):
    from simulon_b200.neighbor import reference_rc2
    cut = torch.tensor(4.4, dtype=dtype) + torch.tensor(0.5, dtype=dtype)
    npd = np.float32 if dtype == torch.float32 else np.float64
    assert reference_rc2(cut, dtype) == onb.rc2_like_reference(4.4, 0.5, npd)


@pytest.fixture(scope="module")
def pot(tmp_path_factory):
    return oin.write_fs_w_setfl(str(tmp_path_factory.mktemp("pot") / "W_synthetic.eam.fs"))


def test_eam_parser_matches_oracle(pot):
    from simulon_b200 import EAMParser
    a, b = EAMParser(pot), oeam.parse_eam(pot)
    assert a.elements == b.elements and a.is_fs_format == b.is_fs_format and a.cutoff == b.cutoff
    for name in ("embedding_splines", "density_splines", "density_deriv_splines"):
        assert np.array_equal(getattr(a, name)[0].c, getattr(b, name)[0].c)
    assert np.array_equal(a.pair_potential_splines[0][0].c, b.pair_potential_splines[0][0].c)


def test_device_tables_match_oracle_fp64(pot):
    from simulon_b200 import EAMParser, EAMDeviceTables
    t = EAMDeviceTables(EAMParser(pot), "cpu")
    o = oeam.EAMTables(oeam.parse_eam(pot), dtype=torch.float64)
    for mine, theirs in (("density", o.density), ("density_deriv", o.density_deriv), ("pair", o.pair),
                         ("pair_deriv", o.pair_deriv), ("embed", o.embed), ("embed_deriv", o.embed_deriv)):
        np.testing.assert_allclose(t.host64[mine], theirs.numpy(), rtol=1e-13, atol=1e-12)
    assert abs(t.inv_dr - o.inv_dr) < 1e-9 and t.rho_min64[0] == o.rho_min[0]


def test_alloy_and_setfl_formats(tmp_path):
    """Two-element eam/alloy and single-element setfl files parse like the oracle."""
    from simulon_b200 import EAMParser
    nr, nrho = 200, 150
    r = np.arange(nr) * 0.03
    rho = np.arange(nrho) * 0.2
    lines = ["c1", "c2", "c3", "2 Ni Al", f"{nrho} 0.2 {nr} 0.03 5.97", "28 58.69 3.52 fcc"]
    blocks = [-np.sqrt(rho), np.exp(-r), "13 26.98 4.05 fcc", -0.8 * np.sqrt(rho), 0.7 * np.exp(-r),
              r * np.exp(-2 * r), r * 0.5 * np.exp(-2 * r), r * 0.25 * np.exp(-2 * r)]
    for b in blocks:
        if isinstance(b, str):
            lines.append(b)
        else:
            lines += [" ".join(repr(float(v)) for v in b[k:k + 4]) for k in range(0, len(b), 4)]
    path = tmp_path / "NiAl.eam.alloy"
    path.write_text("\n".join(lines) + "\n")
    a, b = EAMParser(str(path)), oeam.parse_eam(str(path))
    assert a.elements == ["Ni", "Al"] and not a.is_fs_format and not b.is_fs_format
    assert np.array_equal(a.pair_potential_splines[0][1].c, b.pair_potential_splines[0][1].c)
    assert np.array_equal(a.density_splines_by_pair[0][1].c, b.density_splines_by_pair[0][1].c)


def test_lj_constants_follow_reference_float32():
    from simulon_b200.forces import lj_type_pair_params
    p = lj_type_pair_params({"[0 0]": {"epsilon": 0.0104, "sigma": 3.405}}, 1, 7.0, "cpu")
    eps = torch.tensor([0.0104], dtype=torch.float32)
    assert float(p["c24eps"]) == float(24.0 * eps)            # formed in float32, as the reference
    assert float(p["sigma"]) == float(np.float32(3.405))
    sr = torch.tensor([3.405], dtype=torch.float32) / 7.0
    assert float(p["f_rc"]) == float(24.0 * eps * (1.0 / 7.0) * (2.0 * (sr ** 6) ** 2 - sr ** 6))


def test_product_path_refuses_cpu():
    import simulon_b200 as sb
    x, L = oin.bcc_lattice(3)
    with pytest.raises(RuntimeError):
        sb.MDEngine(x, np.zeros(len(x), np.int32), [oin.W_MASS], np.diag([L] * 3), 4.4, 0.5, device="cpu")


def test_package_references_resolve():
    """Every `_lib.<name>` / `engine.<name>` attribute the package uses exists
    (these modules cannot be exercised end to end without a GPU)."""
    import ast
    import glob
    from simulon_b200 import _lib, engine
    mods = {"_lib": _lib}
    missing = []
    for path in glob.glob(os.path.join(ROOT, "simulon_b200", "*.py")) + [os.path.join(ROOT, "bench.py")]:
        tree = ast.parse(open(path).read())
        for node in ast.walk(tree):
            if isinstance(node, ast.Attribute) and isinstance(node.value, ast.Name) and node.value.id in mods:
                if not hasattr(mods[node.value.id], node.attr):
                    missing.append(f"{os.path.basename(path)}: {node.value.id}.{node.attr}")
    assert not missing, missing
    # status bits mirror the header
    hdr = open(os.path.join(ROOT, "include", "simb200.h")).read()
    for name in ("SIM_OK", "SIM_ERR_ARG", "SIM_ERR_CUDA", "SIM_STATUS_OVERFLOW", "SIM_STATUS_NONFINITE",
                 "SIM_STATUS_HALO", "SIM_STATUS_MLP_NEIGHBORS", "SIM_STATUS_MLP_TIMEOUT"):
        val = int(re.search(rf"#define {name}\s+(\d+)", hdr).group(1))
        assert getattr(_lib, name) == val, name
    assert engine.TILE == int(re.search(r"#define SIM_TILE\s+(\d+)", hdr).group(1))


def test_clock_summary_keeps_samples_of_the_timed_region():
    """The bench's clock record: samples between entering and leaving the
    timed region, the next later one when the region was shorter than the
    sampling interval, throttle reasons from the "Active" columns."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)

    def row(mhz, power_cap="Not Active", thermal="Not Active"):
        return f"0, {mhz}, 1965, 700.0, 0x0, Not Active, Not Active, {thermal}, {power_cap}"

    c = bench.ClockSampler("GPU-x")
    c.t0, c.t1 = 10.0, 11.0
    c.lines = [(9.9, row(300)), (10.2, row(1965)), (10.5, row(1900, power_cap="Active")), (10.8, row(1965)),
               (11.1, row(300, thermal="Active"))]
    s = c.summary()
    assert s == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3, "in_region": 3}
    c.lines = [(9.9, row(300)), (11.05, row(1950)), (11.15, row(1000))]
    s = c.summary()
    assert s["sm_mhz"] == 1950.0 and s["samples"] == 1 and s["in_region"] == 0
    c.lines = []
    assert c.summary()["samples"] == 0
