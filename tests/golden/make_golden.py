"""Generate golden vectors by running the reference implementation itself.

Run from the repository root in a container where the reference checkout is
available (default path below, or SIMULON_REFERENCE=<dir>):

    python tests/golden/make_golden.py

The reference is imported unmodified; two third-party imports it makes at
module level but does not use on this path (pymatgen.core and
torch_geometric.data.Data) are replaced by minimal stand-ins.  Inputs come
from the seeded generators in ``oracle.inputs``.  Each case is written as a
small .npz next to this script; the tests read only those files.
"""
from __future__ import annotations

import json
import os
import sys
import tempfile
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
REF = os.environ.get("SIMULON_REFERENCE", "/root/reference")

from oracle import inputs as oin  # noqa: E402
from oracle.philox import langevin_normals  # noqa: E402


def _stub_imports():
    pm = types.ModuleType("pymatgen")
    pmc = types.ModuleType("pymatgen.core")

    class _Placeholder:  # never instantiated on the hot path
        pass

    pmc.Structure = _Placeholder
    pmc.Lattice = _Placeholder
    sys.modules.setdefault("pymatgen", pm)
    sys.modules.setdefault("pymatgen.core", pmc)
    tg = types.ModuleType("torch_geometric")
    tgd = types.ModuleType("torch_geometric.data")

    class Data:
        def __init__(self, **kw):
            for k, v in kw.items():
                setattr(self, k, v)

        def get(self, k, default=None):
            return getattr(self, k, default)

    tgd.Data = Data
    sys.modules.setdefault("torch_geometric", tg)
    sys.modules.setdefault("torch_geometric.data", tgd)
    sys.path.insert(0, REF)


def _reader(tmp, name, coords, symbol, box, cutoff, skin, params=None, is_fs=False):
    from io_utils.reader import AtomFileReader
    path = oin.write_xyz(os.path.join(tmp, name + ".xyz"), coords, symbol)
    H = np.asarray(box, dtype=np.float64)
    kw = {}
    if H.ndim == 2:
        kw["box_vectors"] = torch.tensor(H)
        bl = float(np.linalg.norm(H[0]))
    else:
        bl = float(H) if H.ndim == 0 else H.tolist()
    return AtomFileReader(filename=path, box_length=bl, cutoff=cutoff, device=torch.device("cpu"),
                          parameter=params, skin_thickness=skin, is_fs=is_fs, **kw)


def _save(name, **arrays):
    out = {k: (v.detach().cpu().numpy() if torch.is_tensor(v) else np.asarray(v)) for k, v in arrays.items()}
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"wrote {name}.npz  ({', '.join(f'{k}{list(np.shape(v))}' for k, v in out.items())})")


def neighbor_cases(tmp):
    cases = []
    x, L = oin.fcc_lattice(3)
    cases.append(("nbr_ar108_f64", oin.jitter(x, 0.05, 0), L, 7.0, 0.5, torch.float64))
    x, L = oin.bcc_lattice(5)
    cases.append(("nbr_w250_f32", oin.jitter(x, 0.05, 2), L, 4.4, 0.5, torch.float32))
    x, H = oin.bcc_triclinic(6)
    cases.append(("nbr_wtri432_f32", oin.jitter(x, 0.05, 3), H, 4.4, 0.5, torch.float32))
    cases.append(("nbr_wtri432_f64", oin.jitter(x, 0.05, 3), H, 4.4, 0.5, torch.float64))
    rng = np.random.default_rng(4)
    box = np.array([20.0, 22.0, 25.0])
    gas = rng.uniform(-0.5, 1.5, size=(300, 3)) * box      # unwrapped, partly outside the box
    cases.append(("nbr_gas300_orth_f32", gas, np.diag(box), 4.0, 1.0, torch.float32))
    cases.append(("nbr_pair2_f64", np.array([[0.1, 0.2, 0.3], [9.9, 0.2, 0.3]]), 10.0, 3.0, 0.5, torch.float64))
    cases.append(("nbr_far3_f32", np.array([[0.0, 0.0, 0.0], [5.0, 5.0, 5.0], [5.0, 0.0, 5.0]]), 12.0, 2.0, 0.5, torch.float32))
    for name, coords, box, rc, skin, dt in cases:
        torch.set_default_dtype(dt)
        try:
            mol = _reader(tmp, name, coords, "W", box, rc, skin, is_fs=True)
            ei = mol.graph_data.edge_index
            _save(name, pos=mol.coordinates, box=mol.box.H, cutoff=rc, skin=skin,
                  i=ei[0], j=ei[1], dist=mol.graph_data.edge_attr)
        finally:
            torch.set_default_dtype(torch.float32)


def lj_cases(tmp):
    from core.force.lennard_jones_force import LennardJonesForce
    torch.set_default_dtype(torch.float64)
    try:
        x, L = oin.fcc_lattice(3)
        x = oin.jitter(x, 0.05, 0)
        params = {"[0 0]": {"epsilon": 0.0104, "sigma": 3.405}}
        for mode in ("raw", "fs", "switch"):
            mol = _reader(tmp, "ar108", x, "Ar", L, 7.0, 0.5, params=params)
            mol.is_fs = mode == "fs"
            mol.is_switch = mode == "switch"
            out = LennardJonesForce(mol)()
            ei = mol.graph_data.edge_index
            _save(f"lj_ar108_{mode}_f64", pos=mol.coordinates, box=mol.box.H, i=ei[0], j=ei[1],
                  eps=mol.pair_params[0], sigma=mol.pair_params[1], rc=7.0, rs=0.9 * 7.0,
                  energy=out["energy"], forces=out["forces"], virial=out["virial"],
                  virial_tensor=out["virial_tensor"])
    finally:
        torch.set_default_dtype(torch.float32)


def eam_cases(tmp):
    from io_utils.eam_parser import EAMParser
    from core.force.eam_force_cu import EAMForceCUDAExt
    pot = oin.write_fs_w_setfl(os.path.join(tmp, "W_synthetic.eam.fs"))
    parser = EAMParser(pot, torch.device("cpu"))
    x, L = oin.bcc_lattice(5)
    for name, coords in (("eam_w250_jitter_f32", oin.jitter(x, 0.05, 5)), ("eam_w250_perfect_f32", x)):
        mol = _reader(tmp, name, coords, "W", L, parser.cutoff, 0.5, is_fs=True)
        ff = EAMForceCUDAExt(parser, mol, use_extension=False)
        out = ff()
        ei = mol.graph_data.edge_index
        _save(name, pos=mol.coordinates, box=mol.box.H, i=ei[0], j=ei[1], dist=mol.graph_data.edge_attr,
              energy=out["energy"], forces=out["forces"], virial=out["virial"],
              virial_tensor=out["virial_tensor"], embedding_energy=out["embedding_energy"],
              pair_potential=out["pair_potential"],
              density_table=ff.density_table[0, 0], density_deriv_table=ff.density_deriv_table[0, 0],
              pair_table=ff.pair_table[0, 0], pair_deriv_table=ff.pair_deriv_table[0, 0],
              embed_table=ff.embed_table[0], embed_deriv_table=ff.embed_deriv_table[0])
    xt, H = oin.bcc_triclinic(6)
    mol = _reader(tmp, "eam_wtri432_f32", oin.jitter(xt, 0.05, 6), "W", H, parser.cutoff, 0.5, is_fs=True)
    out = EAMForceCUDAExt(parser, mol, use_extension=False)()
    ei = mol.graph_data.edge_index
    _save("eam_wtri432_f32", pos=mol.coordinates, box=mol.box.H, i=ei[0], j=ei[1],
          energy=out["energy"], forces=out["forces"], virial=out["virial"], virial_tensor=out["virial_tensor"])


class _NoisePatch:
    """Replace torch.randn_like with Philox normals so a run can be replayed."""

    def __init__(self, seed):
        self.seed, self.step, self.orig = seed, 0, None

    def __enter__(self):
        self.orig = torch.randn_like

        def fake(t, *a, **k):
            z = torch.as_tensor(langevin_normals(t.shape[0], self.step, self.seed)).to(t.dtype)
            self.step += 1
            return z
        torch.randn_like = fake
        return self

    def __exit__(self, *exc):
        torch.randn_like = self.orig


def md_cases(tmp):
    from core.force.lennard_jones_force import LennardJonesForce
    from core.force.eam_force_cu import EAMForceCUDAExt
    from core.integrator.integrator import VerletIntegrator
    from core.md_model import BaseModel, SumBackboneInterface
    from core.barostat import BerendsenBarostat
    from io_utils.eam_parser import EAMParser

    # LJ argon, FP64, NVE and Langevin NVT (config 1 inputs), 30 steps each.
    torch.set_default_dtype(torch.float64)
    try:
        x, L = oin.fcc_lattice(3)
        x = oin.jitter(x, 0.05, 0)
        v0 = oin.maxwell_boltzmann(np.full(len(x), oin.AR_MASS), 94.4, 1)
        params = {"[0 0]": {"epsilon": 0.0104, "sigma": 3.405}}
        for ens in ("NVE", "NVT"):
            mol = _reader(tmp, "ar108md", x, "Ar", L, 7.0, 0.5, params=params)
            integ = VerletIntegrator(mol, dt=0.002, ensemble=ens,
                                     temperature=(94.4, 94.4) if ens == "NVT" else None,
                                     gamma=10.0 if ens == "NVT" else None)
            mol.atom_velocities = torch.tensor(v0)
            model = BaseModel(SumBackboneInterface([LennardJonesForce(mol)], mol), integ, mol)
            rec = {k: [] for k in ("energy", "kinetic_energy", "temperature")}
            with _NoisePatch(seed=1234):
                for _ in range(30):
                    out = model()
                    for k in rec:
                        rec[k].append(float(out[k]))
            _save(f"md_ar108_{ens.lower()}_f64", x0=x, v0=v0, box=L, dt=0.002, steps=30, noise_seed=1234,
                  T=94.4, gamma=10.0, x=mol.coordinates, v=mol.atom_velocities, forces=out["forces"],
                  rebuilds=mol.profile["neighbor_builds"],
                  **{k: np.array(v) for k, v in rec.items()})
    finally:
        torch.set_default_dtype(torch.float32)

    # EAM-W 250 FP32: NVE and Berendsen NPT (the reference EAM path is FP32 only).
    pot = oin.write_fs_w_setfl(os.path.join(tmp, "W_synthetic.eam.fs"))
    parser = EAMParser(pot, torch.device("cpu"))
    x, L = oin.bcc_lattice(5)
    x = oin.jitter(x, 0.02, 7)
    v0 = oin.maxwell_boltzmann(np.full(len(x), oin.W_MASS), 300.0, 8)
    for ens in ("NVE", "NPT"):
        mol = _reader(tmp, "w250md", x, "W", L, parser.cutoff, 0.5, is_fs=True)
        integ = VerletIntegrator(mol, dt=0.002, ensemble=ens,
                                 temperature=(300.0, 300.0) if ens == "NPT" else None,
                                 gamma=10.0 if ens == "NPT" else None)
        mol.atom_velocities = torch.tensor(v0, dtype=torch.float32)
        baro = BerendsenBarostat(mol, target_pressure=0.0, tau_p=0.5) if ens == "NPT" else None
        model = BaseModel(SumBackboneInterface([EAMForceCUDAExt(parser, mol, use_extension=False)], mol),
                          integ, mol, barostat=baro)
        rec = {k: [] for k in ("energy", "kinetic_energy", "temperature", "pressure")}
        with _NoisePatch(seed=99):
            for _ in range(20):
                out = model()
                for k in rec:
                    if k in out:
                        rec[k].append(float(out[k]))
        _save(f"md_w250_{ens.lower()}_f32", x0=x, v0=v0, box0=L, box=mol.box.H, dt=0.002, steps=20,
              noise_seed=99, T=300.0, gamma=10.0, tau_p=0.5, x=mol.coordinates, v=mol.atom_velocities,
              rebuilds=mol.profile["neighbor_builds"], **{k: np.array(v) for k, v in rec.items() if v})


def mech_cases(tmp):
    """Tensile-workflow callers of the force path (LJ argon 108, FP64, NVE, 20
    steps): UniaxialTensileLoader on axis 0 with the AnisotropicNPTBarostat on
    the lateral axes (run_scripts/w_tensile.py's stress-free mode), and the
    barostat alone on all axes towards 500 bar."""
    from core.force.lennard_jones_force import LennardJonesForce
    from core.integrator.integrator import VerletIntegrator
    from core.md_model import BaseModel, SumBackboneInterface
    from core.barostat import AnisotropicNPTBarostat
    from core.mechanics.loading import UniaxialTensileLoader

    torch.set_default_dtype(torch.float64)
    try:
        x, L = oin.fcc_lattice(3)
        x = oin.jitter(x, 0.05, 0)
        v0 = oin.maxwell_boltzmann(np.full(len(x), oin.AR_MASS), 94.4, 1)
        params = {"[0 0]": {"epsilon": 0.0104, "sigma": 3.405}}
        cases = {
            "tensile": (dict(axis=0, strain_rate=2.0, lateral_mode="fixed"),
                        dict(target_pressure_bar=[0.0, 0.0, 0.0], control_axes=(False, True, True))),
            "aniso": (None, dict(target_pressure_bar=[500.0, 500.0, 500.0], control_axes=(True, True, True))),
        }
        for name, (load, baro_kw) in cases.items():
            mol = _reader(tmp, f"ar108{name}", x, "Ar", L, 7.0, 0.5, params=params)
            integ = VerletIntegrator(mol, dt=0.002, ensemble="NVE")
            mol.atom_velocities = torch.tensor(v0)
            baro = AnisotropicNPTBarostat(mol, temperature_k=94.4, tau_p=0.2, gamma_p=2.0,
                                          compressibility_bar_inv=3.2e-5, pressure_tolerance_bar=25.0, **baro_kw)
            model = BaseModel(SumBackboneInterface([LennardJonesForce(mol)], mol), integ, mol, barostat=baro)
            loader = UniaxialTensileLoader(mol, **load) if load else None
            rec = {k: [] for k in ("energy", "kinetic_energy", "pressure", "strain", "H", "eta_dot")}
            for _ in range(20):
                rec["strain"].append(loader.step(0.002) if loader else 0.0)
                out = model()
                rec["energy"].append(float(out["energy"]))
                rec["kinetic_energy"].append(float(out["kinetic_energy"]))
                rec["pressure"].append(out["pressure"].detach().numpy().copy())
                rec["H"].append(mol.box.H.detach().numpy().copy())
                rec["eta_dot"].append(baro.eta_dot.detach().numpy().copy())
            _save(f"mech_ar108_{name}_f64", x0=x, v0=v0, box0=L, dt=0.002, steps=20, x=mol.coordinates,
                  v=mol.atom_velocities, rebuilds=mol.profile["neighbor_builds"],
                  load=np.array(json.dumps(load)), baro=np.array(json.dumps(baro_kw)),
                  **{k: np.array(v) for k, v in rec.items()})
    finally:
        torch.set_default_dtype(torch.float32)


def indenter_cases(tmp):
    """LJ argon 108 (FP64, NVE, 20 steps) with the SphericalIndenterForce as a
    second backbone, its centre lowered 0.05 A per step into the top layer."""
    from core.force.lennard_jones_force import LennardJonesForce
    from core.integrator.integrator import VerletIntegrator
    from core.md_model import BaseModel, SumBackboneInterface
    from core.mechanics.indenter import SphericalIndenterForce

    torch.set_default_dtype(torch.float64)
    try:
        x, L = oin.fcc_lattice(3)
        x = oin.jitter(x, 0.05, 0)
        v0 = oin.maxwell_boltzmann(np.full(len(x), oin.AR_MASS), 94.4, 1)
        params = {"[0 0]": {"epsilon": 0.0104, "sigma": 3.405}}
        mol = _reader(tmp, "ar108ind", x, "Ar", L, 7.0, 0.5, params=params)
        integ = VerletIntegrator(mol, dt=0.002, ensemble="NVE")
        mol.atom_velocities = torch.tensor(v0)
        R, K = 4.0, 0.05
        c0 = np.array([0.5 * L, 0.5 * L, float(np.max(x[:, 2])) + R - 0.5])
        ind = SphericalIndenterForce(mol, radius=R, stiffness=K, center=c0)
        model = BaseModel(SumBackboneInterface([LennardJonesForce(mol), ind], mol), integ, mol)
        rec = {k: [] for k in ("energy", "kinetic_energy", "virial", "virial_tensor", "force_on_indenter",
                               "indenter_energy", "contact_atoms", "center")}
        for s in range(20):
            c = c0 - np.array([0.0, 0.0, 0.05 * s])
            ind.set_center(c)
            out = model()
            rec["energy"].append(float(out["energy"]))
            rec["kinetic_energy"].append(float(out["kinetic_energy"]))
            rec["virial"].append(float(out["virial"]))
            rec["virial_tensor"].append(out["virial_tensor"].detach().numpy().copy())
            rec["force_on_indenter"].append(ind.force_on_indenter.detach().numpy().copy())
            rec["indenter_energy"].append(float(ind.last_energy))
            rec["contact_atoms"].append(int(ind.contact_atoms))
            rec["center"].append(c)
        _save("ind_ar108_f64", x0=x, v0=v0, box0=L, dt=0.002, steps=20, radius=R, stiffness=K, x=mol.coordinates,
              v=mol.atom_velocities, **{k: np.array(v) for k, v in rec.items()})
    finally:
        torch.set_default_dtype(torch.float32)


def crack_cases(tmp):
    """Crack observables of run_scripts/w_crack.py (_select_mouth_groups,
    _estimate_crack_length, _project_to_lattice_axes) on a precracked BCC-W
    slab as built and with its upper half opened (a smooth opening profile
    around the crack plus seeded jitter), and the stress projection of a
    seeded symmetric tensor."""
    for name in ("matplotlib", "matplotlib.pyplot"):
        if name not in sys.modules:
            m = types.ModuleType(name)
            m.use = lambda *a, **k: None
            m.rcParams = {}
            sys.modules[name] = m
    sys.modules["matplotlib"].pyplot = sys.modules["matplotlib.pyplot"]
    from run_scripts.w_crack import _estimate_crack_length, _project_to_lattice_axes, _select_mouth_groups
    from simulon_b200.batch import crack_slab

    rep = crack_slab(3000, seed=5)
    H = torch.tensor(rep.H)
    x0 = torch.tensor(rep.positions)
    x_unit = H[0] / torch.linalg.norm(H[0])
    y_unit = H[1] / torch.linalg.norm(H[1])
    yc = float(rep.meta["crack_plane_y"])
    half = float(rep.meta["crack_half_length"])
    vx, vy = x0 @ x_unit, x0 @ y_unit
    x_min, x_max = float(vx.min()), float(vx.max())
    xc = 0.5 * (x_min + x_max)
    up, lo = _select_mouth_groups(vx, vy, xc, yc, half)
    cmod0 = float(vy[up].mean() - vy[lo].mean())
    rng = np.random.default_rng(6)
    x1 = x0.clone()
    sel = vy > yc
    open_by = 1.8 * torch.exp(-((vx - xc) / (1.6 * half)) ** 2)
    x1[sel, 1] += open_by[sel]
    x1 += torch.tensor(rng.normal(0.0, 0.05, x1.shape))
    res = {}
    for tag, xx in (("0", x0), ("1", x1)):
        L, ext = _estimate_crack_length(xx, x_unit, y_unit, yc, x_min, x_max, xc, half, 1.0, 160)
        vyy = xx @ y_unit
        res[f"length{tag}"], res[f"extension{tag}"] = L, ext
        res[f"cmod{tag}"] = float(vyy[up].mean() - vyy[lo].mean()) - cmod0
    A = rng.normal(0.0, 1.0e4, (3, 3))
    sigma = torch.tensor(A + A.T)
    proj = _project_to_lattice_axes(sigma, types.SimpleNamespace(H=H))
    _save("crack_obs_w3000", x0=x0, x1=x1, H=H, crack_plane_y=yc, half_length=half, upper=up.numpy(),
          lower=lo.numpy(), sigma=sigma, projected=proj, threshold=1.0, bins=160, **res)


def main():
    if not os.path.isdir(REF):
        raise SystemExit(f"reference checkout not found at {REF}")
    _stub_imports()
    import builtins
    quiet = builtins.print
    with tempfile.TemporaryDirectory() as tmp:
        builtins.print = lambda *a, **k: None if str(a[0] if a else "").startswith("[EAM") else quiet(*a, **k)
        try:
            neighbor_cases(tmp)
            lj_cases(tmp)
            eam_cases(tmp)
            md_cases(tmp)
            mech_cases(tmp)
            indenter_cases(tmp)
            crack_cases(tmp)
        finally:
            builtins.print = quiet


if __name__ == "__main__":
    main()
