"""Descriptor-MLP surrogate of the EAM force field (C ABI group 4).

No counterpart in the reference: this is the learned form of the force path.
Per atom: 8 radial and 8 angular symmetry-function descriptors of the
in-cutoff neighbourhood (r < 4.4 A, cosine cutoff), a 16 -> 64 -> 64 -> 1 SiLU
network for the atom's energy (BF16 operands on the tensor cores, FP32
accumulation), forces = -dE/dx through network and descriptors.

* ``MLPNet`` holds the FP32 parameters and their BF16 operand images.
* ``MLPEnergy`` / ``mlp_energy``: the energy as a ``torch.autograd.Function``
  whose backward is the library's force kernel.
* ``MLPForce`` is a force-field backbone with the ``BackboneInterface``
  contract of the reference (core/md_model.py:9-12): energy, forces.
* ``generate_dataset`` runs the engine's EAM at several temperatures and
  strains and records descriptors with per-atom EAM energies.
* ``train`` fits the network on the GPU with the library's own forward,
  backward and Adam kernels.
* ``SurrogateRun`` advances a system with MLP forces and checks them against
  EAM every ``judge_every`` steps, switching to EAM when the force RMSE
  exceeds ``tolerance``.
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np
import torch

from . import _lib
from .engine import MDEngine, integrator_params

N_DESC, N_HID = 16, 64
OFF = dict(W1=(0, (16, 64)), b1=(1024, (64,)), W2=(1088, (64, 64)), b2=(5184, (64,)), w3=(5248, (64,)),
           b3=(5312, ()))
N_PARAMS = 5313


class MLPNet:
    """Parameters (one FP32 device array) + descriptor normalisation + BF16 images."""

    def __init__(self, device=None, params: dict | None = None, seed: int = 0):
        self.device = torch.device(device or "cuda")
        if self.device.type != "cuda":
            raise RuntimeError("MLPNet runs on CUDA devices only (no CPU fallback)")
        self.lib = _lib.load()
        self.flat = torch.zeros(N_PARAMS, device=self.device, dtype=torch.float32)
        self.mu = torch.zeros(N_DESC, device=self.device, dtype=torch.float32)
        self.inv_sigma = torch.ones(N_DESC, device=self.device, dtype=torch.float32)
        self.images = [torch.zeros(n, device=self.device, dtype=torch.int16) for n in (1024, 4096, 4096, 1024)]
        self.status = torch.zeros(1, device=self.device, dtype=torch.int32)
        if params is None:
            params = init_params(seed)
        self.load_dict(params)

    # ---- parameters ------------------------------------------------------
    def load_dict(self, p: dict):
        flat = np.zeros(N_PARAMS, np.float32)
        for k, (o, shp) in OFF.items():
            flat[o:o + int(np.prod(shp)) if shp else o + 1] = np.asarray(p[k], np.float32).reshape(-1)
        self.flat.copy_(torch.from_numpy(flat))
        if "mu" in p:
            self.mu.copy_(torch.as_tensor(np.asarray(p["mu"], np.float32)))
        if "sigma" in p:
            self.inv_sigma.copy_(torch.as_tensor(1.0 / np.asarray(p["sigma"], np.float32)))
        self.pack()

    def to_dict(self) -> dict:
        flat = self.flat.cpu().numpy()
        out = {k: flat[o:o + int(np.prod(shp))].reshape(shp) if shp else flat[o:o + 1].reshape(())
               for k, (o, shp) in OFF.items()}
        out["mu"] = self.mu.cpu().numpy()
        out["sigma"] = 1.0 / self.inv_sigma.cpu().numpy()
        return {k: np.asarray(v, np.float64) for k, v in out.items()}

    def save(self, path: str):
        np.savez(path, **self.to_dict())

    @classmethod
    def load(cls, path: str, device=None) -> "MLPNet":
        with np.load(path) as z:
            return cls(device, {k: z[k] for k in z.files})

    def set_normalisation(self, G: torch.Tensor):
        """Descriptor mean and standard deviation from rows of G."""
        G = G.float()
        self.mu.copy_(G.mean(0))
        self.inv_sigma.copy_(1.0 / G.std(0).clamp_min(1e-6))

    def pack(self):
        p = _lib.ptr
        _lib.call("sim_mlp_pack", p(self.flat), *(p(t) for t in self.images), self._stream())
        self._make_struct()

    def _make_struct(self):
        s = _lib.SimMLP()
        p = _lib.ptr
        s.w1t_img, s.w2t_img, s.w2_img, s.w1_img = (p(t) for t in self.images)
        base = self.flat.data_ptr()
        s.b1, s.b2 = base + 4 * OFF["b1"][0], base + 4 * OFF["b2"][0]
        s.w3, s.b3 = base + 4 * OFF["w3"][0], base + 4 * OFF["b3"][0]
        s.mu, s.inv_sigma = p(self.mu), p(self.inv_sigma)
        self.st = s
        self.ref = ctypes.byref(s)

    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    # ---- kernels -----------------------------------------------------------
    def forward(self, G: torch.Tensor, n: int):
        """(E_i [n], dE/dG [n,16]) for the first n rows of G [>=n, 16] FP32."""
        e = torch.empty(n, device=self.device, dtype=torch.float32)
        d = torch.empty(n, N_DESC, device=self.device, dtype=torch.float32)
        _lib.call("sim_mlp_forward", self.ref, _lib.ptr(G), int(n), _lib.ptr(e), _lib.ptr(d), _lib.ptr(self.status),
                  self._stream())
        return e, d

    def forward_into(self, G: torch.Tensor, n: int, e: torch.Tensor, d: torch.Tensor):
        """forward() into preallocated e [>=n] and d [>=n,16] (no allocation)."""
        _lib.call("sim_mlp_forward", self.ref, _lib.ptr(G), int(n), _lib.ptr(e), _lib.ptr(d), _lib.ptr(self.status),
                  self._stream())

    def train_grads(self, G: torch.Tensor, target: torch.Tensor, grads: torch.Tensor, loss: torch.Tensor):
        _lib.call("sim_mlp_train_grads", self.ref, _lib.ptr(G), _lib.ptr(target), int(target.numel()),
                  _lib.ptr(grads), _lib.ptr(loss), _lib.ptr(self.status), self._stream())

    def train_step(self, G: torch.Tensor, target: torch.Tensor, n: int, grads: torch.Tensor, adam_m: torch.Tensor,
                   adam_v: torch.Tensor, lr: float, step: int, loss: torch.Tensor, u: torch.Tensor | None = None,
                   w_energy: float = 1.0, w_force: float = 1.0, n_force_atoms: int = 0):
        """Gradient (energy only, or energy and force matching along u), Adam
        step and BF16 repack in one library call."""
        p = _lib.ptr
        _lib.call("sim_mlp_train_step", self.ref, p(self.flat), *(p(t) for t in self.images), p(G), p(target),
                  p(u) if u is not None else None, int(n), float(w_energy), float(w_force),
                  int(n_force_atoms or n), p(grads), p(adam_m), p(adam_v), float(lr), int(step), p(loss),
                  p(self.status), self._stream())

    def train_grads_fm(self, G: torch.Tensor, target: torch.Tensor, u: torch.Tensor, n: int, w_energy: float,
                       w_force: float, n_force_atoms: int, grads: torch.Tensor, loss: torch.Tensor):
        """Gradient of w_energy * mean (E - target)^2 + the force-matching term
        whose descriptor contraction is u [n,16] (see ``force_contract``)."""
        _lib.call("sim_mlp_train_grads_fm", self.ref, _lib.ptr(G), _lib.ptr(target), _lib.ptr(u), int(n),
                  float(w_energy), float(w_force), int(n_force_atoms), _lib.ptr(grads), _lib.ptr(loss),
                  _lib.ptr(self.status), self._stream())


def init_params(seed: int = 0) -> dict:
    rng = np.random.default_rng(seed)
    return dict(W1=rng.normal(0, 1 / math.sqrt(N_DESC), (N_DESC, N_HID)), b1=np.zeros(N_HID),
                W2=rng.normal(0, 1 / math.sqrt(N_HID), (N_HID, N_HID)), b2=np.zeros(N_HID),
                w3=rng.normal(0, 1 / math.sqrt(N_HID), N_HID), b3=np.array(0.0),
                mu=np.zeros(N_DESC), sigma=np.ones(N_DESC))


def descriptors(engine: MDEngine) -> torch.Tensor:
    """G [n_pad, 16] of the engine's slots."""
    G = torch.zeros(engine.n_pad, N_DESC, device=engine.device, dtype=torch.float32)
    _lib.call("sim_mlp_descriptors", engine.st_ref, _lib.ptr(G), engine.stream)
    return G


def mlp_forces(engine: MDEngine, dEdG: torch.Tensor):
    """-dE/dx of every slot into engine.f32 from dE/dG [n, 16]."""
    _lib.call("sim_mlp_backward", engine.st_ref, _lib.ptr(dEdG), engine.stream)
    engine._last_force_precision = 0
    engine.forces_valid = True


def force_contract(engine: MDEngine, ferr: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
    """u [n_pad,16] with u_i = sum_m ferr_m . dG_i/dx_m, from per-slot force
    errors ferr [n_pad,4] (x, y, z, unused)."""
    u = out if out is not None else torch.zeros(engine.n_pad, N_DESC, device=engine.device, dtype=torch.float32)
    _lib.call("sim_mlp_force_contract", engine.st_ref, _lib.ptr(ferr), _lib.ptr(u), engine.stream)
    return u


def eam_atom_energy(engine: MDEngine, tables) -> torch.Tensor:
    """Per-atom EAM energies of the engine's slots [n_pad]."""
    out = torch.zeros(engine.n_pad, device=engine.device, dtype=torch.float32)
    _lib.call("sim_eam_atom_energy", engine.st_ref, tables.ref, _lib.ptr(out), engine.stream)
    return out


class MLPEnergy(torch.autograd.Function):
    """Total surrogate energy of positions x [N,3] (original atom order) as a
    differentiable torch function.  forward: the engine is loaded with x
    (cell sort and list build), then descriptors, network and the backward
    kernels run; backward: dE/dx = -forces, times the incoming gradient."""

    @staticmethod
    def forward(ctx, x, engine, net):
        engine.set_positions(x.detach())
        G = descriptors(engine)
        e, d = net.forward(G, engine.n)
        mlp_forces(engine, d)
        ctx.save_for_backward(-engine.gather("f").to(x.dtype))
        return e.sum().to(x.dtype)

    @staticmethod
    def backward(ctx, grad_out):
        (dEdx,) = ctx.saved_tensors
        return grad_out * dEdx, None, None


def mlp_energy(x: torch.Tensor, engine: MDEngine, net: MLPNet) -> torch.Tensor:
    """E(x) with forces = -dE/dx from the library's backward kernels."""
    return MLPEnergy.apply(x, engine, net)


class MLPForce:
    """Force-field backbone with MLP energies and forces (BackboneInterface contract)."""

    def __init__(self, net: MLPNet, molecular):
        self.net = net
        self.molecular = molecular
        self.force_precision = 0

    def compute(self):
        eng = self.molecular.engine
        G = descriptors(eng)
        e, d = self.net.forward(G, eng.n)
        mlp_forces(eng, d)
        self.atom_energy = e

    def __call__(self):
        return self.forward()

    def forward(self):
        self.compute()
        eng = self.molecular.engine
        return {"energy": self.atom_energy.sum(), "forces": eng.gather("f").to(self.molecular.dtype)}


# ---------------------------------------------------------------------------
# training data and training

def bcc_cell(n: int, a: float = 3.165):
    g = np.arange(n)
    cells = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0.5]])
    return (cells[:, None, :] + basis[None]).reshape(-1, 3).astype(np.float64) * a


def generate_dataset(tables, *, n_cells: int = 10, temperatures=(300.0, 700.0, 1100.0, 1500.0),
                     strains=(-0.03, 0.0, 0.03), frames_per_run: int = 20, stride: int = 20,
                     equilibrate: int = 200, dt: float = 0.001, seed: int = 0, device=None,
                     with_forces: bool = False):
    """Descriptors and per-atom EAM energies (and optionally EAM forces and
    positions) of frames from Langevin runs of BCC W (2 n^3 atoms) at each
    temperature and isotropic strain."""
    dev = torch.device(device or "cuda")
    rng = np.random.default_rng(seed)
    Gs, Es, frames = [], [], []
    a0 = 3.165
    for T in temperatures:
        for eps in strains:
            a = a0 * (1.0 + eps + rng.uniform(-0.005, 0.005))
            x = bcc_cell(n_cells, a)
            L = n_cells * a
            m = 183.84 * 1.036427e-4
            v = rng.normal(0.0, math.sqrt(8.617333262e-5 * T / m), x.shape)
            eng = MDEngine(x, np.zeros(len(x), np.int32), [183.84], np.diag([L] * 3), 4.4, 0.5, velocities=v,
                           device=dev)
            ip = integrator_params(eng, dt, langevin=True, temperature=T, gamma=10.0, seed=int(rng.integers(1 << 30)))
            eng.eam_forces(tables)

            def advance(k):
                for _ in range(k):
                    eng.integrate_first(ip, 0)
                    eng.rebuild_if_needed()
                    eng.eam_forces_integrate(tables, ip)
            advance(equilibrate)
            for _ in range(frames_per_run):
                advance(stride)
                eng.eam_forces(tables)
                G = descriptors(eng)[:eng.n].clone()
                E = eam_atom_energy(eng, tables)[:eng.n].clone()
                Gs.append(G)
                Es.append(E)
                if with_forces:
                    frames.append(dict(x=eng.gather("x").cpu().numpy(), f=eng.gather("f").cpu().numpy(), H=np.diag([L] * 3)))
            if eng.status() & ~_lib.SIM_STATUS_MLP_NEIGHBORS:
                raise RuntimeError(f"EAM run for training data failed (status {eng.status():#x})")
    G = torch.cat(Gs)
    E = torch.cat(Es)
    return (G, E, frames) if with_forces else (G, E)


def train(net: MLPNet, G: torch.Tensor, E: torch.Tensor, *, steps: int = 2000, batch: int = 16384,
          lr: float = 3e-3, lr_final: float = 1e-4, seed: int = 0, log_every: int = 0):
    """Per-atom energy regression with Adam, all on the GPU.  Returns the
    per-step losses (device tensor)."""
    dev = net.device
    n = G.shape[0]
    net.set_normalisation(G)
    with torch.no_grad():
        p = net.to_dict()
        p["b3"] = np.array(float(E.double().mean()))
        net.load_dict(p)
    grads = torch.zeros(N_PARAMS, device=dev, dtype=torch.float32)
    m1 = torch.zeros_like(grads)
    m2 = torch.zeros_like(grads)
    loss = torch.zeros(1, device=dev, dtype=torch.float32)
    losses = torch.zeros(steps, device=dev, dtype=torch.float32)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    Gb = torch.empty(batch, N_DESC, device=dev, dtype=torch.float32)
    Eb = torch.empty(batch, device=dev, dtype=torch.float32)
    for s in range(steps):
        idx = torch.randint(0, n, (batch,), device=dev, generator=gen)
        torch.index_select(G, 0, idx, out=Gb)
        torch.index_select(E, 0, idx, out=Eb)
        lr_s = lr * (lr_final / lr) ** (s / max(1, steps - 1))
        net.train_step(Gb, Eb, batch, grads, m1, m2, lr_s, s + 1, loss)
        losses[s:s + 1].copy_(loss)
        if log_every and (s + 1) % log_every == 0:
            print(f"step {s + 1}: loss {float(loss):.3e} eV^2", flush=True)
    if int(net.status.item()):
        raise RuntimeError(f"tensor-core wait timed out in training (status {int(net.status.item()):#x})")
    return losses


class ForceFrame:
    """One EAM reference configuration for force matching: an engine holding
    its positions and neighbour list, the descriptors G [n_pad,16], per-atom
    EAM energies E [n] and EAM forces F [n_pad,4], all in the engine's slot order."""

    def __init__(self, x, H, tables, device=None):
        eng = MDEngine(x, np.zeros(len(x), np.int32), [183.84], H, 4.4, 0.5, device=device)
        eng.eam_forces(tables)
        self.F = eng.f32.clone()
        self.E = eam_atom_energy(eng, tables)[:eng.n].clone()
        self.G = descriptors(eng)
        self.engine = eng
        if eng.status() & ~_lib.SIM_STATUS_MLP_NEIGHBORS:
            raise RuntimeError(f"EAM reference frame failed (status {eng.status():#x})")


class FramePool:
    """Frames of BCC-W cells (2 n_cells^3 atoms) from the engine's own EAM
    runs: n_runs Langevin runs, each at a temperature drawn uniformly from
    t_range and under a diagonal strain with components drawn uniformly from
    +-strain; every `stride`-th step after `equilibrate` steps is a frame.
    Kept per frame: positions (FP64, device), and for energy regression the
    descriptors G and per-atom EAM energies E (rows concatenated over frames).
    pool[k] loads frame k into its run's engine and returns a ForceFrame-like
    view with the EAM forces and energies of those positions as targets
    (buffers reused by the next pool[k])."""

    def __init__(self, tables, *, n_frames: int = 20000, n_cells: int = 10, n_runs: int = 40, stride: int = 10,
                 equilibrate: int = 200, t_range=(300.0, 1500.0), strain: float = 0.03, dt: float = 0.001,
                 seed: int = 0, device=None):
        dev = torch.device(device or "cuda")
        rng = np.random.default_rng(seed)
        self.tables = tables
        self.engines, self.run_T, self.run_strain = [], [], []
        per_run = [n_frames // n_runs + (1 if r < n_frames % n_runs else 0) for r in range(n_runs)]
        x0 = bcc_cell(n_cells)
        n = len(x0)
        self.n = n
        self.X = torch.empty(n_frames, n, 3, device=dev, dtype=torch.float64)
        self.G = torch.empty(n_frames * n, N_DESC, device=dev, dtype=torch.float32)
        self.E = torch.empty(n_frames * n, device=dev, dtype=torch.float32)
        self.run_of = np.empty(n_frames, np.int64)
        m = 183.84 * 1.036427e-4
        f = 0
        for r in range(n_runs):
            T = float(rng.uniform(*t_range))
            eps = rng.uniform(-strain, strain, 3)
            H = np.diag(n_cells * 3.165 * (1.0 + eps))
            x = x0 * (1.0 + eps)
            v = rng.normal(0.0, math.sqrt(8.617333262e-5 * T / m), x.shape)
            eng = MDEngine(x, np.zeros(n, np.int32), [183.84], H, 4.4, 0.5, velocities=v, device=dev)
            ip = integrator_params(eng, dt, langevin=True, temperature=T, gamma=10.0, seed=int(rng.integers(1 << 30)))
            eng.eam_forces(tables)

            def advance(k):
                for _ in range(k):
                    eng.integrate_first(ip, 0)
                    eng.rebuild_if_needed()
                    eng.eam_forces_integrate(tables, ip)
            advance(equilibrate)
            for _ in range(per_run[r]):
                advance(stride)
                eng.eam_forces(tables)
                self.X[f].copy_(eng.gather("x"))
                self.G[f * n:(f + 1) * n].copy_(descriptors(eng)[:n])
                self.E[f * n:(f + 1) * n].copy_(eam_atom_energy(eng, tables)[:n])
                self.run_of[f] = r
                f += 1
            if eng.status() & ~_lib.SIM_STATUS_MLP_NEIGHBORS:
                raise RuntimeError(f"EAM run for training data failed (status {eng.status():#x})")
            self.engines.append(eng)
            self.run_T.append(T)
            self.run_strain.append(eps)
        P = self.engines[0].n_pad
        self._F = torch.zeros(P, 4, device=dev, dtype=torch.float32)
        self._Et = torch.zeros(P, device=dev, dtype=torch.float32)
        self._G = torch.zeros(P, N_DESC, device=dev, dtype=torch.float32)

    def __len__(self):
        return self.X.shape[0]

    def __getitem__(self, k):
        eng = self.engines[int(self.run_of[k])]
        eng.load(self.X[k])
        eng.eam_forces(self.tables)
        self._F.copy_(eng.f32)
        self._Et.copy_(eam_atom_energy(eng, self.tables))
        _lib.call("sim_mlp_descriptors", eng.st_ref, _lib.ptr(self._G), eng.stream)

        class View:
            pass
        fr = View()
        fr.engine, fr.G, fr.E, fr.F = eng, self._G, self._Et[:eng.n], self._F
        return fr


def train_forces(net: MLPNet, frames, *, steps: int = 4000, lr: float = 1e-3, lr_final: float = 1e-4,
                 w_energy: float = 1.0, w_force: float = 1.0, frames_per_step: int = 1, seed: int = 0,
                 log_every: int = 0):
    """Energy and force matching with Adam on ``frames`` (a list of
    ``ForceFrame`` or a ``FramePool``), frames_per_step frames per step (their
    gradients averaged): loss per frame = w_energy mean_i (E_i - E_i^EAM)^2
                                       + w_force sum_m |F_m - F_m^EAM|^2 / (3 n).
    The network keeps its normalisation (train on energies first).  Returns
    the per-step force mean squares (device tensor, (eV/A)^2)."""
    dev = net.device
    grads = torch.zeros(N_PARAMS, device=dev, dtype=torch.float32)
    gsum = torch.zeros_like(grads)
    m1 = torch.zeros_like(grads)
    m2 = torch.zeros_like(grads)
    loss = torch.zeros(1, device=dev, dtype=torch.float32)
    fmse = torch.zeros(steps, device=dev, dtype=torch.float32)
    P = max(fr.engine.n_pad for fr in frames) if isinstance(frames, list) else frames.engines[0].n_pad
    e = torch.zeros(P, device=dev, dtype=torch.float32)
    d = torch.zeros(P, N_DESC, device=dev, dtype=torch.float32)
    ferr = torch.zeros(P, 4, device=dev, dtype=torch.float32)
    u = torch.zeros(P, N_DESC, device=dev, dtype=torch.float32)
    B = max(1, int(frames_per_step))
    order = np.random.default_rng(seed).permutation(steps * B) % len(frames)
    st = torch.cuda.current_stream(dev).cuda_stream
    for s in range(steps):
        gsum.zero_()
        for b in range(B):
            fr = frames[int(order[s * B + b])]
            eng = fr.engine
            n, np_ = eng.n, eng.n_pad
            net.forward_into(fr.G, n, e, d)
            _lib.call("sim_mlp_backward", eng.st_ref, _lib.ptr(d), eng.stream)
            fe = ferr[:np_]
            torch.sub(eng.f32, fr.F, out=fe)
            fmse[s] += fe[:n, :3].square().mean() / B
            _lib.call("sim_mlp_force_contract", eng.st_ref, _lib.ptr(fe), _lib.ptr(u), eng.stream)
            net.train_grads_fm(fr.G, fr.E, u, n, w_energy / B, w_force / B, n, grads, loss)
            gsum += grads
        lr_s = lr * (lr_final / lr) ** (s / max(1, steps - 1))
        _lib.call("sim_mlp_adam", _lib.ptr(net.flat), _lib.ptr(gsum), _lib.ptr(m1), _lib.ptr(m2), float(lr_s), s + 1,
                  st)
        _lib.call("sim_mlp_pack", _lib.ptr(net.flat), *(_lib.ptr(t) for t in net.images), st)
        if log_every and (s + 1) % log_every == 0:
            print(f"step {s + 1}: force RMSE {math.sqrt(float(fmse[s + 1 - log_every:s + 1].mean())):.4f} eV/A, "
                  f"energy loss {float(loss):.3e} eV^2", flush=True)
    if int(net.status.item()):
        raise RuntimeError(f"tensor-core wait timed out in training (status {int(net.status.item()):#x})")
    return fmse


def force_rmse(net: MLPNet, tables, frames, device=None) -> float:
    """RMSE of MLP forces against the recorded EAM forces of frames."""
    dev = torch.device(device or "cuda")
    se, cnt = 0.0, 0
    for fr in frames:
        eng = MDEngine(fr["x"], np.zeros(len(fr["x"]), np.int32), [183.84], fr["H"], 4.4, 0.5, device=dev)
        G = descriptors(eng)
        _, d = net.forward(G, eng.n)
        mlp_forces(eng, d)
        f = eng.gather("f").cpu().numpy()
        se += float(((f - fr["f"]) ** 2).sum())
        cnt += f.size
    return math.sqrt(se / max(cnt, 1))


def default_weights_path() -> str:
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "w_surrogate.npz")


class SurrogateRun:
    """MD of one system with MLP forces, judged against EAM.

    Every ``judge_every`` steps the EAM forces of the current positions are
    compared with the MLP forces; when their RMSE exceeds ``tolerance``
    (eV/A) the run continues with EAM forces.  Steps between judgements are
    captured in a CUDA graph: first half-step and conditional rebuild, then
    per step descriptors, network and forces followed by one pass that
    finishes the step and starts the next (Langevin when the integrator
    parameters say so), the last step ending with a plain second half."""

    def __init__(self, engine: MDEngine, net: MLPNet, tables, integ, *, judge_every: int = 100,
                 tolerance: float = 0.05):
        self.eng, self.net, self.tables, self.integ = engine, net, tables, integ
        self.judge_every, self.tolerance = int(judge_every), float(tolerance)
        n = engine.n
        self.G = torch.zeros(engine.n_pad, N_DESC, device=engine.device, dtype=torch.float32)
        self.e = torch.zeros(n, device=engine.device, dtype=torch.float32)
        self.d = torch.zeros(n, N_DESC, device=engine.device, dtype=torch.float32)
        self.use_mlp = True
        self.rmse_history: list[float] = []
        self._graph = None
        self._mlp_forces()

    def _mlp_forces(self):
        eng = self.eng
        _lib.call("sim_mlp_descriptors", eng.st_ref, _lib.ptr(self.G), eng.stream)
        self.net.forward_into(self.G, eng.n, self.e, self.d)
        _lib.call("sim_mlp_backward", eng.st_ref, _lib.ptr(self.d), eng.stream)

    def _chunk(self, k: int):
        """k steps, launches only: the second half of each step but the last
        runs together with the first half of the next (same forces)."""
        eng = self.eng
        eng.integrate_first(self.integ, 0)
        eng.rebuild_if_needed()
        for s in range(k):
            last = s == k - 1
            if self.use_mlp:
                self._mlp_forces()
                if last:
                    eng.integrate_second(self.integ, 0)
                else:
                    eng.integrate_second_first(self.integ, 0)
            elif last:
                eng.eam_forces_integrate(self.tables, self.integ)
            else:
                eng.eam_forces_integrate_drift(self.tables, self.integ)
            if not last:
                eng.rebuild_if_needed()

    def judge(self) -> float:
        """Force RMSE of MLP against EAM at the current positions (synchronises);
        leaves the forces of the model in use in the engine."""
        eng = self.eng
        f_mlp = eng.gather("f")
        eng.eam_forces(self.tables)
        f_eam = eng.gather("f")
        rmse = float(torch.sqrt(((f_mlp - f_eam) ** 2).mean()))
        self.rmse_history.append(rmse)
        if rmse > self.tolerance:
            self.use_mlp = False
            self._graph = None
        else:
            self._mlp_forces()
        return rmse

    def run(self, n_steps: int, judge: bool = True):
        done = 0
        while done < n_steps:
            k = min(self.judge_every, n_steps - done)
            if k == self.judge_every:
                if self._graph is None:
                    s = torch.cuda.Stream(self.eng.device)
                    s.wait_stream(torch.cuda.current_stream(self.eng.device))
                    g = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(g, stream=s):
                        self._chunk(k)
                    torch.cuda.current_stream(self.eng.device).wait_stream(s)
                    self._graph = g
                self._graph.replay()
            else:
                self._chunk(k)
            done += k
            if judge and self.use_mlp and k == self.judge_every:
                self.judge()
        return self


TRAINING_NOTE = ("python -m simulon_b200.mlp: 20,000 frames of 2,000-atom BCC-W cells from 40 Langevin EAM runs "
                 "(T uniform in 300-1500 K, diagonal strain uniform in +-3 %, every 10th step of dt 1 fs after 200), "
                 "per-atom EAM energies and EAM forces as targets; 20,000 Adam steps of energy regression "
                 "(16,384 atoms each), then 12,000 steps of energy + force matching (4 frames each)")


def main(argv=None):
    """Train the surrogate on the engine's EAM data and save its weights:
    python -m simulon_b200.mlp POTENTIAL OUT.npz [--frames F] [--steps N] [--fm-steps M] ...
    Energy regression on per-atom EAM energies first, then energy and force
    matching on whole frames (targets recomputed from the frame's positions)."""
    import argparse
    import time
    from .eam_parser import EAMDeviceTables, EAMParser
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("potential")
    ap.add_argument("out")
    ap.add_argument("--frames", type=int, default=20000, help="training frames")
    ap.add_argument("--runs", type=int, default=40, help="EAM runs the frames come from")
    ap.add_argument("--cells", type=int, default=10, help="BCC cells per side (2 n^3 atoms per frame)")
    ap.add_argument("--stride", type=int, default=10, help="MD steps between frames")
    ap.add_argument("--steps", type=int, default=20000, help="energy-regression steps")
    ap.add_argument("--batch", type=int, default=16384, help="atoms per energy-regression step")
    ap.add_argument("--fm-steps", type=int, default=12000, help="force-matching steps")
    ap.add_argument("--fm-batch", type=int, default=4, help="frames per force-matching step")
    ap.add_argument("--w-force", type=float, default=1.0)
    ap.add_argument("--lr-fm", type=float, default=1e-3)
    a = ap.parse_args(argv)
    dev = torch.device("cuda")
    tables = EAMDeviceTables(EAMParser(a.potential), dev)
    t0 = time.perf_counter()
    pool = FramePool(tables, n_frames=a.frames, n_cells=a.cells, n_runs=a.runs, stride=a.stride, seed=0,
                     device=dev)
    val = {}
    for T, seed in ((300.0, 99), (1500.0, 98)):
        _, _, raw = generate_dataset(tables, n_cells=a.cells, temperatures=(T,), strains=(0.0,), frames_per_run=2,
                                     stride=40, equilibrate=200, seed=seed, device=dev, with_forces=True)
        val[T] = raw
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    net = MLPNet(dev, seed=0)
    losses = train(net, pool.G, pool.E, steps=a.steps, batch=a.batch, log_every=max(1, a.steps // 10))
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    before = {T: force_rmse(net, tables, fr, dev) for T, fr in val.items()}
    fmse = train_forces(net, pool, steps=a.fm_steps, lr=a.lr_fm, w_force=a.w_force, frames_per_step=a.fm_batch,
                        log_every=max(1, a.fm_steps // 10)) if a.fm_steps else torch.zeros(1)
    torch.cuda.synchronize()
    t3 = time.perf_counter()
    after = {T: force_rmse(net, tables, fr, dev) for T, fr in val.items()}
    net.save(a.out)
    print(f"frames {len(pool)} x {pool.n} atoms from {len(pool.engines)} runs "
          f"(T {min(pool.run_T):.0f}-{max(pool.run_T):.0f} K); data {t1 - t0:.1f} s, "
          f"energy fit {t2 - t1:.1f} s, force fit {t3 - t2:.1f} s")
    print(f"energy loss {float(losses[-100:].mean()):.3e} eV^2, force MSE (last 5%) "
          f"{float(fmse[-max(1, len(fmse) // 20):].mean()):.3e} (eV/A)^2")
    for T in val:
        print(f"validation force RMSE at {T:.0f} K: {before[T]:.4f} (energy fit) -> {after[T]:.4f} eV/A")
    print(f"-> {a.out}")


if __name__ == "__main__":
    main()

