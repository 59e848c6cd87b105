"""Mechanics callers of the force path: uniaxial tensile loading
(core/mechanics/loading.py:6-81) and the spherical indenter backbone
(core/mechanics/indenter.py:7-68).

Loader:
The box update runs on the device in FP64 (``sim_box_scale``): H <- diag(s) H,
positions through fractional coordinates of the old box into the new one and
wrapped (box.py:132-142), posq refreshed, the skin test against the last
rebuild, and the reference's reset of last_positions.  ``step`` returns the
engineering strain of the loading axis as a Python float (it reads the
device box, which also holds a barostat's changes of the other axes).

Beyond the reference: the cell grid is rebuilt before the box shrinks below
rc + skin per cell (``MDEngine.regrid``, asked for by the device with a
margin), and the list is rebuilt whenever the box has strained by more than
a quarter of the skin over the list cutoff since the last such rebuild (the
skin test compares fractional positions, which an affine box change leaves
unchanged).  That bookkeeping runs on the device, so loader and MD steps can
be captured together in CUDA graphs.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib
from .forces import BackboneInterface, _force_outputs


class UniaxialTensileLoader:
    """Uniaxial loading (loading.py:6-81): each step scales the loading axis
    of the box by 1 + strain_rate dt (and, with lateral_mode "poisson", the
    other axes by the Poisson contraction) and maps the atoms through
    fractional coordinates, on the device.  The step's bookkeeping runs on the
    device too (``sim_loader_check``): the engineering strain, the list
    rebuild forced after an affine strain of a quarter of the skin over the
    list cutoff, and the request to regrid before the cells become narrower
    than the list cutoff.

    ``step(dt)`` keeps the reference's contract (returns the engineering
    strain as a float, so it synchronises and regrids when asked).
    ``launch(dt)`` only enqueues the work (returns the strain as a device
    scalar), so ``model.run(n, pre_step=...)`` can capture loader and MD
    steps together in CUDA graphs; ``run(model, n_steps, dt)`` does that in
    chunks and regrids between them (``maintain``).  With an anisotropic
    barostat the model then runs the barostat's atom scaling of step s, the
    loader's update and the first half of step s+1 as one pass
    (``launch_after``)."""

    def __init__(self, molecular, axis: int = 0, strain_rate: float = 1.0e-3, lateral_mode: str = "fixed",
                 poisson_ratio: float = 0.28, max_lateral_scale_step: float = 2.0e-3, regrid_margin: float = 0.01,
                 regrid_headroom: float = 0.06):
        self.molecular = molecular
        self.axis = int(axis)
        self.strain_rate = float(strain_rate)
        self.lateral_mode = str(lateral_mode).lower()
        self.poisson_ratio = float(poisson_ratio)
        self.max_lateral_scale_step = float(max_lateral_scale_step)
        self.regrid_margin = float(regrid_margin)
        self.regrid_headroom = max(float(regrid_headroom), self.regrid_margin)
        if self.axis not in (0, 1, 2):
            raise ValueError(f"axis must be 0/1/2, got {axis}")
        if not hasattr(molecular, "engine"):
            raise NotImplementedError("UniaxialTensileLoader requires a device-resident molecular (engine)")
        if self.lateral_mode not in ("fixed", "poisson"):
            raise ValueError(f"unsupported lateral_mode={lateral_mode}")
        eng = molecular.engine
        H = eng.box_matrix()
        self.initial_lengths = torch.tensor(np.linalg.norm(H, axis=1), dtype=torch.float64)
        self.total_engineering_strain = 0.0
        self.work = torch.zeros(_lib.BOXSCALE_WORK, dtype=torch.float64, device=eng.device)
        self.state = torch.zeros(_lib.LOADER_STATE, dtype=torch.float64, device=eng.device)
        self._reset_list_box(H)
        self.state[9:12] = self.initial_lengths.to(eng.device)
        skin = 2.0 * math.sqrt(float(eng.st.skin_half2))
        self._check = _lib.SimLoaderCheck()
        self._check.axis = self.axis
        self._check.rebuild_strain = 0.25 * skin / float(eng.x_rc)
        self._check.regrid_margin = self.regrid_margin
        self._hooks = {}
        self.regrids = 0

    def _reset_list_box(self, H):
        self.state[0:9] = torch.as_tensor(np.asarray(H, np.float64).reshape(-1), dtype=torch.float64)

    def _scale_vector(self, dt: float) -> list:
        dstrain = self.strain_rate * float(dt)
        scale = [1.0, 1.0, 1.0]
        scale[self.axis] = 1.0 + dstrain
        if self.lateral_mode == "poisson":
            lat = max(1.0 - self.poisson_ratio * dstrain, 1.0 - self.max_lateral_scale_step)
            for ax in range(3):
                if ax != self.axis:
                    scale[ax] = lat
        return scale

    def launch(self, dt: float) -> torch.Tensor:
        """The box update and its bookkeeping, launches only (capturable)."""
        eng = self.molecular.engine
        s = _lib.SimBoxScale()
        s.scale[:] = self._scale_vector(dt)
        s.vel_scale[:] = [1.0, 1.0, 1.0]
        s.reset_reference = 1
        _lib.call("sim_box_scale", eng.st_ref, ctypes.byref(s), _lib.ptr(self.work), eng.stream)
        _lib.call("sim_loader_check", eng.st_ref, ctypes.byref(self._check), _lib.ptr(self.state), eng.stream)
        return self.state[12]

    def launch_after(self, barostat, integrator, dt: float) -> torch.Tensor:
        """The next step's start in one pass: the barostat's box update prepared
        by barostat.controller(), this loader's update, and integrator's
        first half (sim_box_scale_after_first), then the bookkeeping and the
        conditional rebuild; the same bits as barostat.step(), launch(dt) and
        integrator.first_half() one after another."""
        eng = self.molecular.engine
        s = _lib.SimBoxScale()
        s.scale[:] = self._scale_vector(dt)
        s.vel_scale[:] = [1.0, 1.0, 1.0]
        s.reset_reference = 1
        _lib.call("sim_box_scale_after_first", eng.st_ref, _lib.ptr(barostat.work), int(barostat._st.reset_reference),
                  ctypes.byref(s), _lib.ptr(self.work), integrator.params.ref, int(integrator.force_precision),
                  eng.stream)
        _lib.call("sim_loader_check", eng.st_ref, ctypes.byref(self._check), _lib.ptr(self.state), eng.stream)
        eng.rebuild_if_needed()
        return self.state[12]

    def link(self, barostat, integrator, dt: float) -> torch.Tensor:
        """The end of this step and the start of the next with an anisotropic
        barostat, in one call (sim_tensile_link): the barostat's controller,
        the step's log row, then launch_after's work; the same bits as
        barostat.controller(dt), the engine's log_step() and
        launch_after(barostat, integrator, dt) one after another, in three
        kernels instead of seven."""
        eng = self.molecular.engine
        barostat._st.dt = float(integrator.dt)
        s = _lib.SimBoxScale()
        s.scale[:] = self._scale_vector(dt)
        s.vel_scale[:] = [1.0, 1.0, 1.0]
        s.reset_reference = 1
        _lib.call("sim_tensile_link", eng.st_ref, barostat._ref, _lib.ptr(barostat.work), _lib.ptr(eng.step_ctr),
                  _lib.ptr(eng.extra), int(eng.extra.numel()), _lib.ptr(eng.log), eng.log_capacity, ctypes.byref(s),
                  _lib.ptr(self.work), integrator.params.ref, int(integrator.force_precision),
                  ctypes.byref(self._check), _lib.ptr(self.state), eng.stream)
        return self.state[12]

    def hook(self, dt: float):
        """The per-step callable for BaseModel.run(pre_step=...): launch(dt),
        marked so that the model can fuse it with a barostat's scaling and
        the first half-step (launch_after)."""
        h = self._hooks.get(float(dt))
        if h is None:
            h = self._hooks[float(dt)] = _LoaderHook(self, float(dt))
        return h

    def maintain(self) -> bool:
        """Regrid when the device asked for it (synchronises); True if it did.
        The device asks once the cells come within regrid_margin of the list
        cutoff; the new cells are at least regrid_headroom wider than it, so
        a box that keeps shrinking regrids about once per
        regrid_headroom - regrid_margin of strain rather than at every cell
        it loses (a regrid reloads the engine and recaptures its graphs)."""
        if float(self.state[17].item()) == 0.0:
            return False
        eng = self.molecular.engine
        eng.regrid(margin=self.regrid_headroom)
        self.regrids += 1
        self.state[17] = 0.0
        self._reset_list_box(eng.box_matrix())
        return True

    def step(self, dt: float) -> float:
        self.launch(dt)
        self.maintain()
        mol = self.molecular
        if hasattr(mol, "box"):
            mol.box.H = torch.as_tensor(mol.engine.box_matrix())
        self.total_engineering_strain = float(self.state[12].item())
        return self.total_engineering_strain

    def run(self, model, n_steps: int, dt: float, graph_steps: int = 20) -> torch.Tensor:
        """n_steps of (loader step, MD step) captured together in CUDA graphs of
        graph_steps steps, regridding between graphs when asked; returns the
        engineering strain as a device scalar."""
        hook = self.hook(dt)
        done = 0
        while done < int(n_steps):
            k = min(int(graph_steps), int(n_steps) - done)
            model.run(k, graph_steps=graph_steps, pre_step=hook)
            self.maintain()
            done += k
        return self.state[12]

    @property
    def forced_rebuilds(self) -> int:
        return int(self.state[16].item())

    def current_lengths(self) -> torch.Tensor:
        return torch.tensor(np.linalg.norm(self.molecular.engine.box_matrix(), axis=1), dtype=torch.float64)


class _LoaderHook:
    """UniaxialTensileLoader.launch(dt) as a BaseModel.run pre-step."""

    def __init__(self, loader, dt: float):
        self.loader, self.dt = loader, float(dt)

    def __call__(self):
        return self.loader.launch(self.dt)


class SphericalIndenterForce(BackboneInterface):
    """Repulsive sphere (indenter.py:7-68): for atoms with d = |x - c| < R,
    U = K/3 (R - d)^3 and F = K (R - d)^2 (x - c)/d.  On the device: added to
    the engine's forces, energy and virial after the force field's pass (as a
    further backbone of SumBackboneInterface), with its own energy, force on
    the indenter and contact count in ``out``.  The centre is device memory,
    so ``set_center`` between CUDA-graph replays takes effect.  Positions are
    the unwrapped ones, without periodic images (as the reference).  The
    engine's virial tensor is symmetric: the indenter's F (x) x enters it with
    its upper triangle."""

    # its force depends on the atom's own position only, so an EAM force pass
    # can add it in its per-atom epilogue (sim_eam_force_integrate_indenter)
    fusable_into_force_pass = True

    def __init__(self, molecular, radius: float, stiffness: float, center):
        super().__init__()
        self.molecular = molecular
        self.device = molecular.device
        self.radius = float(radius)
        self.stiffness = float(stiffness)
        c = torch.as_tensor(center, dtype=torch.float64).reshape(-1)
        if c.numel() != 3:
            raise ValueError("center must have three components")
        self._center = c.to(self.device).clone()
        self.out = torch.zeros(11, dtype=torch.float64, device=self.device)
        self._st = _lib.SimIndenter()
        self._st.center, self._st.out = _lib.ptr(self._center), _lib.ptr(self.out)
        self._st.radius, self._st.stiffness = self.radius, self.stiffness
        self._ref = ctypes.byref(self._st)
        self.force_precision = 0

    @property
    def center(self) -> torch.Tensor:
        return self._center

    def set_center(self, center) -> None:
        self._center.copy_(torch.as_tensor(center, dtype=torch.float64).reshape(3))

    @property
    def force_on_indenter(self) -> torch.Tensor:
        return self.out[1:4]

    @property
    def last_energy(self) -> torch.Tensor:
        return self.out[0]

    @property
    def contact_atoms(self) -> int:
        return int(self.out[4].item())

    def add_to_engine(self, force_precision: int = 0):
        eng = self.molecular.engine
        _lib.call("sim_indenter_add", eng.st_ref, self._ref, int(force_precision), eng.stream)

    def compute(self):
        """Alone (the only backbone): the engine's forces and sums are zeroed first."""
        eng = self.molecular.engine
        eng.f32.zero_()
        if eng.f64 is not None:
            eng.f64.zero_()
        eng.red_out.zero_()
        self.add_to_engine(self.force_precision)
        eng.forces_valid = True

    def forward(self):
        self.compute()
        return _force_outputs(self.molecular)
