"""Step model with the interface of core/md_model.py (SumBackboneInterface, BaseModel).

``BaseModel.forward`` keeps the reference's order (md_model.py:88-166):
first call computes forces; then first_half (with the skin/2 trigger and a
conditional list rebuild) -> forces -> second_half -> optional Berendsen.
Unlike the reference it makes no host synchronisation: every quantity stays
on the device and the returned mapping materialises values when read.

``BaseModel.run(n)`` executes n such steps through captured CUDA graphs
(``graph_steps`` steps per graph), logging energy, kinetic energy, virial,
pressure and the status word of every step into a device ring buffer.
"""
from __future__ import annotations

import torch
import torch.nn as nn

from . import _lib
from .forces import BackboneInterface, LazyOutputs
from .integrator import IntegratorInterface

__all__ = ["BackboneInterface", "IntegratorInterface", "SumBackboneInterface", "BaseModel"]


class SumBackboneInterface(nn.Module):
    """Sum of force-field backbones (md_model.py:19-52).  The first backbone
    is the device force field (it writes the engine's forces, energy and
    virial); each further one must add its terms on the device
    (``add_to_engine``: ``LennardJonesForce`` with FP32 pairs,
    ``SphericalIndenterForce``).  The outputs are the engine's sums, as the
    reference's summed buffers: the scalar virials are added as each force
    field defines its own (EAM sum s r, LJ sum F r), as the reference adds
    them."""

    def __init__(self, backbones, molecular):
        super().__init__()
        self.backbones = nn.ModuleList(backbones)
        self.molecular = molecular
        self.device = molecular.device
        self.atom_num = molecular.atom_count
        if len(self.backbones) < 1:
            raise ValueError("at least one force field is needed")
        for b in list(self.backbones)[1:]:
            if not hasattr(b, "add_to_engine"):
                raise NotImplementedError(f"{type(b).__name__} cannot be summed on the device (needs add_to_engine)")
        self.force_precision = getattr(self.backbones[0], "force_precision", 0)

    @property
    def single(self) -> bool:
        return len(self.backbones) == 1

    def compute(self):
        self.backbones[0].compute()
        for b in list(self.backbones)[1:]:
            b.add_to_engine(self.force_precision)

    def forward(self):
        if self.single:
            return self.backbones[0]()
        self.compute()
        from .forces import _force_outputs
        return _force_outputs(self.molecular)


class BaseModel(nn.Module):
    def __init__(self, sum_bone, integrator, molecular, barostat=None):
        super().__init__()
        self.sum_bone = sum_bone
        self.Integrator = integrator
        self.molecular = molecular
        self.barostat = barostat
        self.engine = molecular.engine
        integrator.force_precision = sum_bone.force_precision
        self._first_call = True
        self.steps_done = 0
        self.profile = {"pair_time": 0.0, "integrate_time": 0.0, "pair_calls": 0, "integrate_calls": 0}
        self._graphs = {}

    # one step, launches only (no host sync)
    def _indenter_fused(self):
        """(EAM backbone, indenter) when the pair can run as one force pass with
        the integrator fused (one element type, FP32 pairs, no barostat)."""
        bb = self.sum_bone.backbones
        if (self.barostat is not None or len(bb) != 2 or not hasattr(bb[0], "compute_finish_with_indenter")
                or not getattr(bb[1], "fusable_into_force_pass", False) or not hasattr(self.Integrator, "params")
                or self.engine.use_tiles or getattr(bb[0], "E", 0) != 1 or bb[0].force_precision != 0):
            return None
        return bb[0], bb[1]

    def _forces_and_second_half(self):
        pair = self._indenter_fused()
        if pair is not None:
            pair[0].compute_finish_with_indenter(self.Integrator, pair[1], 1)
            return
        fused = getattr(self.sum_bone.backbones[0], "compute_and_finish", None) if self.sum_bone.single else None
        if fused is not None and hasattr(self.Integrator, "params"):
            fused(self.Integrator)        # EAM: second half fused into pass 2
        else:
            self.sum_bone.compute()
            self.Integrator.second_half()

    def _step_launches(self):
        self.Integrator.first_half()
        self._forces_and_second_half()
        if self.barostat is not None:
            self.barostat.step(self.Integrator.dt)
        self.engine.log_step()

    def _drift_fusable(self) -> bool:
        bone = self.sum_bone.backbones[0]
        return (self.barostat is None and self.sum_bone.single and hasattr(bone, "compute_finish_and_drift")
                and hasattr(self.Integrator, "params") and not self.engine.use_tiles)

    def _launch_steps(self, k: int, pre_step=None):
        """k steps, launches only.  ``pre_step`` (launches only, e.g.
        UniaxialTensileLoader.launch) runs before each step; the steps then
        run unfused.  For EAM without a barostat the first half of
        step s+1 runs inside step s's force pass (same arithmetic, one pass over
        the atoms fewer per step); the last step ends with full-step velocities.
        With a spherical indenter as EAM's second backbone, the indenter's force
        is added inside that pass.  With a Berendsen barostat the atoms'
        scaling of step s runs inside step s+1's first half; the last step
        scales them itself."""
        if pre_step is not None:
            loader = getattr(pre_step, "loader", None)
            baro = self.barostat
            if (k > 1 and loader is not None and callable(getattr(loader, "link", None))
                    and callable(getattr(baro, "controller", None)) and hasattr(baro, "work")
                    and hasattr(self.Integrator, "params")):
                # tensile loop: the barostat's atom scaling of step s, the
                # loader's update and the first half of step s+1 in one pass
                pre_step()
                self.Integrator.first_half()
                for s in range(k):
                    self._forces_and_second_half()
                    if s < k - 1:
                        loader.link(baro, self.Integrator, pre_step.dt)
                    else:
                        baro.step(self.Integrator.dt)
                        self.engine.log_step()
                return
            for _ in range(k):
                pre_step()
                self._step_launches()
            return
        if k > 1 and not self._drift_fusable() and callable(getattr(self.barostat, "deferred_first_half", None)) \
                and hasattr(self.Integrator, "params"):
            for s in range(k):
                if s == 0:
                    self.Integrator.first_half()
                else:
                    self.barostat.deferred_first_half(self.Integrator)
                self._forces_and_second_half()
                if s < k - 1:
                    self.barostat.controller(self.Integrator.dt)
                else:
                    self.barostat.step(self.Integrator.dt)
                self.engine.log_step()
            return
        pair = self._indenter_fused() if k > 1 else None
        if pair is not None:     # EAM + indenter: the indenter inside the drift-fused force pass
            eam, ind = pair
            self.Integrator.first_half()
            for s in range(k):
                if s < k - 1:
                    eam.step_drift_with_indenter(self.Integrator, ind)
                else:
                    eam.compute_finish_with_indenter(self.Integrator, ind, 1)
                    self.engine.log_step()
            return
        if k <= 1 or not self._drift_fusable():
            for _ in range(k):
                self._step_launches()
            return
        bone = self.sum_bone.backbones[0]
        self.Integrator.first_half()
        for s in range(k):
            if s < k - 1:
                if hasattr(bone, "step_and_drift"):
                    bone.step_and_drift(self.Integrator)   # log row and rebuild decision inside pass 2
                else:
                    bone.compute_finish_and_drift(self.Integrator)
                    self.engine.log_step(after_drift=True)
                    self.engine.rebuild_if_needed()
            else:
                bone.compute_and_finish(self.Integrator)
                self.engine.log_step()

    def _outputs(self):
        eng, mol = self.engine, self.molecular
        dt = mol.dtype
        red = eng.red_out
        n = mol.atom_count
        kB = self.Integrator.BOLTZMAN
        ke = lambda: red[_lib.RED_KE].to(dt)
        prod = dict(forces=lambda: eng.gather("f").to(dt),
                    energy=lambda: eng.potential_energy().to(dt),
                    virial=lambda: red[_lib.RED_VIRIAL].to(dt),
                    virial_tensor=lambda: eng.virial_tensor().to(dt),
                    updated_coordinates=lambda: mol.coordinates,
                    kinetic_energy=ke,
                    temperature=lambda: (2.0 / 3.0) * ke() / (n * kB))
        if self.barostat is not None:
            prod["pressure"] = self.barostat.pressure
        return LazyOutputs(**prod)

    def _prime(self):
        # forces of the current positions are needed by the first half step:
        # on the first call (md_model.py:91-102) and after coordinates were replaced
        if self._first_call or not self.engine.forces_valid:
            self.sum_bone.compute()
            self._first_call = False

    def forward(self):
        self._prime()
        self._step_launches()
        self.steps_done += 1
        self.profile["pair_calls"] += 1
        self.profile["integrate_calls"] += 1
        return self._outputs()

    # ---- graph-captured multi-step execution ------------------------------
    def _graph(self, k: int, pre_step=None):
        if getattr(self, "_graph_generation", None) != self.engine.generation:
            self._graphs = {}   # the engine's buffers were reallocated (MDEngine.regrid)
            self._graph_generation = self.engine.generation
        key = (k, pre_step)
        if key not in self._graphs:
            if len(self._graphs) >= 8:                     # keep the cache bounded
                self._graphs.pop(next(iter(self._graphs)))
            s = torch.cuda.Stream(self.engine.device)
            s.wait_stream(torch.cuda.current_stream(self.engine.device))
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=s):
                self._launch_steps(k, pre_step)
            torch.cuda.current_stream(self.engine.device).wait_stream(s)
            self._graphs[key] = g
        return self._graphs[key]

    def run(self, n_steps: int, graph_steps: int = 20, pre_step=None):
        """Advance n_steps with CUDA graphs (no host sync); returns the last outputs.

        ``pre_step``: a callable that only launches device work (for example
        UniaxialTensileLoader.launch with its dt bound), run before every step
        and captured with it.  Capturing records launches without executing
        them, so the device state is unchanged by the capture itself.
        """
        n_steps = int(n_steps)
        if pre_step is not None and n_steps > 0 and (self._first_call or not self.engine.forces_valid):
            # as the reference's loop (loader.step(); model()): the first call's
            # forces are those of the positions after the first pre-step
            pre_step()
            self._prime()
            self._step_launches()
            self.steps_done += 1
            self.profile["pair_calls"] += 1
            self.profile["integrate_calls"] += 1
            n_steps -= 1
        self._prime()
        full, rest = divmod(n_steps, int(graph_steps))
        if full:
            g = self._graph(int(graph_steps), pre_step)
            for _ in range(full):
                g.replay()
        self._launch_steps(rest, pre_step)
        self.steps_done += n_steps
        self.profile["pair_calls"] += n_steps
        self.profile["integrate_calls"] += n_steps
        return self._outputs()

    def step_log(self, first_step: int, count: int) -> torch.Tensor:
        """Rows of the per-step device log for steps [first_step, first_step+count)
        (columns: reduction slots, pressure, mu, status)."""
        cap = self.engine.log_capacity
        if count > cap:
            raise ValueError("log window exceeds the ring buffer")
        idx = torch.arange(first_step, first_step + count, device=self.engine.device) % cap
        return self.engine.log[idx]
