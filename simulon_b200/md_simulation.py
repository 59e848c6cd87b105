"""Run loop with the interface of core/md_simulation.py (MDSimulator).

``run`` advances the model in graph-captured chunks between print intervals
(no per-step host synchronisation) and reports the same profile and the
same Matom-step/s figure as the reference (md_simulation.py:252-293:
steps * atoms / loop_time / 1e6).  Per-step energies come from the device
log.  When ``store_outputs`` is on (the reference does this whenever
num_steps <= 2000, md_simulation.py:57-68,190-194) forces, energies and
coordinates of every step are kept on the device in float16, which forces a
per-step path.
"""
from __future__ import annotations

import time

import torch


class MDSimulator:
    def __init__(self, model, num_steps: int, print_interval: int = 10, store_outputs: bool | None = None,
                 graph_steps: int = 20, verbose: bool = True, **unused):
        self.model = model
        self.num_steps = int(num_steps)
        self.print_interval = int(print_interval)
        self.device = model.engine.device
        self.graph_steps = int(graph_steps)
        self.verbose = verbose
        self._max_store_steps = 2000
        self.store_outputs = (num_steps <= self._max_store_steps) if store_outputs is None else bool(store_outputs)
        n = model.molecular.atom_count
        if self.store_outputs:
            k = min(self.num_steps, self._max_store_steps)
            self.gpu_trajectory = torch.empty((k, n, 3), device=self.device, dtype=torch.float16)
            self.gpu_forces = torch.empty((k, n, 3), device=self.device, dtype=torch.float16)
            self.gpu_energies = torch.empty(k, device=self.device, dtype=torch.float16)
        self.sim_profile = {"output_time": 0.0}
        self.energy_log = []

    def run(self, enable_minimize_energy: bool = False):
        if enable_minimize_energy:
            raise NotImplementedError("energy minimisation is not part of this package; "
                                      "call run(enable_minimize_energy=False)")
        model = self.model
        mol = model.molecular
        if self.verbose:
            print(f"Simulation will run on GPU: {torch.cuda.get_device_name(self.device)}")
        torch.cuda.synchronize(self.device)
        t0 = time.perf_counter()
        step = 0
        first_log = model.steps_done
        while step < self.num_steps:
            chunk = min(self.print_interval - (step % self.print_interval), self.num_steps - step)
            if self.store_outputs:
                for _ in range(chunk):
                    out = model()
                    k = step % self._max_store_steps
                    self.gpu_forces[k] = out["forces"].to(torch.float16)
                    self.gpu_energies[k] = out["energy"].to(torch.float16)
                    self.gpu_trajectory[k] = out["updated_coordinates"].to(torch.float16)
                    step += 1
            else:
                model.run(chunk, graph_steps=self.graph_steps)
                step += chunk
            if step % self.print_interval == 0 or step == self.num_steps:
                t_out = time.perf_counter()
                row = model.step_log(model.steps_done - 1, 1)[0].cpu()
                pot = float(row[0] + row[1])
                kin = float(row[9])
                temp = (2.0 / 3.0) * kin / (mol.atom_count * model.Integrator.BOLTZMAN)
                status = int(row[-1])
                if status:
                    raise RuntimeError(f"device status {status:#x} at step {step} (overflow/non-finite)")
                self.energy_log.append((step, pot, kin, pot + kin, temp))
                if self.verbose:
                    print(f"Step {step}/{self.num_steps}:Tot_E={pot + kin:.4f} ev, Pot_E = {pot:.4f} ev, "
                          f"Kin_E = {kin:.4f} ev, T = {temp:.4f} K")
                self.sim_profile["output_time"] += time.perf_counter() - t_out
        torch.cuda.synchronize(self.device)
        self.sim_profile["loop_time"] = time.perf_counter() - t0
        self.first_step_logged = first_log
        return {"energies": self.energy_log}

    def summarize_profile(self):
        mol = self.model.molecular
        loop = self.sim_profile.get("loop_time", 0.0)
        steps, atoms = self.num_steps, mol.atom_count
        dt_ps = getattr(self.model.Integrator, "dt", 0.0)
        sim_ns = steps * dt_ps / 1000.0
        out = dict(loop_time=loop, steps_per_s=steps / loop if loop > 0 else 0.0,
                   matom_steps_per_s=steps * atoms / loop / 1e6 if loop > 0 else 0.0,
                   ns_per_day=sim_ns / (loop / 86400.0) if loop > 0 else 0.0,
                   output_time=self.sim_profile["output_time"])
        if self.verbose:
            print(f"Performance: {out['ns_per_day']:.3f} ns/day, {out['steps_per_s']:.3f} steps/s, "
                  f"{out['matom_steps_per_s']:.3f} Matom-step/s")
        return out


__all__ = ["MDSimulator"]
