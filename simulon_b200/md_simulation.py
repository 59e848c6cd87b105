"""Run loop with the interface of core/md_simulation.py (MDSimulator).

``run`` advances the model in graph-captured chunks between print intervals
(no per-step host synchronisation) and reports the same profile and the
same Matom-step/s figure as the reference (md_simulation.py:252-293:
steps * atoms / loop_time / 1e6).  Per-step energies come from the device
log.  When ``store_outputs`` is on (the reference does this whenever
num_steps <= 2000, md_simulation.py:57-68,190-194) forces, energies and
coordinates of every step are kept on the device in float16, which forces a
per-step path.

Output files as the reference's (md_simulation.py:30-100,125-168):
``output_dir`` with ``traj.xyz`` every ``traj_interval`` steps ("n", "Step s,
Energy = E", "type x y z"), ``energies.csv`` (step, potential, kinetic, total,
temperature; every step or every ``energies_interval``) and
``forces/forces_<step>.pt``.  The run stays in CUDA graphs up to each
output step; positions, forces and the step log rows go to pinned host
buffers by asynchronous copies, and a background thread writes the files
(trajectory rows formatted by the library, sim_format_xyz_rows) while the
device runs on (no synchronisation per output step).
"""
from __future__ import annotations

import ctypes
import os
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np
import torch

from . import _lib


XYZ_THREADS = min(8, os.cpu_count() or 1)   # threads formatting one trajectory frame


class MDSimulator:
    def __init__(self, model, num_steps: int, print_interval: int = 10, store_outputs: bool | None = None,
                 graph_steps: int = 20, verbose: bool = True, output_dir: str | None = None, dump_interval: int = 0,
                 dump_format: str = "xyz", write_forces: bool = False, write_energies: bool = False,
                 traj_interval: int | None = None, forces_interval: int | None = None,
                 energies_interval: int | None = None, **unused):
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
        # files (md_simulation.py:30-100)
        self.output_dir = Path(output_dir) if output_dir else None
        self.dump_format = (dump_format or "xyz").lower()
        self.write_forces = bool(write_forces)
        self.write_energies = bool(write_energies)
        self.dump_interval = int(dump_interval or 0)
        self.traj_interval = int(traj_interval) if traj_interval is not None else self.dump_interval
        self.forces_interval = int(forces_interval) if forces_interval is not None else self.dump_interval
        self.energies_interval = int(energies_interval) if energies_interval is not None else None
        any_traj = self.traj_interval > 0 and self.dump_format == "xyz"
        any_forces = self.write_forces and self.forces_interval > 0
        self.output_enabled = bool(self.output_dir and (any_traj or any_forces or self.write_energies))
        self._paths = {}
        self._pending = []
        self._writer = None      # one background thread writes the files in step order
        self._formatters = None  # threads formatting the blocks of one trajectory frame
        self._jobs = []
        self._profile_lock = threading.Lock()   # output_time is added to from both threads
        if self.output_enabled:
            self.output_dir.mkdir(parents=True, exist_ok=True)
            if any_traj:
                self._paths["traj"] = str(self.output_dir / "traj.xyz")
                open(self._paths["traj"], "w", encoding="utf-8").close()
            if self.write_energies:
                self._paths["energies"] = str(self.output_dir / "energies.csv")
                with open(self._paths["energies"], "w", encoding="utf-8") as f:
                    f.write("step,potential,kinetic,total,temperature\n")
            if any_forces:
                (self.output_dir / "forces").mkdir(parents=True, exist_ok=True)
                self._paths["forces_dir"] = str(self.output_dir / "forces")

    # ---- outputs: device -> pinned host by async copies, written later ------
    def _output_due(self, step_i: int) -> bool:
        return bool(("traj" in self._paths and step_i % self.traj_interval == 0) or
                    ("forces_dir" in self._paths and step_i % self.forces_interval == 0))

    def _next_stop(self, step: int) -> int:
        """Steps from `step` to the next print or output step."""
        k = self.print_interval - (step % self.print_interval)
        for iv, key in ((self.traj_interval, "traj"), (self.forces_interval, "forces_dir")):
            if key in self._paths and iv > 0:
                k = min(k, iv - (step % iv))
        return min(k, self.num_steps - step)

    def _stage(self, step_i: int, log_from: int, log_count: int):
        """Queue the copies for outputs of step_i and the log rows since the last stage."""
        model = self.model
        eng = model.engine
        item = {"step": step_i}
        stream = torch.cuda.current_stream(self.device)
        if "traj" in self._paths and step_i % self.traj_interval == 0:
            x = eng.gather("x")
            item["x"] = torch.empty(x.shape, dtype=x.dtype, pin_memory=True)
            item["x"].copy_(x, non_blocking=True)
        if "forces_dir" in self._paths and step_i % self.forces_interval == 0:
            f = eng.gather("f").to(model.molecular.dtype)
            item["f"] = torch.empty(f.shape, dtype=f.dtype, pin_memory=True)
            item["f"].copy_(f, non_blocking=True)
        if "energies" in self._paths or "traj" in self._paths:
            rows = model.step_log(log_from, log_count)
            item["log_first"] = log_from
            item["log"] = torch.empty(rows.shape, dtype=rows.dtype, pin_memory=True)
            item["log"].copy_(rows, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(stream)
        item["event"] = ev
        self._pending.append(item)

    def _xyz_table(self):
        """Per-atom type indices and the symbol table for sim_format_xyz_rows."""
        if not hasattr(self, "_xyz_types"):
            mol = self.model.molecular
            names = getattr(mol, "atom_types", None)
            names = list(names) if names is not None and len(names) == mol.atom_count else ["X"] * mol.atom_count
            symbols = sorted(set(names))
            index = {sym: k for k, sym in enumerate(symbols)}
            self._xyz_types = np.array([index[sym] for sym in names], dtype=np.int32)
            self._xyz_symbols = (ctypes.c_char_p * len(symbols))(*[sym.encode() for sym in symbols])
            self._xyz_width = max(len(sym) for sym in symbols) + 196
        return self._xyz_types, self._xyz_symbols, self._xyz_width

    def _write_item(self, item, n, kB):
        """Append one staged output step to the files (runs on the writer thread;
        the library's row formatter releases the GIL while it works)."""
        t0 = time.perf_counter()
        step_i = item["step"]
        log = item.get("log")
        if log is not None and "energies" in self._paths:
            with open(self._paths["energies"], "a", encoding="utf-8") as f:
                for r, row in enumerate(log.tolist()):
                    s = item["log_first"] - self._first_log + r + 1
                    if self.energies_interval is not None and (self.energies_interval <= 0 or
                                                               s % self.energies_interval):
                        continue
                    pot, kin = row[0] + row[1], row[9]
                    temp = (2.0 / 3.0) * kin / (n * kB)
                    f.write(f"{s},{pot:.8f},{kin:.8f},{pot + kin:.8f},{temp:.6f}\n")
        if "x" in item:
            pot = log[-1, 0].item() + log[-1, 1].item()
            types, symbols, width = self._xyz_table()
            xyz = item["x"].numpy()
            lib = _lib.load()
            # row blocks formatted on parallel threads (the call releases the GIL)
            bounds = np.linspace(0, n, min(XYZ_THREADS, max(1, n // 4096)) + 1).astype(np.int64)

            def block(k):
                a, b = int(bounds[k]), int(bounds[k + 1])
                buf = np.empty(max(1, (b - a) * width), dtype=np.uint8)
                nb = lib.sim_format_xyz_rows(xyz[a:].ctypes.data, types[a:].ctypes.data, b - a, symbols,
                                             len(symbols), buf.ctypes.data, buf.size)
                if nb < 0:
                    raise RuntimeError("sim_format_xyz_rows: bad arguments or buffer")
                return memoryview(buf)[:nb]
            if self._formatters is None:
                self._formatters = ThreadPoolExecutor(max_workers=XYZ_THREADS)
            parts = list(self._formatters.map(block, range(len(bounds) - 1)))
            with open(self._paths["traj"], "ab") as f:
                f.write(f"{n}\nStep {step_i}, Energy = {pot:.6f}\n".encode())
                for part in parts:
                    f.write(part)
        if "f" in item:
            torch.save(item["f"].clone(), os.path.join(self._paths["forces_dir"], f"forces_{step_i:06d}.pt"))
        with self._profile_lock:
            self.sim_profile["output_time"] += time.perf_counter() - t0

    def _write_ready(self, wait: bool = False):
        """Hand every staged output whose copies have landed to the writer
        thread; with wait, also the rest, and wait until all files are written."""
        mol = self.model.molecular
        kB = self.model.Integrator.BOLTZMAN
        n = mol.atom_count
        if self._writer is None:
            self._writer = ThreadPoolExecutor(max_workers=1)
        while self._pending and (wait or self._pending[0]["event"].query()):
            item = self._pending.pop(0)
            item["event"].synchronize()
            self._jobs.append(self._writer.submit(self._write_item, item, n, kB))
        if wait:
            jobs, self._jobs = self._jobs, []
            for job in jobs:
                job.result()            # re-raises a failed write here
            self._writer.shutdown()
            self._writer = None
            if self._formatters is not None:
                self._formatters.shutdown()
                self._formatters = None
        else:
            self._jobs = [j for j in self._jobs if not j.done() or j.exception() is not None]

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
        self._first_log = first_log
        staged_upto = first_log
        while step < self.num_steps:
            chunk = self._next_stop(step) if self.output_enabled else \
                min(self.print_interval - (step % self.print_interval), self.num_steps - step)
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
            if self.output_enabled and (self._output_due(step) or step % self.print_interval == 0 or
                                        step == self.num_steps):
                self._stage(step, staged_upto, model.steps_done - staged_upto)
                staged_upto = model.steps_done
                self._write_ready()
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
                with self._profile_lock:
                    self.sim_profile["output_time"] += time.perf_counter() - t_out
        if self.output_enabled:
            self._write_ready(wait=True)
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
