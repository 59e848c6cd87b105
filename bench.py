#!/usr/bin/env python
"""Throughput of the EAM-W per-step force path on B200 (atom-steps/s).

Workload (one step = one MD step through BaseModel: first half-kick + drift
with the skin/2 trigger, conditional Verlet-list rebuild, two-pass EAM,
second half-kick): BCC tungsten 2 n^3 atoms (n = 80 -> 1,024,000), a = 3.165 A,
synthetic Finnis-Sinclair potential tabulated in eam/fs layout, skin 0.5 A,
NVE from Maxwell-Boltzmann velocities at 300 K, dt = 2 fs; FP32 pair/EAM
arithmetic, FP64 integration and reductions.  Inputs are seeded synthetic
data.  The device state (~0.4 GB) exceeds the 126 MB L2, so no L2 flush is
needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

With N > 1 (launched by torchrun) every rank runs an independent replica
(weak scaling, no collective on the data path); the time is the max over
ranks and the value is the total atom-steps of all ranks per second.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "atom-steps/s (EAM-W, 1 B200): plain vs batched vs MLP at stated force RMSE"
UNIT = "atom-steps/s"
PASS2_DRAM_BYTES_PER_ATOM = (67890176 + 1833216) / 524288   # k_eam_force<1,1,1>, ncu --set full
A_W, M_W = 3.165, 183.84


def warm_steps(args, graph_steps):
    """Untimed warm-up steps: at least W, and at least three replays of a graph of
    graph_steps steps. The first replays of a freshly instantiated graph run about 4%
    slower than later ones (0.203 against 0.194 ms per step on the 1,024,000-atom EAM
    step, measured on B200), so a region timed after a single replay reads low."""
    return max(args.warmup, 3 * graph_steps)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=2000)
    p.add_argument("--warmup", type=int, default=40)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--n", type=int, default=80, help="BCC cells per side (atoms = 2 n^3)")
    p.add_argument("--graph-steps", type=int, default=20)
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--no-extras", action="store_true", help="skip e2e / cpu baseline (profiling runs)")
    p.add_argument("--no-batched", action="store_true", help="skip the batched-replica form")
    p.add_argument("--no-lj", action="store_true", help="skip the LJ argon form")
    p.add_argument("--no-mlp", action="store_true", help="skip the MLP-surrogate form")
    p.add_argument("--no-autotune", action="store_true",
                   help="keep the built-in launch shapes (profiling runs: fewer launches before the timed ones)")
    p.add_argument("--forms", default="plain,lj,mlp,batched,variants,mechanics",
                   help="forms to run (profiling runs: e.g. --forms mlp prints only the mlp object)")
    p.add_argument("--lj-n", type=int, default=63, help="FCC cells per side of the LJ form (atoms = 4 n^3)")
    p.add_argument("--batch-replicas", type=int, default=48)
    p.add_argument("--batch-skin", type=float, default=0.75)
    return p.parse_args()


def bcc(n):
    g = np.arange(n)
    cells = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0.5]])
    return ((cells[:, None, :] + basis[None]).reshape(-1, 3) * A_W).astype(np.float64), n * A_W


def write_potential(path, n=5000, d_rho=0.012, cutoff=4.4):
    """Synthetic Finnis-Sinclair W in eam/fs layout: phi = (r-c)^2 (c0 + c1 r + c2 r^2),
    rho = (r-d)^2, F = -A sqrt(rho); 5000-point r and rho grids; pair block holds r*phi."""
    c, d, A, c0, c1, c2 = 3.25, 4.400224, 1.896373, 47.1346499, -33.7665655, 6.2541999
    dr = cutoff / n
    r = np.arange(n) * dr
    rho = np.arange(n) * d_rho
    F = -A * np.sqrt(rho)
    f = np.where(r < d, (r - d) ** 2, 0.0)
    phi = np.where(r < c, (r - c) ** 2 * (c0 + c1 * r + c2 * r * r), 0.0)
    out = ["synthetic Finnis-Sinclair W", "eam/fs layout", "", "1 W", f"{n} {d_rho!r} {n} {dr!r} {cutoff!r}",
           f"74 {M_W} {A_W} bcc"]
    for blk in (F, f, r * phi):
        out += [" ".join(f"{v:.16e}" for v in blk[k:k + 5]) for k in range(0, n, 5)]
    with open(path, "w") as fh:
        fh.write("\n".join(out) + "\n")
    return path


def mb_velocities(n_atoms, T, seed):
    rng = np.random.default_rng(seed)
    m = M_W * 1.036427e-4
    v = rng.standard_normal((n_atoms, 3)) * np.sqrt(8.617333262e-5 * T / m)
    return v - v.mean(0)


class ClockSampler:
    """nvidia-smi samples during the timed region (clocks, power, throttle reasons).

    Entering waits (up to 3 s) for the first sample, so that sampling runs
    before the timed work starts; the summary keeps the samples taken between
    entering and leaving (the nearest later one if the region was shorter
    than the 100 ms sampling interval, reported with "in_region": 0)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", self.gpu_id], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            give_up = time.monotonic() + 3.0
            while not self.lines and self.proc.poll() is None and time.monotonic() < give_up:
                time.sleep(0.005)
        except (OSError, ValueError):
            self.proc = None
        self.t0 = time.monotonic()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def __exit__(self, *exc):
        self.t1 = time.monotonic()
        if self.proc is not None:
            # one more sample when the region was shorter than the interval
            give_up = self.t1 + 0.3
            while not any(t >= self.t1 for t, _ in self.lines) and self.proc.poll() is None \
                    and time.monotonic() < give_up:
                time.sleep(0.005)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        t0, t1 = getattr(self, "t0", 0.0), getattr(self, "t1", float("inf"))
        inside = [line for t, line in self.lines if t0 <= t <= t1]
        later = [line for t, line in self.lines if t > t1][:1]
        for line in inside or later:
            parts = [s.strip() for s in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0, "in_region": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm), "in_region": len(sm) if inside else 0}


def settle():
    """Before a timed region: collect garbage (so that the destruction of an
    earlier form's CUDA graphs and buffers cannot fall inside the region) and
    drain the device."""
    import torch
    gc.collect()
    torch.cuda.synchronize()


def measured_peaks(key: str = "hbm_gbs"):
    """(peak, "measured"|"fallback"): HBM GB/s, or dense BF16 TFLOP/s (burst)."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        if key in d:
            return float(d[key]), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}[key], "fallback"


# ------------------------------------------------------------------ CPU baseline (oracle port)
def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(seconds: float, n_cells: int = 80):
    """The oracle's restatement of the reference CPU path (FP32 EAM, the
    reference EAM path's only precision; torch CPU ops on all host threads)
    on the bench's own workload, BCC W 2 n^3 atoms: force + integrate steps
    timed for about ``seconds`` (at least two), the list built by the
    oracle's cell search (proven pair-set equal to the reference's search);
    the reference's own O(N^2) search is timed on 16,000 atoms by its C
    restatement and extrapolated by N^2, reported separately."""
    import torch
    from oracle import eam as oeam
    from oracle import inputs as oin
    from oracle import neighbor as onb
    from oracle.box import OracleBox
    from oracle.integrator import OracleMD
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    with tempfile.TemporaryDirectory() as tmp:
        pot = oin.write_fs_w_setfl(os.path.join(tmp, "W.eam.fs"))
        tables = oeam.EAMTables(oeam.parse_eam(pot), dtype=torch.float32)
    x, L = bcc(n_cells)
    box = OracleBox(L)
    types = np.zeros(len(x), np.int64)
    t_setup = time.perf_counter()
    md = OracleMD(x.astype(np.float32), mb_velocities(len(x), 300.0, 5).astype(np.float32), np.full(len(x), M_W),
                  box, lambda xx, i, j: oeam.eam_forward(xx, i, j, types, box, tables), cutoff=4.4, skin=0.5,
                  dt=0.002, ensemble="NVE", dtype=torch.float32)
    t_list = time.perf_counter() - t_setup
    md.step()                                   # warm-up (first call: two force evaluations)
    steps, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds or steps < 2:
        md.step()
        steps += 1
    dt = time.perf_counter() - t0
    # the reference's O(N^2) search (gpu_kdtree.py:90-155), its C restatement on 16,000 atoms
    xs, Ls = bcc(20)
    tb = time.perf_counter()
    onb.half_list(xs.astype(np.float32), OracleBox(Ls), onb.rc2_like_reference(4.4, 0.5, np.float32), mode="brute")
    t_brute = time.perf_counter() - tb
    return {"value": len(x) * steps / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "cpu": cpu_model(),
            "sample": f"oracle FP32 restatement of the reference CPU path (torch CPU, {threads} threads), BCC W "
                      f"{len(x):,} atoms (the bench workload), {steps} NVE force + integrate steps in {dt:.1f} s "
                      f"after one warm-up step, list by the oracle's cell search ({t_list:.1f} s incl. setup; "
                      f"{md.rebuilds - 1} rebuilds inside the timed steps)",
            "rebuild_o_n2_extrapolated_s": t_brute * (len(x) / len(xs)) ** 2,
            "rebuild_note": f"the reference's O(N^2) pair search restated in C, {t_brute:.2f} s on {len(xs):,} atoms, "
                            f"scaled by (N/{len(xs):,})^2 (extrapolated, not run)"}


def oracle_force_rmse(x, H, f_gpu, tables64, seed: int, radius: float = 20.0, cutoff: float = 4.4):
    """RMSE of the GPU forces against the FP64 oracle on the atoms within
    ``radius`` of a seeded random point of the box (~2,000 atoms in bulk W):
    the oracle evaluates the atoms within radius + 2 cutoffs of that point, so
    the densities of the sampled atoms' neighbours are complete."""
    import torch
    from oracle import eam as oeam
    from oracle import neighbor as onb
    from oracle.box import OracleBox
    box = OracleBox(H)
    x = np.asarray(x, np.float64)
    rng = np.random.default_rng(seed)
    c = rng.random(3) @ np.asarray(H, np.float64)
    d = np.linalg.norm(box.minimum_image(torch.tensor(x - c)).numpy(), axis=1)
    inner = np.nonzero(d < radius)[0]
    outer = np.nonzero(d < radius + 2.0 * cutoff + 0.1)[0]
    if len(inner) == 0:
        return None, 0
    xs = x[outer]
    hl = onb.half_list(xs, box, (cutoff * (1.0 + 1e-9)) ** 2, mode="brute" if len(xs) < 4096 else "auto")
    o = oeam.eam_forward(torch.tensor(xs), hl["i"], hl["j"], np.zeros(len(xs), np.int64), box, tables64)
    pos_in_outer = np.searchsorted(outer, inner)
    err = np.asarray(f_gpu, np.float64)[inner] - o["forces"].numpy()[pos_in_outer]
    return float(np.sqrt((err ** 2).mean())), int(len(inner))


def oracle_checks(pot, checks):
    """The oracle as the checker of the forms' forces (this CPU leg only):
    force RMSE against the FP64 oracle for each recorded state."""
    import torch
    from oracle import eam as oeam
    t64 = oeam.EAMTables(oeam.parse_eam(pot), dtype=torch.float64)
    out = {}
    for name, c in checks.items():
        if name == "batched":
            per = []
            for k, (x, H, f) in enumerate(c):
                r, n = oracle_force_rmse(x, H, f, t64, seed=100 + k)
                if r is not None:
                    per.append((r, n))
            out[name] = {"max_replica_rmse_ev_per_a": max(r for r, _ in per),
                         "mean_replica_rmse_ev_per_a": float(np.mean([r for r, _ in per])),
                         "replicas_checked": len(per), "atoms_checked": int(sum(n for _, n in per))}
        else:
            x, H, f = c
            r, n = oracle_force_rmse(x, H, f, t64, seed=7)
            out[name] = {"rmse_ev_per_a": r, "atoms_checked": n}
    return out


def config1_cpu():
    """Config 1 on the CPU: LJ argon 108 atoms (FCC 3^3, a 5.26 A, jitter 0.05 A
    seed 0), FP64, Langevin 94.4 K gamma 10/ps, dt 2 fs, 1,000 steps through
    the oracle's restatement of the reference step (torch CPU)."""
    import torch
    from oracle import inputs as oin
    from oracle.box import OracleBox
    from oracle.integrator import OracleMD
    from oracle.lj import lj_forward
    torch.set_num_threads(os.cpu_count() or 1)
    x, L = oin.fcc_lattice(3)
    x = oin.jitter(x, 0.05, 0)
    v = oin.maxwell_boltzmann(np.full(len(x), oin.AR_MASS), 94.4, 1)
    box = OracleBox(L)
    eps = torch.tensor(0.0104, dtype=torch.float32)
    sig = torch.tensor(3.405, dtype=torch.float32)
    md = OracleMD(x, v, np.full(len(x), oin.AR_MASS), box,
                  lambda xx, i, j: lj_forward(xx, i, j, eps.expand(len(i)), sig.expand(len(i)), box, 7.0),
                  cutoff=7.0, skin=0.5, dt=0.002, ensemble="NVT", temperature=94.4, gamma=10.0,
                  dtype=torch.float64, noise_fn=lambda step: torch.randn(len(x), 3, dtype=torch.float64))
    for _ in range(5):
        md.step()
    t0 = time.perf_counter()
    for _ in range(1000):
        md.step()
    dt = time.perf_counter() - t0
    return {"value": len(x) * 1000 / dt, "unit": UNIT, "steps_per_s": 1000 / dt, "ms_per_step": dt,
            "steps": 1000, "atoms": len(x), "kind": "port", "cores": os.cpu_count() or 1,
            "workload": "LJ Ar FCC 3^3 = 108 atoms, FP64, Langevin 94.4 K gamma 10/ps, dt 2 fs, rc 7.0 A, skin 0.5 A"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    # the oracle port on the GPU arm's workload, timed over the timed steps'
    # share of a fixed two-minute budget (at least two MD steps)
    seconds = 90.0 * args.steps / max(1, args.steps + args.warmup)
    base = cpu_baseline(seconds=seconds, n_cells=args.n)
    line = {"metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * 2 * args.n ** 3 / base["value"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"EAM-W bulk BCC 2*{args.n}^3 = {2 * args.n ** 3:,} atoms, synthetic FS potential, "
                                   "NVE from 300 K, dt 2 fs, skin 0.5 A", "atoms": 2 * args.n ** 3},
            "impl": "reference", "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not args.no_extras:
        line["config1"] = config1_cpu()
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ GPU arm
def eng_state_bytes(eng) -> int:
    """Device bytes a step touches: the engine's per-slot arrays and its list."""
    import torch
    return sum(t.numel() * t.element_size() for t in (eng.x, eng.v, eng.posq, eng.posfp, eng.xref, eng.f32, eng.nbr,
                                                       eng.nnbr) if isinstance(t, torch.Tensor))


def energy_drift(model, first: int, k: int, n_atoms: int, dt_ps: float):
    """Least-squares slope of the total energy per atom (eV/atom/ns) over the
    logged steps [first, first + k) (at most the log's capacity)."""
    count, k = int(k), min(int(k), model.engine.log_capacity)
    if k < 2:
        return None
    rows = model.step_log(first + count - k, k).cpu().numpy()
    etot = (rows[:, 0] + rows[:, 1] + rows[:, 9]) / n_atoms
    t_ns = np.arange(k) * dt_ps * 1e-3
    return float(np.polyfit(t_ns, etot, 1)[0])


def clock_window(gpu_id: str, fn, seconds: float = 1.5):
    """Clock samples over repeats of the timed work (fn) for about `seconds`
    right after the timed region, for runs whose timed region is shorter than
    the sampler's 100 ms interval."""
    import torch
    with ClockSampler(gpu_id) as clocks:
        t0 = time.monotonic()
        reps = 0
        while time.monotonic() - t0 < seconds:
            fn()
            torch.cuda.synchronize()
            reps += 1
    out = clocks.summary()
    out["repeats"] = reps
    return out


def config1_gpu(sb, dev, G):
    """Config 1 on the GPU: LJ argon 108 atoms (FCC 3^3, a 5.26 A, jitter 0.05 A
    seed 0), FP64, Langevin 94.4 K gamma 10/ps, dt 2 fs, 1,000 steps through
    BaseModel.run (graphs of G steps), timed with events."""
    import torch
    a = 5.26
    g = np.arange(3)
    cells = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    x = ((cells[:, None, :] + basis[None]).reshape(-1, 3) * a).astype(np.float64)
    x = x + np.random.default_rng(0).normal(0.0, 0.05, size=x.shape)
    L = 3 * a
    m = 39.948 * 1.036427e-4
    rng = np.random.default_rng(1)
    v = rng.standard_normal(x.shape) * np.sqrt(8.617333262e-5 * 94.4 / m)
    v -= v.mean(0)
    old = torch.get_default_dtype()
    torch.set_default_dtype(torch.float64)
    try:
        mol = sb.AtomFileReader.from_arrays(["Ar"] * len(x), x, L, 7.0, device=dev, skin_thickness=0.5,
                                            parameter={"[0 0]": {"epsilon": 0.0104, "sigma": 3.405}})
        integ = sb.VerletIntegrator(mol, dt=0.002, ensemble="NVT", temperature=(94.4, 94.4), gamma=10.0, seed=1)
        mol.atom_velocities = torch.tensor(v, device=dev)
        model = sb.BaseModel(sb.SumBackboneInterface([sb.LennardJonesForce(mol)], mol), integ, mol)
    finally:
        torch.set_default_dtype(old)
    model.run(5 * G, graph_steps=G)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    settle()
    e0.record()
    out = model.run(1000, graph_steps=G)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    return {"value": len(x) * 1000 / (ms / 1e3), "unit": UNIT, "steps_per_s": 1000 / (ms / 1e3),
            "ms_per_step": ms / 1000, "steps": 1000, "atoms": len(x), "temperature_k": float(out["temperature"]),
            "status": mol.engine.status(),
            "workload": "LJ Ar FCC 3^3 = 108 atoms, FP64, Langevin 94.4 K gamma 10/ps, dt 2 fs, rc 7.0 A, skin 0.5 A"}


def launches_for(steps: int, graph_steps: int) -> int:
    """Kernels of ours launched by BaseModel.run(steps): per run of k > 1 steps,
    the first half-step and its IF-node condition, then per step EAM pass 1
    and pass 2 (fused with the second half and the next first half; its last
    block writes the step log row and sets the next IF node's value), the last
    step's pass 2 finishing without the drift and followed by its log kernel
    (2k + 3); a single step is first half, condition, pass 1, pass 2 + second
    half, log (5).  Each triggered rebuild adds the 10 kernels of the IF body."""
    full, rest = divmod(int(steps), int(graph_steps))
    per = lambda k: 0 if k == 0 else (5 if k == 1 else 2 * k + 3)
    return full * per(int(graph_steps)) + per(rest)


def run_b200(args):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    import simulon_b200 as sb
    from simulon_b200 import _lib

    def barrier():
        if world > 1:
            dist.barrier()

    forms = set(f.strip() for f in args.forms.split(",") if f.strip())
    tmp = tempfile.mkdtemp()
    pot = write_potential(os.path.join(tmp, "W_synthetic.eam.fs"))
    if "plain" not in forms:   # profiling runs of single forms
        line = {"metric": METRIC, "unit": UNIT, "n_gpus": world, "forms": sorted(forms)}
        if "lj" in forms and not args.no_lj:
            line["lj"] = lj_form(args, sb, dev, world)
        if "mlp" in forms and not args.no_mlp:
            line["mlp"] = mlp_form(args, sb, pot, dev, world)
        if "batched" in forms and not args.no_batched:
            line["batched"] = batched_form(args, sb, pot, dev, world, rank, barrier)
        if "variants" in forms:
            line["eam_variants"] = eam_variants_form(args, sb, pot, dev, world)
        if "mechanics" in forms and world == 1:
            line["mechanics"] = mechanics_form(args, sb, pot, dev, world)
        if world > 1:
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps(line), flush=True)
        return
    x, L = bcc(args.n)
    N = len(x)
    v = mb_velocities(N, 300.0, 1000 + rank)
    parser = sb.EAMParser(pot)
    mol = sb.AtomFileReader.from_arrays(["W"] * N, x, L, parser.cutoff, device=dev, skin_thickness=0.5, is_fs=True)
    mol.atom_velocities = torch.tensor(v, device=dev)
    ff = sb.EAMForceCUDAExt(parser, mol)
    integ = sb.VerletIntegrator(mol, dt=0.002, ensemble="NVE")
    model = sb.BaseModel(sb.SumBackboneInterface([ff], mol), integ, mol)
    eng = mol.engine
    G = args.graph_steps
    # launch shapes of the two EAM passes, timed on this system (not cached)
    from simulon_b200 import autotune
    shapes = {"density_threads": 0, "force_threads": 0, "ms": {}} if args.no_autotune else \
        autotune.tune_eam(eng, ff.tables, reps=10, use_cache=False)

    # warm-up (captures the graph, runs W steps)
    model.run(warm_steps(args, G), graph_steps=G)
    torch.cuda.synchronize()
    if eng.status():
        raise RuntimeError(f"device status {eng.status():#x} after warm-up")
    rb0 = int(eng.flags[3].item())

    # timed region: K steps, events on the launching stream, barrier + sync both sides
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    uuid = str(torch.cuda.get_device_properties(dev).uuid)
    gpu_id = uuid if uuid.startswith("GPU-") else f"GPU-{uuid}"
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(gpu_id) as clocks:
        settle()
        e0.record(stream)
        model.run(args.steps, graph_steps=G)
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    status = eng.status()
    rebuilds = int(eng.flags[3].item()) - rb0
    value = world * N * args.steps / (ms / 1e3)
    drift = energy_drift(model, model.steps_done - args.steps, args.steps, N, 0.002)
    drift_steps = args.steps
    window = None
    if ms < 300:
        # short timed region: clock samples over repeats of the same steps, and
        # the NVE drift over the longest window the step log holds
        first = model.steps_done
        window = clock_window(gpu_id, lambda: model.run(args.steps, graph_steps=G))
        done = model.steps_done - first
        if done > args.steps:
            drift_steps = min(done, eng.log_capacity)
            drift = energy_drift(model, model.steps_done - drift_steps, drift_steps, N, 0.002)
    # state for the oracle's force check (CPU leg): forces recomputed at the current positions
    eng.eam_forces(ff.tables)
    checks = {"plain": (eng.gather("x").cpu().numpy(), eng.box_matrix(), eng.gather("f").cpu().numpy())}
    nbr = eng.neighbor_stats()
    nbar = nbr["mean"]

    # dominant kernel: EAM pass 2 with the fused second half-step (forces, pair
    # energy, virial, half kick, kinetic tensor), timed alone with events
    R = 50
    ka, kb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    eng.eam_forces(ff.tables)
    torch.cuda.synchronize()
    ka.record(stream)
    for _ in range(R):
        _lib.call("sim_eam_force_integrate", eng.st_ref, ff.tables.ref, integ.params.ref, eng.stream)
    kb.record(stream)
    torch.cuda.synchronize()
    k_ms = ka.elapsed_time(kb) / R
    pa, pb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pa.record(stream)
    for _ in range(R):
        _lib.call("sim_eam_density", eng.st_ref, ff.tables.ref, eng.stream)
    pb.record(stream)
    torch.cuda.synchronize()
    p1_ms = pa.elapsed_time(pb) / R
    peak, peak_kind = measured_peaks()
    bytes_pass2 = N * (16 + 4 * nbar + 4 + 16 + 48)      # posq, list, own F', force out, v read+write
    bytes_pass1 = N * (16 + 4 * nbar + 4)                # posq, list, F' out
    achieved = bytes_pass2 / (k_ms / 1e3) / 1e9
    # measured DRAM bytes per atom of this kernel: dram__bytes_read.sum +
    # dram__bytes_write.sum of one ncu capture on BCC W 2*64^3 = 524,288 atoms,
    # scaled by the atom count (traffic grows with the atoms processed)
    traffic = N * PASS2_DRAM_BYTES_PER_ATOM
    # step-level algorithmic bytes per atom-step (EAM: pass1 + pass2 + integrator 152 + rebuild/K)
    rebuild_bytes = 16 + 88 + 4 * nbar
    K_rb = args.steps / max(rebuilds, 1)
    B_step = (16 + 4 * nbar + 4) + (16 + 4 * nbar + 4 + 16) + 152 + rebuild_bytes / K_rb
    step_achieved = value / world * B_step / 1e9

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic",
            "config": {"workload": f"EAM-W bulk BCC 2*{args.n}^3 = {N:,} atoms per GPU, synthetic FS W (eam/fs "
                                   "tables 5000 pts), NVE from 300 K MB velocities, dt 2 fs, skin 0.5 A",
                       "form": "plain", "atoms_per_gpu": N, "graph_steps": G,
                       "warmup_steps_run": warm_steps(args, G),
                       "l2": (f"state ~{eng_state_bytes(eng) / 1e9:.2f} GB > 126 MB L2 (no flush needed)"
                              if eng_state_bytes(eng) > 126e6 else
                              f"state ~{eng_state_bytes(eng) / 1e6:.0f} MB fits the 126 MB L2 (small case: L2-resident)"),
                       "neighbors_mean": nbar, "neighbor_capacity": nbr["cap"], "rebuilds_in_timed": rebuilds,
                       "launch_shapes": {"density_threads": shapes["density_threads"],
                                         "force_threads": shapes["force_threads"], "autotune_ms": shapes["ms"]},
                       "parallelism": f"replicas x{world}"},
            "status": status,
            "roofline": {"bound": "hbm", "kernel": "k_eam_force<single,integ,ortho> (EAM pass 2 + second half-step)",
                         "achieved": achieved,
                         "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "traffic_source": "ncu capture at 524,288 atoms, scaled per atom",
                         "bytes_per_launch": bytes_pass2, "launch_ms": k_ms,
                         "pass1_ms": p1_ms, "pass1_bytes": bytes_pass1},
            "step_roofline": {"bytes_per_atom_step": B_step, "achieved": step_achieved, "peak": peak,
                              "frac": step_achieved / peak, "unit": "GB/s"},
            "clocks": clocks.summary(),
            "energy_drift_ev_per_atom_per_ns": drift,
            "energy_drift_steps": min(drift_steps, eng.log_capacity),
            "energy_drift_window": "timed steps" if drift_steps == args.steps else
                                   "the NVE steps of the timed region and of the clock window after it",
            "gpu_launches": launches_for(args.steps, G) + 10 * rebuilds}
    if window is not None:
        line["clocks_window"] = dict(window, note="repeats of the timed steps for 1.5 s right after the timed "
                                                 "region (the timed region is shorter than the 100 ms sampling)")

    if not args.no_extras and rank == 0:
        line["e2e"] = e2e(model, mol, x, v, args, dev)
    if not args.no_lj and "lj" in forms:
        line["lj"] = lj_form(args, sb, dev, world)
    if not args.no_mlp and "mlp" in forms:
        line["mlp"] = mlp_form(args, sb, pot, dev, world)
    if not args.no_batched and "batched" in forms:
        line["batched"] = batched_form(args, sb, pot, dev, world, rank, barrier, checks)
    if "variants" in forms:
        line["eam_variants"] = eam_variants_form(args, sb, pot, dev, world, checks)
    if "mechanics" in forms and world == 1:
        line["mechanics"] = mechanics_form(args, sb, pot, dev, world)
    if not args.no_extras and world == 1:
        line["config1"] = config1_gpu(sb, dev, G)
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        if not args.no_extras and world == 1:
            # CPU leg: the timed baseline, then the oracle as the checker of the forces
            line["cpu_baseline"] = cpu_baseline(args.cpu_seconds, n_cells=args.n)
            rm = oracle_checks(pot, checks)
            line["force_rmse_vs_fp64_ev_per_a"] = rm["plain"]["rmse_ev_per_a"]
            line["force_check"] = rm["plain"]
            if "batched" in rm and "batched" in line:
                line["batched"]["force_rmse_vs_fp64"] = rm["batched"]
            if "triclinic_nve" in rm and "eam_variants" in line:
                line["eam_variants"]["triclinic_nve"]["force_rmse_vs_fp64"] = rm["triclinic_nve"]
        print(json.dumps(line), flush=True)


def batched_form(args, sb, pot, dev, world, rank, barrier, checks=None):
    """Batched form: seeded sweep of crack slabs (BCC W, sizes log-uniform in
    [2,000, 250,000], temperatures 50..1200 K, Langevin gamma 10/ps, dt 1 fs,
    grips opening 1e-4 A/step; list skin 0.75 A by default -- a neighbour-list
    parameter that changes no trajectory, chosen between the reference crack
    script's 1.0 A (w_crack.py:325-333) and the bulk 0.5 A as the fastest of
    the three on this workload), all replicas of a rank advanced together.  With N > 1
    the replicas are split over ranks by LPT bin packing (strong scaling, no
    per-step collective); the time is the max over ranks."""
    import torch
    import torch.distributed as dist
    from simulon_b200.batch import BatchedEngine, crack_sweep, gather_replica_table, partition_replicas
    reps = crack_sweep(args.batch_replicas, seed=0, grip_rate=1e-4)
    sizes = [len(r.positions) for r in reps]
    mine = partition_replicas(sizes, world)[rank]
    parser = sb.EAMParser(pot)
    tables = sb.EAMDeviceTables(parser, dev)
    be = BatchedEngine([reps[k] for k in mine], M_W, parser.cutoff, args.batch_skin, device=dev, nbr_cap=64)
    integ = be.integrator(0.001, gamma=10.0, langevin=True, seed=11)
    G = args.graph_steps
    be.run(tables, integ, warm_steps(args, G), graph_steps=G)
    torch.cuda.synchronize()
    rb0 = be.rebuild_counts().copy()
    ev0 = int(be.flags[3].item())
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    settle()
    e0.record(stream)
    be.run(tables, integ, args.steps, graph_steps=G)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    rebuilds = be.rebuild_counts() - rb0
    events = int(be.flags[3].item()) - ev0
    status = be.status()
    if checks is not None:       # per-replica state for the oracle's force check (CPU leg)
        be.eam_forces(tables)
        X, F = be.gather("x").cpu().numpy(), be.gather("f").cpu().numpy()
        checks["batched"] = [(X[be.replica_slice(k)], np.asarray(be.replicas[k].H, np.float64).reshape(3, 3),
                              F[be.replica_slice(k)]) for k in range(be.n_rep)]
    T = be.temperature().cpu()
    table = gather_replica_table(mine, torch.stack([T, torch.tensor(rebuilds, dtype=torch.float64)], 1),
                                 len(reps))
    total = int(sum(sizes))
    # a graph of k steps: first half + counter advance + IF condition, then per
    # step pass 1, pass 2, the two per-replica sum kernels, and (all but the
    # last step) the counter advance and IF condition: 6k + 1; an eager tail of
    # k steps runs the 10 rebuild kernels in place of each condition: 15k + 1.
    # A rebuild event in a graph adds the 10 kernels of the IF body.
    full, rest = divmod(args.steps, G)
    launches = full * (6 * G + 1) + (15 * rest + 1 if rest else 0) + 10 * events
    return {"value": total * args.steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / args.steps,
            "replicas": len(reps), "atoms_total": total, "atoms_min": int(min(sizes)), "atoms_max": int(max(sizes)),
            "scaling": "strong", "status": status, "rebuild_events_in_timed": events,
            "replica_rebuilds_in_timed": int(table[:, 1].sum()),
            "temperature_k_min_max": [float(table[:, 0].min()), float(table[:, 0].max())],
            "gpu_launches": launches,
            "config": {"workload": f"{len(reps)} BCC-W crack slabs, sizes log-uniform 2,000-250,000 (seeded), "
                                   "precrack L_x/4, 3-layer grips opening 1e-4 A/step, T 50-1200 K Langevin "
                                   f"gamma 10/ps, dt 1 fs, skin {args.batch_skin} A",
                       "parallelism": f"LPT over {world} rank(s)", "graph_steps": G,
                       "warmup_steps_run": warm_steps(args, G)}}


def eam_variants_form(args, sb, pot, dev, world, checks=None):
    """The other EAM-W bulk cases of the plain form, 2 n^3 = 1,024,000 atoms:
    NVE in a triclinic box (rows (L,0,0), (0.02 L, L, 0), (0,0,L), the BCC
    sites sheared with it) and Berendsen NPT at P0 = 0 bar with a 300 K
    Langevin thermostat (gamma 10/ps, tau_p 1 ps, orthogonal box); both from
    300 K Maxwell-Boltzmann velocities, dt 2 fs, each timed like the plain
    line (CUDA events around BaseModel.run, graphs of 20 steps)."""
    import torch
    import torch.distributed as dist
    x, L = bcc(args.n)
    N = len(x)
    v = mb_velocities(N, 300.0, 3000 + int(os.environ.get("RANK", "0")))
    parser = sb.EAMParser(pot)
    out = {}
    for name in ("triclinic_nve", "berendsen_npt"):
        if name == "triclinic_nve":
            H = np.array([[L, 0.0, 0.0], [0.02 * L, L, 0.0], [0.0, 0.0, L]])
            xs = (x / L) @ H
            mol = sb.AtomFileReader.from_arrays(["W"] * N, xs, L, parser.cutoff, device=dev, skin_thickness=0.5,
                                                is_fs=True, box_vectors=H)
        else:
            mol = sb.AtomFileReader.from_arrays(["W"] * N, x, L, parser.cutoff, device=dev, skin_thickness=0.5,
                                                is_fs=True)
        ff = sb.EAMForceCUDAExt(parser, mol)
        if name == "triclinic_nve":
            integ = sb.VerletIntegrator(mol, dt=0.002, ensemble="NVE")
            baro = None
        else:
            integ = sb.VerletIntegrator(mol, dt=0.002, ensemble="NPT", temperature=(300.0, 300.0), gamma=10.0, seed=5)
            baro = sb.BerendsenBarostat(mol, 0.0, 1.0)
        mol.atom_velocities = torch.tensor(v, device=dev)   # the seeded draw, after the integrator's own
        model = sb.BaseModel(sb.SumBackboneInterface([ff], mol), integ, mol, barostat=baro)
        eng = mol.engine
        model.run(warm_steps(args, args.graph_steps), graph_steps=args.graph_steps)
        torch.cuda.synchronize()
        rb0 = int(eng.flags[3].item())
        V0 = abs(float(np.linalg.det(eng.box_matrix())))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        settle()
        e0.record()
        outs = model.run(args.steps, graph_steps=args.graph_steps)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        row = {"value": world * N * args.steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / args.steps,
               "status": eng.status(), "rebuilds_in_timed": int(eng.flags[3].item()) - rb0,
               "temperature_k": float(outs["temperature"])}
        if baro is None:
            # short timed regions: continue the same NVE run (untimed) so the
            # drift is fitted over at least 2,000 steps
            extra = max(0, 2000 - args.steps) // args.graph_steps * args.graph_steps
            if extra:
                model.run(extra, graph_steps=args.graph_steps)
            k = min(args.steps + extra, eng.log_capacity)
            row["energy_drift_ev_per_atom_per_ns"] = energy_drift(model, model.steps_done - k, k, N, 0.002)
            row["energy_drift_steps"] = k
            if checks is not None:
                ff.compute()
                checks[name] = (eng.gather("x").cpu().numpy(), eng.box_matrix(), eng.gather("f").cpu().numpy())
        if baro is not None:
            row["pressure_bar"] = float(baro.pressure())
            row["volume_change"] = abs(float(np.linalg.det(eng.box_matrix()))) / V0 - 1.0
        out[name] = row
        del model, ff, integ, mol, eng
        torch.cuda.empty_cache()
    out["config"] = {"workload": f"EAM-W bulk BCC 2*{args.n}^3 = {N:,} atoms per GPU, synthetic FS W, dt 2 fs, "
                                 "skin 0.5 A: triclinic NVE (xy tilt 0.02) and Berendsen NPT (P0 0 bar, tau_p 1 ps, "
                                 "Langevin 300 K)", "scaling": "weak", "parallelism": f"replicas x{world}"}
    return out


def mechanics_form(args, sb, pot, dev, world):
    """The tensile and indentation callers of the EAM-W force path at 2 n^3
    atoms (BCC W, synthetic FS potential, dt 2 fs, 300 K Maxwell-Boltzmann
    velocities): (1) uniaxial tension along x at 0.1 / ps with the anisotropic
    NPT barostat holding y and z at 0 bar (core/mechanics/loading.py:6-81,
    core/barostat.py:78-208), loader step + MD step per step as the
    reference's loop, captured in CUDA graphs (UniaxialTensileLoader.run); (2) a spherical indenter (radius
    20 A, stiffness 0.05 eV/A^3) on the top layer as a second backbone
    (core/mechanics/indenter.py:7-68), its centre lowered 0.04 A between
    20-step graph replays.  Each timed with CUDA events like the plain line."""
    import torch
    from simulon_b200.barostat import AnisotropicNPTBarostat
    from simulon_b200.mechanics import SphericalIndenterForce, UniaxialTensileLoader
    x, L = bcc(args.n)
    N = len(x)
    v = mb_velocities(N, 300.0, 4000 + int(os.environ.get("RANK", "0")))
    parser = sb.EAMParser(pot)
    out = {}
    for name in ("tensile", "indentation"):
        mol = sb.AtomFileReader.from_arrays(["W"] * N, x, L, parser.cutoff, device=dev, skin_thickness=0.5,
                                            is_fs=True)
        integ = sb.VerletIntegrator(mol, dt=0.002, ensemble="NVE")
        mol.atom_velocities = torch.tensor(v, device=dev)
        ff = sb.EAMForceCUDAExt(parser, mol)
        eng = mol.engine
        if name == "tensile":
            baro = AnisotropicNPTBarostat(mol, [0.0, 0.0, 0.0], temperature_k=300.0, control_axes=(False, True, True))
            loader = UniaxialTensileLoader(mol, axis=0, strain_rate=0.1)
            model = sb.BaseModel(sb.SumBackboneInterface([ff], mol), integ, mol, barostat=baro)

            def steps(k):
                # loader and MD steps captured together in CUDA graphs; the
                # loader's bookkeeping runs on the device (no per-step host read)
                loader.run(model, k, 0.002, graph_steps=args.graph_steps)
                return model._outputs()
        else:
            top = float(x[:, 2].max())
            center = np.array([0.5 * L, 0.5 * L, top + 20.0 - 1.0])
            ind = SphericalIndenterForce(mol, radius=20.0, stiffness=0.05, center=center)
            model = sb.BaseModel(sb.SumBackboneInterface([ff, ind], mol), integ, mol)
            depth = [0.0]

            def steps(k):
                o = None
                for _ in range(k // args.graph_steps):
                    depth[0] += 0.04
                    ind.set_center(center - np.array([0.0, 0.0, depth[0]]))
                    o = model.run(args.graph_steps, graph_steps=args.graph_steps)
                return o
        # the first step runs eagerly (the first call's forces), so the graph of
        # graph_steps steps is captured here and then replayed
        steps(warm_steps(args, args.graph_steps))
        torch.cuda.synchronize()
        rb0 = int(eng.flags[3].item())
        K = (args.steps // args.graph_steps) * args.graph_steps
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        settle()
        e0.record()
        o = steps(K)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        row = {"value": N * K / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / K, "steps": K, "status": eng.status(),
               "rebuilds_in_timed": int(eng.flags[3].item()) - rb0, "temperature_k": float(o["temperature"])}
        if name == "tensile":
            row["engineering_strain"] = float(loader.state[12])
            row["regrids"] = int(loader.regrids)
            row["forced_rebuilds"] = int(loader.forced_rebuilds)
            row["pressure_bar"] = [float(p) for p in o["pressure"].reshape(-1)[:3]]
        else:
            row["force_on_indenter_ev_per_a"] = [float(f) for f in ind.force_on_indenter]
            row["contact_atoms"] = int(ind.contact_atoms)
        out[name] = row
        del model, ff, integ, mol, eng
        torch.cuda.empty_cache()
    # (3) the simulator's output path (core/md_simulation.py:125-168): NVE run
    # through MDSimulator writing traj.xyz and energies.csv every 100 steps
    # from pinned asynchronous copies while the next steps run
    mol = sb.AtomFileReader.from_arrays(["W"] * N, x, L, parser.cutoff, device=dev, skin_thickness=0.5, is_fs=True)
    integ = sb.VerletIntegrator(mol, dt=0.002, ensemble="NVE")
    mol.atom_velocities = torch.tensor(v, device=dev)
    ff = sb.EAMForceCUDAExt(parser, mol)
    model = sb.BaseModel(sb.SumBackboneInterface([ff], mol), integ, mol)
    model.run(warm_steps(args, args.graph_steps), graph_steps=args.graph_steps)
    K = max(100, (args.steps // 100) * 100)
    with tempfile.TemporaryDirectory() as tmp:
        sim = sb.MDSimulator(model, num_steps=K, print_interval=100, store_outputs=False, verbose=False,
                             graph_steps=args.graph_steps, output_dir=tmp, traj_interval=100, write_energies=True)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        settle()
        e0.record()
        sim.run()
        e1.record()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        ms = e0.elapsed_time(e1)
        size = sum(os.path.getsize(os.path.join(tmp, f)) for f in os.listdir(tmp))
    out["simulator_output"] = {"value": N * K / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / K, "steps": K,
                               "wall_s": wall, "bytes_written": size, "status": mol.engine.status()}
    del sim, model, ff, integ, mol
    torch.cuda.empty_cache()
    out["config"] = {"workload": f"EAM-W BCC 2*{args.n}^3 = {N:,} atoms, synthetic FS W, dt 2 fs, 300 K: uniaxial "
                                 "tension 0.1/ps along x with anisotropic NPT at 0 bar on y, z (loader + MD steps in "
                                 "CUDA graphs); "
                                 "spherical indenter r 20 A, k 0.05 eV/A^3, lowered 0.04 A per 20-step graph; "
                                 "MDSimulator NVE writing traj.xyz and energies.csv every 100 steps",
                     "parallelism": "replicas x1"}
    return out


def lj_form(args, sb, dev, world):
    """LJ argon scaling point: FCC 4 n^3 atoms, a = 5.26 A,
    eps 0.0104 eV, sigma 3.405 A, cutoff 7.0 A, skin 0.5 A, NVE from 94.4 K
    Maxwell-Boltzmann velocities, dt 2 fs; the FP32-pair / FP64-integration
    form and the FP64 form, each timed like the plain EAM line, with the force
    RMSE of the FP32 form against the FP64 form on the same positions and the
    drift of the total energy per atom over the timed steps."""
    import torch
    import torch.distributed as dist
    n = args.lj_n
    a = 5.26
    g = np.arange(n)
    cells = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    x = ((cells[:, None, :] + basis[None]).reshape(-1, 3) * a).astype(np.float64)
    L = n * a
    N = len(x)
    m = 39.948 * 1.036427e-4
    rng = np.random.default_rng(7)
    v = rng.standard_normal((N, 3)) * np.sqrt(8.617333262e-5 * 94.4 / m)
    v -= v.mean(0)
    G = args.graph_steps
    out, f0 = {}, {}
    for name, dtype in (("fp32_pair", torch.float32), ("fp64", torch.float64)):
        old = torch.get_default_dtype()
        torch.set_default_dtype(dtype)
        try:
            mol = sb.AtomFileReader.from_arrays(["Ar"] * N, x, L, 7.0, device=dev, skin_thickness=0.5,
                                                parameter={"[0 0]": {"epsilon": 0.0104, "sigma": 3.405}})
            mol.atom_velocities = torch.tensor(v, dtype=dtype, device=dev)
            ff = sb.LennardJonesForce(mol)
            integ = sb.VerletIntegrator(mol, dt=0.002, ensemble="NVE")
            model = sb.BaseModel(sb.SumBackboneInterface([ff], mol), integ, mol)
        finally:
            torch.set_default_dtype(old)
        eng = mol.engine
        ff.compute()
        f0[name] = eng.gather("f").double()
        model.run(warm_steps(args, G), graph_steps=G)
        torch.cuda.synchronize()
        stream = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        first = model.steps_done
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        settle()
        e0.record(stream)
        model.run(args.steps, graph_steps=G)
        e1.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ms = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        k = min(args.steps, eng.log_capacity)
        rows = model.step_log(first + args.steps - k, k).cpu().numpy()
        etot = (rows[:, 0] + rows[:, 1] + rows[:, 9]) / N
        t_ns = np.arange(k) * 0.002e-3
        drift = float(np.polyfit(t_ns, etot, 1)[0]) if k > 1 else None
        out[name] = {"value": world * N * args.steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / args.steps,
                     "energy_drift_ev_per_atom_per_ns": drift, "status": eng.status(),
                     "neighbors_mean": eng.neighbor_stats()["mean"]}
        del model, mol, ff, integ, eng
        torch.cuda.empty_cache()
    rmse = float(torch.sqrt(((f0["fp32_pair"] - f0["fp64"]) ** 2).mean()))
    out["fp32_pair"]["force_rmse_vs_fp64_ev_per_a"] = rmse
    out["config"] = {"workload": f"LJ Ar FCC 4*{n}^3 = {N:,} atoms per GPU, a 5.26 A, eps 0.0104 eV, sigma 3.405 A, "
                                 "rc 7.0 A, skin 0.5 A, NVE from 94.4 K, dt 2 fs", "scaling": "weak",
                     "parallelism": f"replicas x{world}"}
    return out


def mlp_form(args, sb, pot, dev, world):
    """MLP-surrogate form: the committed surrogate weights
    (trained on the GPU by python -m simulon_b200.mlp on the engine's own EAM
    data), 1,024,000 W atoms NVT at 300 K (Langevin gamma 10/ps, dt 2 fs), EAM
    judging the force RMSE every 100 steps and taking over above 0.05 eV/A;
    the judgements run inside the timed region."""
    import torch
    import torch.distributed as dist
    from simulon_b200 import mlp
    x, L = bcc(args.n)
    N = len(x)
    v = mb_velocities(N, 300.0, 2000 + int(os.environ.get("RANK", "0")))
    parser = sb.EAMParser(pot)
    tables = sb.EAMDeviceTables(parser, dev)
    net = mlp.MLPNet.load(mlp.default_weights_path(), dev)
    eng = sb.MDEngine(x, np.zeros(N, np.int32), [M_W], np.diag([L] * 3), parser.cutoff, 0.5, velocities=v, device=dev)
    ip = sb.engine.integrator_params(eng, 0.002, langevin=True, temperature=300.0, gamma=10.0, seed=5)
    from simulon_b200 import autotune
    G0 = mlp.descriptors(eng)
    _, d0 = net.forward(G0, N)
    shapes = {"desc_group": 0, "force_group": 0, "ms": {}} if args.no_autotune else \
        autotune.tune_mlp(eng, reps=10, use_cache=False, dEdG=d0)
    run = mlp.SurrogateRun(eng, net, tables, ip, judge_every=100, tolerance=0.05)
    run.run(max(args.warmup, 100) // 100 * 100)
    torch.cuda.synchronize()
    K = max(100, args.steps // 100 * 100)
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    settle()
    e0.record(stream)
    run.run(K)
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    rm = run.rmse_history
    # the step's kernels timed alone (events, 20 launches each, after the run)
    from simulon_b200 import _lib

    def each(fn, reps=20):
        fn()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps
    k_ms = {"descriptors": each(lambda: _lib.call("sim_mlp_descriptors", eng.st_ref, _lib.ptr(run.G), eng.stream)),
            "network": each(lambda: net.forward_into(run.G, N, run.e, run.d)),
            "forces": each(lambda: _lib.call("sim_mlp_backward", eng.st_ref, _lib.ptr(run.d), eng.stream))}
    flops = 2 * (16 * 64 + 64 * 64 + 64 * 64 + 64 * 16) * N     # the four BF16 GEMMs per atom
    tf = flops / (k_ms["network"] / 1e3) / 1e12
    peak_tf, kind_tf = measured_peaks("bf16_tflops")
    return {"value": world * N * K / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / K, "steps": K,
            "kernels_ms": k_ms,
            "tensor": {"kernel": "k_mlp_fwd (Z1, Z2, dZ2 W2^T, dZ1 W1^T on tcgen05, BF16 in, FP32 in TMEM)",
                       "flops_per_atom": flops // N, "achieved": tf, "peak": peak_tf, "peak_kind": kind_tf,
                       "unit": "TFLOP/s", "frac": tf / peak_tf},
            "launch_shapes": {"desc_group": shapes["desc_group"], "force_group": shapes["force_group"],
                              "autotune_ms": shapes["ms"]},
            "force_rmse_vs_eam_ev_per_a": {"last": rm[-1] if rm else None, "max": max(rm) if rm else None,
                                           "judgements": len(rm)},
            "fell_back_to_eam": not run.use_mlp, "status": eng.status(), "net_status": int(net.status.item()),
            "config": {"workload": f"EAM-W surrogate: BCC 2*{args.n}^3 = {N:,} atoms per GPU, NVT 300 K Langevin "
                                   "gamma 10/ps, dt 2 fs, skin 0.5 A; descriptors 8 radial + 8 angular (rc 4.4 A), "
                                   "MLP 16-64-64-1 SiLU, BF16 tensor-core GEMMs with FP32 accumulation",
                       "judge": "EAM force RMSE every 100 steps (inside the timed region), fallback above 0.05 eV/A",
                       "training": mlp.TRAINING_NOTE}}


def e2e(model, mol, x, v, args, dev):
    """Same metric through the public API with host buffers: pinned H2D of the
    state, K steps, D2H of every step's scalars and of the final state into
    pinned buffers.  The state crosses in the API's dtype (the reader's
    ``dtype``, torch's default as in the reference reader: float32 here),
    which is what ``update_coordinates`` takes and ``coordinates`` /
    ``atom_velocities`` return.  One untimed pass of the same path first (it
    loads the kernels this path uses that the device-resident run does
    not)."""
    import torch
    N = len(x)
    io = mol.dtype
    xh = torch.tensor(x, dtype=io).pin_memory()
    vh = torch.tensor(v, dtype=io).pin_memory()
    K = args.steps
    G = args.graph_steps
    log_h = torch.empty(K, model.engine.log.shape[1], dtype=torch.float64).pin_memory()
    x_out = torch.empty(N, 3, dtype=io).pin_memory()
    v_out = torch.empty(N, 3, dtype=io).pin_memory()

    def one_pass(n_steps):
        mol.update_coordinates(xh, velocities=vh)     # H2D of both + cell sort + list build
        done = 0
        while done < n_steps:
            k = min(G * 5, n_steps - done)
            model.run(k, graph_steps=G)
            log_h[done:done + k].copy_(model.step_log(model.steps_done - k, k), non_blocking=True)
            done += k
        x_out.copy_(mol.coordinates, non_blocking=True)
        v_out.copy_(mol.atom_velocities, non_blocking=True)
        torch.cuda.synchronize()
    one_pass(min(K, G * 5))
    t0 = time.perf_counter()
    one_pass(K)
    dt = time.perf_counter() - t0
    assert torch.isfinite(x_out).all() and torch.isfinite(v_out).all() and torch.isfinite(log_h).all()
    row_bytes = log_h.shape[1] * 8
    state_bytes = 2 * N * 3 * x_out.element_size()
    return {"value": N * K / dt, "unit": UNIT, "h2d_bytes_per_step": state_bytes / K,
            "d2h_bytes_per_step": row_bytes + state_bytes / K, "seconds": dt, "io_dtype": str(io).split(".")[-1],
            "path": "AtomFileReader.update_coordinates(x, velocities=v) -> BaseModel.run -> coordinates/velocities + "
                    "step log"}


if __name__ == "__main__":
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_b200(a)
