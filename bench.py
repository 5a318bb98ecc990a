#!/usr/bin/env python
"""Headline benchmark: frequency-solves/s of the exterior Burton-Miller
direct-system path on the oscillating-sphere workload.

Workload (one "step" = one frequency solve): icosphere of radius 0.1 m
subdivided 5 times (F = 20,480 faces, N = 10,242 P1 unknowns), R = 16
excitations (RHS 0 a rigid translation along z, i.e. u_n = n_f . z; RHS 1-15
seeded complex normal velocities, default_rng(1000 + r), Re/Im ~ N(0,1)),
air c = 343 m/s, rho = 1.21 kg/m^3, frequencies cycling 0.5 / 2 / 6 kHz,
order-4 regular and singular rules, exp(-i omega t).  A frequency solve is
assembly + one LU + R-column solve (+ FP64 GMRES refinement in the mixed
form) + the far-field pattern at 541 directions (360 equator + 181 meridian)
for all R.

``value``: device-timed throughput of the mixed form (FP32 assembly, FP16
split tensor-core LU, FP64 GMRES refinement) with q already in HBM: the K
timed steps (frequencies) run as one beat_b200_sweep_device call, which
pipelines them over up to six solve lanes (one frequency's assembly beside
another's factorisation).
``e2e``: the same K frequencies through the host C-ABI sweep (beat_b200_sweep)
from pinned host buffers, results copied back to the host.
``fp64_value`` / ``fp64_e2e``: the same for the plain FP64 form (four lanes),
on its own context; ``speedup_vs_fp64`` = value / fp64_value.
``accuracy``: per-RHS relative L2 error of the timed mixed solutions against
the timed FP64 solutions of the same frequencies, and of both forms against
the FP64 oracle's solution of this workload (tests/golden/headline_F20480.npz),
at 0.5, 2 and 6 kHz; computed after the timed regions.
``stages_ms`` are one frequency solved alone.

``--impl reference`` times the CPU restatement of the reference's FP64 path
(oracle/, OpenMP on all host cores + LAPACK LU) piece by piece (CpuRecipe) and
reports the freq-solves/s it accounts for.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "freq-solves/s at N=20480 ≤1e-6 rel err: mixed FP32+IR vs FP64 LU, 1 B200"
UNIT = "freq-solves/s"
FREQS = (500.0, 2000.0, 6000.0)
C0, RHO = 343.0, 1.21


def workload(sub: int, R: int):
    from beat_engine_b200 import mesh as M
    mesh = M.reference_sphere(0.1, sub)
    F = mesh.num_faces
    vel = np.zeros((F, R), dtype=np.complex128)
    vel[:, 0] = mesh.normals[:, 2]
    for r in range(1, R):
        rng = np.random.default_rng(1000 + r)
        vel[:, r] = rng.standard_normal(F) + 1j * rng.standard_normal(F)
    dirs = M.equator_meridian_directions(360, 181)
    return mesh, vel, dirs


def neumann(vel, f):
    om = 2 * math.pi * f
    return 1j * RHO * om * vel  # neumann_scale(rho, omega) * u, s = +1


# --------------------------------------------------------------------------
# clocks sampled during the timed region
# --------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def wait_first_sample(self, limit_s: float = 3.0):
        """Blocks until nvidia-smi has written its first row (or limit_s has
        passed), so that its start-up (driver queries, NVML set-up) falls
        before the timed region rather than inside it."""
        t0 = time.time()
        while self.proc is not None and time.time() - t0 < limit_s:
            self.fh.flush()
            if os.path.getsize(self.path) > 0:
                return
            time.sleep(0.02)

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for ln in open(self.path):
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())
                if any(r[3].replace(".", "").isdigit() for r in rows) else None}


# --------------------------------------------------------------------------
# CPU baseline: the oracle on a bounded sample (one recipe for both CPU legs)
# --------------------------------------------------------------------------
CPU_SLICES = 16   # a frequency's assembly is cut into 16 equal slices of test faces
CPU_FREQ = 2000.0


class CpuRecipe:
    """The FP64 CPU restatement of the reference path (oracle/: assembly in
    C/OpenMP, LAPACK LU), timed piece by piece on the host so that one
    frequency solve of the full workload is accounted for without running all
    of it:

    * assembly: the test faces are cut into CPU_SLICES equal slices; each
      timed slice assembles its test faces against every trial face (regular
      and touching pairs) into one shared A and b without clearing them.
      ``fixed`` is the rest of an assembly (clearing A and b, the identity
      term, set-up), timed once; ``overhead`` is the per-call set-up that a
      slice call repeats (timed once with an empty slice) and is taken out of
      every slice.  One frequency's assembly = fixed + sum over all slices of
      (slice - overhead), unmeasured slices at the measured mean;
    * LU: one full LAPACK zgetrf + zgetrs of the N x N system with R columns,
      timed in full;
    * far field: the full 541-direction far field of all R columns, timed.

    Nothing is scaled by a power law: every piece is timed at the full size."""

    def __init__(self, mesh, vel, dirs, threads):
        import oracle
        self.oracle = oracle
        self.mesh, self.vel, self.dirs, self.threads = mesh, vel, dirs, threads
        self.F, self.N, self.R = mesh.num_faces, mesh.num_vertices, vel.shape[1]
        self.k = 2 * math.pi * CPU_FREQ / C0
        self.q = neumann(vel, CPU_FREQ)
        self.A = np.zeros((self.N, self.N), dtype=np.complex128, order="F")
        self.b = np.zeros((self.N, self.R), dtype=np.complex128, order="F")
        self.bounds = np.linspace(0, self.F, CPU_SLICES + 1).astype(int)
        self.slice_s = {}
        self.fixed_s = self.overhead_s = self.lu_s = self.ff_s = None

    def _assemble(self, lo, hi, flags):
        t0 = time.perf_counter()
        self.oracle.assemble(self.mesh, self.k, 1.0 / self.k, self.q, threads=self.threads, flags=flags,
                             test_range=(lo, hi), out=(self.A, self.b))
        return time.perf_counter() - t0

    def time_fixed(self):
        o = self.oracle
        self.fixed_s = self._assemble(0, 0, 0)  # clear + identity + set-up
        self.overhead_s = self._assemble(0, 0, o.NO_CLEAR | o.SKIP_IDENTITY)
        return self.fixed_s + self.overhead_s

    def time_slice(self, i):
        o = self.oracle
        j = i % CPU_SLICES
        t = self._assemble(int(self.bounds[j]), int(self.bounds[j + 1]), o.NO_CLEAR | o.SKIP_IDENTITY)
        self.slice_s.setdefault(j, []).append(t)
        return t

    def time_lu(self):
        import scipy.linalg as sl
        rng = np.random.default_rng(5)
        # the system's own values do not change LAPACK's work; a diagonally
        # weighted random matrix keeps the pivots well away from zero
        A = np.asfortranarray(rng.standard_normal((self.N, self.N)) + 1j * rng.standard_normal((self.N, self.N)))
        A[np.diag_indices(self.N)] += self.N
        B = rng.standard_normal((self.N, self.R)) + 1j * rng.standard_normal((self.N, self.R))
        t0 = time.perf_counter()
        sl.lu_solve(sl.lu_factor(A, overwrite_a=True, check_finite=False), B, check_finite=False)
        self.lu_s = time.perf_counter() - t0
        return self.lu_s

    def time_farfield(self):
        rng = np.random.default_rng(6)
        p = rng.standard_normal((self.N, self.R)) + 1j * rng.standard_normal((self.N, self.R))
        t0 = time.perf_counter()
        self.oracle.farfield(self.mesh, self.k, self.dirs, p, self.q, threads=self.threads)
        self.ff_s = time.perf_counter() - t0
        return self.ff_s

    def estimate(self):
        per = {j: statistics.median(v) - self.overhead_s for j, v in self.slice_s.items()}
        mean = statistics.mean(per.values())
        asm = self.fixed_s + sum(per.get(j, mean) for j in range(CPU_SLICES))
        total = asm + self.lu_s + self.ff_s
        parts = {"assembly_s": asm, "lu_solve_s": self.lu_s, "farfield_s": self.ff_s, "total_s": total,
                 "slices_timed": len(per), "slices": CPU_SLICES}
        return 1.0 / total, parts

    def describe(self):
        return (f"FP64 C/OpenMP restatement of the reference CPU path (oracle/) on {self.threads} host threads, "
                f"one frequency solve of this workload ({CPU_FREQ:.0f} Hz) accounted piece by piece: assembly as "
                f"{CPU_SLICES} slices of {self.F // CPU_SLICES} test faces x all {self.F} trial faces, "
                f"{len(self.slice_s)} of them timed (the rest at their mean), plus the clear/identity/set-up "
                f"part timed once; one full LAPACK zgetrf+zgetrs at N={self.N} with {self.R} RHS; the full "
                f"{self.dirs.shape[0]}-direction far field")


def cpu_baseline(mesh, vel, dirs, threads, n_slices):
    r = CpuRecipe(mesh, vel, dirs, threads)
    r.time_fixed()
    for i in range(n_slices):
        r.time_slice(i)
    r.time_lu()
    r.time_farfield()
    v, parts = r.estimate()
    return v, parts, r.describe()


def run_reference(args):
    """--impl reference: the CPU restatement of the reference path on the host.
    A step is one slice of a frequency's assembly (1/CPU_SLICES of its test
    faces); the LU and the far field are timed once, in full, after the
    steps.  value = one over the accounted seconds of one frequency solve."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    mesh, vel, dirs = workload(args.sub, args.rhs)
    t_start = time.perf_counter()
    r = CpuRecipe(mesh, vel, dirs, threads)
    r.time_fixed()
    for i in range(args.warmup):  # untimed: first touches of A and the oracle's caches
        r._assemble(int(r.bounds[i % CPU_SLICES]), int(r.bounds[i % CPU_SLICES + 1]),
                    r.oracle.NO_CLEAR | r.oracle.SKIP_IDENTITY)
    step_s = [r.time_slice(i) for i in range(args.steps)]
    r.time_lu()
    r.time_farfield()
    value, parts = r.estimate()
    timed_s = sum(step_s) + r.lu_s + r.ff_s + r.fixed_s + r.overhead_s
    sample = (r.describe() + f"; a step is one assembly slice ({args.steps} timed after {args.warmup} warm-up); "
              f"accounted seconds per frequency solve {json.dumps({k: round(v, 2) for k, v in parts.items()})}; "
              f"measured seconds in this run {timed_s:.1f} (wall {time.perf_counter() - t_start:.1f})")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(step_s), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": config_dict(args, mesh), "impl": "reference",
            "step_basis": f"one of {CPU_SLICES} assembly slices of a frequency solve; value accounts a whole "
                          "frequency solve (all slices, LU and far field, each timed)",
            "timed_region_s": timed_s,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def config_dict(args, mesh):
    return {"workload": f"oscillating sphere: icosphere a=0.1 m subdivided {args.sub} times "
                        f"(F={mesh.num_faces} faces, N={mesh.num_vertices} P1 dofs), R={args.rhs} RHS, "
                        "f cycling 0.5/2/6 kHz, order 4/4, far field at 541 directions",
            "faces": mesh.num_faces, "dofs": mesh.num_vertices, "rhs": args.rhs,
            "precision_form": "mixed (FP32 assembly, FP32 LU with FP16-split tensor-core updates (22 significant bits), FP64 GMRES refinement); "
                              "the FP64 form timed beside it", "lu_split_terms": args.split,
            "l2": "inputs larger than L2: every step rewrites A (N^2 complex) and the N x F RHS operator",
            "parallelism": f"frequency replicas x{args.gpus} (no collective); "
                           + ("up to 6 solve lanes per GPU, 4 in the FP64 form" if args.lanes == 0
                              else f"{args.lanes} solve lane(s) per GPU")
                           + " (pipelined frequency sweep, each lane takes the next frequency when it finishes one)"}


# --------------------------------------------------------------------------
# GPU arm
# --------------------------------------------------------------------------
def count_launches(fn):
    """Kernels of libbeatb200 launched by fn(), counted by the CUDA profiler."""
    import torch
    from torch.profiler import ProfilerActivity, profile
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        fn()
        torch.cuda.synchronize()
    n = 0
    for ev in prof.events():
        if ev.device_type is not None and "cuda" in str(ev.device_type).lower() and "bb::" in ev.name:
            n += 1
    return n


class Form:
    """One precision form on its own context: the sweep lanes of each form
    stay allocated, so neither form's timed sweep pays for the other's."""

    def __init__(self, lib, mesh, device, precision, split, lanes=0):
        import torch
        self.lib = lib
        self.precision = precision
        self.ctx = lib.Context(device)
        self.ctx.set_mesh(mesh.vertices, mesh.faces, 4, 4)
        self.opts = lib.Context.opts(precision, lu_split_terms=split, sweep_lanes=lanes)
        self.stream = torch.cuda.ExternalStream(self.ctx.stream_handle(), device=torch.device("cuda", device))

    def sweep(self, ks, qs, ps, dirs, ffs):
        return self.ctx.sweep_device(ks, 1.0 / ks, qs.data_ptr(), qs.shape[1], ps.data_ptr(), self.opts, dirs,
                                     ffs.data_ptr())


def timed(stream, fn, clocks_device=None):
    """CUDA-event milliseconds of fn() on `stream` (the library's stream: the
    sweep returns after every lane finished, so its end event follows all of
    its work), with the SM clocks sampled meanwhile when clocks_device is set."""
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(clocks_device) if clocks_device is not None else None
    if sampler:
        sampler.__enter__()
        sampler.wait_first_sample()
    try:
        torch.cuda.synchronize()
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
    finally:
        if sampler:
            sampler.__exit__(None, None, None)
    return e0.elapsed_time(e1), out, (sampler.summary() if sampler else None)


def oracle_gold(args):
    """The oracle's FP64 solution of this workload (tests/golden/headline_F20480.npz,
    made by tests/golden/make_headline_fixtures.py), when the workload is that one."""
    path = os.path.join(ROOT, "tests", "golden", "headline_F20480.npz")
    if args.sub != 5 or args.rhs != 16 or not os.path.exists(path):
        return None
    g = dict(np.load(path))
    rng = np.random.default_rng(77)
    n = 10242
    g["W"] = rng.standard_normal((n, 8)) + 1j * rng.standard_normal((n, 8))
    return g


def errors_vs_oracle(gold, f, p, ff):
    """Per-column relative errors of one frequency's solution p (N x R) and far
    field ff (M x R) against the oracle: the stored full columns, the probe
    sketch of every column and the far field of every column (max of each)."""
    tag = f"_{int(f)}"
    keep = list(gold["keep"])
    ref = gold["p_cols" + tag]
    e_cols = np.linalg.norm(p[:, keep] - ref, axis=0) / np.linalg.norm(ref, axis=0)
    e_proj = np.sqrt(np.mean(np.abs(gold["W"].T @ p - gold["proj" + tag]) ** 2, axis=0)) / gold["pnorm" + tag]
    fref = gold["ff" + tag]
    e_ff = np.linalg.norm(ff - fref, axis=0) / np.linalg.norm(fref, axis=0)
    return float(max(e_cols.max(), e_proj.max())), float(e_ff.max())


def run_gpu(args):
    import torch
    import torch.distributed as dist

    from beat_engine_b200 import _lib, sharding

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    mesh, vel, dirs = workload(args.sub, args.rhs)
    F, N, R, M = mesh.num_faces, mesh.num_vertices, args.rhs, dirs.shape[0]
    K = args.steps

    # this rank's share of the job's frequency list (round-robin, as
    # beat_engine_b200.sharding splits a multi-GPU sweep); each rank solves
    # its own frequencies, nothing crosses between ranks
    share = sharding.partition(world * (K + args.warmup + 16), world)[rank]

    def freq(i):
        return FREQS[share[i] % len(FREQS)]

    # device-resident inputs: q per frequency (F x R column-major = R x F row-major)
    q_dev = {f: torch.from_numpy(np.ascontiguousarray(neumann(vel, f).T)).to(dev) for f in FREQS}

    def sweep_inputs(i0, n):
        fs = [freq(i0 + j) for j in range(n)]
        ks = np.array([2 * math.pi * f / C0 for f in fs])
        qs = torch.stack([q_dev[f] for f in fs])  # n x R x F: frequency-major F x R column-major slices
        ps = torch.empty((n, R, N), dtype=torch.complex128, device=dev)
        ffs = torch.empty((n, R, M), dtype=torch.complex128, device=dev)
        return fs, ks, qs, ps, ffs

    def max_over_ranks(ms):
        if world == 1:
            return ms
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def run_form(form, n_steps):
        # warm-up: twice at least one frequency per lane, so every lane exists,
        # holds its workspace and has run its captured factorisation once
        # before the timed sweep
        _, ks, qs, ps, ffs = sweep_inputs(0, max(args.warmup, 6))
        form.sweep(ks, qs, ps, dirs, ffs)
        form.sweep(ks, qs, ps, dirs, ffs)
        fs, ks, qs, ps, ffs = sweep_inputs(args.warmup, n_steps)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ms, diags, clk = timed(form.stream, lambda: form.sweep(ks, qs, ps, dirs, ffs), clocks_device=local)
        ms = max_over_ranks(ms)
        return ms, diags, clk, fs, ps, ffs

    def run_e2e(form, n_steps):
        """The same K frequencies through the host C-ABI sweep (beat_b200_sweep):
        q from pinned host memory in, p and the far field back to the host."""
        fs = [freq(args.warmup + i) for i in range(n_steps)]
        ks = np.array([2 * math.pi * f / C0 for f in fs])
        q_pin = torch.stack([torch.from_numpy(np.ascontiguousarray(neumann(vel, f).T)) for f in fs]).pin_memory()
        qh = q_pin.numpy().transpose(2, 1, 0)  # F x R x n, column-major view of pinned memory
        form.ctx.sweep(ks[:2], 1.0 / ks[:2], qh[:, :, :2], form.opts, dirs)  # sizes the lanes' staging (untimed)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ms, _, _ = timed(form.stream, lambda: form.ctx.sweep(ks, 1.0 / ks, qh, form.opts, dirs))
        return max_over_ranks(ms)

    mixed = Form(_lib, mesh, local, _lib.MIXED_FP32_IR, args.split, args.lanes)
    ms, sweep_diags, clocks, fs, ps_mixed, ff_mixed = run_form(mixed, K)
    value = world * K / (ms / 1e3)
    e2e_ms = run_e2e(mixed, K)
    e2e_value = world * K / (e2e_ms / 1e3)

    fp64 = None
    if not args.no_fp64:
        fp64 = Form(_lib, mesh, local, _lib.FP64, args.split, args.lanes)
        ms64, diags64, clocks64, fs64, ps_64, ff_64 = run_form(fp64, K)
        fp64_value = world * K / (ms64 / 1e3)
        fp64_e2e = world * K / (run_e2e(fp64, K) / 1e3)

    # accuracy of the timed mixed solutions against the timed FP64 solutions of
    # the same frequencies, and of both against the oracle (outside the timed regions)
    acc = None
    if rank == 0:
        pm = ps_mixed.cpu().numpy()
        fm = ff_mixed.cpu().numpy()
        acc = {"basis": "per-RHS relative L2 error of the timed sweeps' solutions (N x 16 per frequency)",
               "by_frequency_hz": {}}
        gold = oracle_gold(args)
        p64 = ps_64.cpu().numpy() if fp64 else None
        f64 = ff_64.cpu().numpy() if fp64 else None
        for f in FREQS:
            idx = [i for i, x in enumerate(fs) if x == f]
            if not idx:
                continue
            row = {}
            if fp64:
                e = [np.linalg.norm(pm[i] - p64[i], axis=1) / np.linalg.norm(p64[i], axis=1) for i in idx]
                row["mixed_vs_fp64_form_max"] = float(np.max(e))
            if gold is not None:
                i = idx[0]
                row["mixed_vs_oracle_max"], row["mixed_farfield_vs_oracle_max"] = errors_vs_oracle(
                    gold, f, pm[i].T, fm[i].T)
                if fp64:
                    row["fp64_vs_oracle_max"], row["fp64_farfield_vs_oracle_max"] = errors_vs_oracle(
                        gold, f, p64[i].T, f64[i].T)
            acc["by_frequency_hz"][str(int(f))] = row
        vals = [v for r in acc["by_frequency_hz"].values() for k2, v in r.items() if k2.startswith("mixed_vs")]
        acc["max_rel_err"] = float(max(vals)) if vals else None
        acc["within_1e-6"] = bool(vals) and max(vals) <= 1e-6
        acc["oracle"] = ("FP64 oracle (oracle/ assembly + LAPACK) solutions stored in "
                         "tests/golden/headline_F20480.npz" if gold is not None else "unavailable for this workload")
    del ps_mixed, ff_mixed
    if fp64:
        del ps_64, ff_64

    # stage times of one frequency solved alone (not timed into value)
    def stages_of(form):
        p_dev = torch.empty((R, N), dtype=torch.complex128, device=dev)
        ff_dev = torch.empty((R, M), dtype=torch.complex128, device=dev)
        diags = []
        for f in FREQS:
            k = 2 * math.pi * f / C0
            diags.append(form.ctx.solve_device(k, 1.0 / k, q_dev[f].data_ptr(), R, p_dev.data_ptr(), form.opts))
            form.ctx.farfield_device(k, dirs, R, p_dev.data_ptr(), q_dev[f].data_ptr(), ff_dev.data_ptr())
        torch.cuda.synchronize()
        st = {k2: round(float(np.mean([d[k2] for d in diags])), 3)
              for k2 in ("assembly_ms", "regular_ms", "singular_ms", "lu_ms", "solve_ms", "ir_ms")}
        st["ir_iterations"] = float(np.mean([d["ir_iterations"] for d in diags]))
        return st, (lambda: (form.ctx.solve_device(2 * math.pi * FREQS[0] / C0, C0 / (2 * math.pi * FREQS[0]),
                                                   q_dev[FREQS[0]].data_ptr(), R, p_dev.data_ptr(), form.opts),
                             form.ctx.farfield_device(2 * math.pi * FREQS[0] / C0, dirs, R, p_dev.data_ptr(),
                                                      q_dev[FREQS[0]].data_ptr(), ff_dev.data_ptr())))

    stages, one_step = stages_of(mixed)
    stages64 = stages_of(fp64)[0] if fp64 else None

    launches = None
    if rank == 0:
        try:
            launches = count_launches(one_step) * K
        except Exception as exc:  # profiler unavailable: report the failure, not a guess
            launches = f"unavailable: {exc}"

    if rank == 0:
        peaks = measured_peaks()
        roof = roofline(args, mesh, stages, peaks)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
                "warmup": args.warmup, "ms_per_step": ms / K, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "c64 (fp16x2-split tensor LU) + c128 refinement",
                "data": "synthetic (seeded velocities on a generated icosphere)",
                "config": config_dict(args, mesh), "stages_ms": stages,
                "stages_basis": "one frequency solved alone (stage times inside the sweep overlap)",
                "sweep_ir_converged": all(d["ir_converged"] == 1 for d in sweep_diags),
                "roofline": roof, "clocks": clocks, "gpu_launches": launches,
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": F * R * 16 + M * 24,
                        "d2h_bytes_per_step": N * R * 16 + M * R * 16, "steps": K}}
        if fp64:
            line.update({"fp64_value": fp64_value, "fp64_e2e": fp64_e2e, "fp64_ms_per_step": ms64 / K,
                         "fp64_steps": K, "speedup_vs_fp64": value / fp64_value,
                         "speedup_vs_fp64_e2e": e2e_value / fp64_e2e, "fp64_clocks": clocks64,
                         "fp64_stages_ms": stages64})
        line["accuracy"] = acc
        if world == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            v, parts, desc = cpu_baseline(mesh, vel, dirs, threads, args.cpu_slices)
            line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                                    "sample": desc + "; accounted seconds " +
                                    json.dumps({k2: round(x, 2) for k2, x in parts.items()})}
        print(json.dumps(line), flush=True)
    mixed.ctx.close()
    if fp64:
        fp64.ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# --------------------------------------------------------------------------
# --config sweep: six uneven enclosures x 64 frequencies, batched
# --------------------------------------------------------------------------
SWEEP_MESHES = (2000, 4000, 6000, 8000, 10000, 12000)
SWEEP_FREQS = 64


def sweep_workload():
    """Rounded-box enclosures 0.2 x 0.3 x 0.25 m with a 0.05 m piston on the
    front face, jittered 5 % of the edge length (seeded), at targets of 2k-12k
    triangles; 64 log-spaced frequencies 100 Hz-8 kHz; the piston at 1 m/s
    plus 4 seeded random-velocity columns (R = 5)."""
    from beat_engine_b200 import mesh as M
    meshes, vels = [], []
    for i, nf in enumerate(SWEEP_MESHES):
        m = M.rounded_box_enclosure(nf, seed=60 + i)
        rng = np.random.default_rng(70 + i)
        v = np.zeros((m.num_faces, 5), complex)
        v[m.physical_tags == 2, 0] = 1.0
        v[:, 1:] = rng.standard_normal((m.num_faces, 4)) + 1j * rng.standard_normal((m.num_faces, 4))
        meshes.append(m)
        vels.append(v)
    return meshes, vels, np.geomspace(100.0, 8000.0, SWEEP_FREQS)


def run_sweep_config(args):
    """The batched sweep (beat_b200_sweep_batch_device, mixed form with
    refinement, lu_block per mesh and the lane count from the autotuner)
    against the per-frequency plain FP64 loop (beat_b200_solve_device, one
    (mesh, frequency) after another), both with inputs resident in HBM and
    timed with CUDA events; plus the batch end to end from host buffers, and
    the mixed results' per-column error against the FP64 loop's over all
    jobs."""
    import torch

    from beat_engine_b200 import _lib, autotune
    dev = torch.device("cuda", 0)
    meshes, vels, freqs = sweep_workload()
    ks = 2 * math.pi * freqs / C0
    ctxs, d_q, d_p, R = [], [], [], []
    for m, v in zip(meshes, vels):
        c = _lib.Context(0)
        c.set_mesh(m.vertices, m.faces, 4, 4)
        ctxs.append(c)
        q = np.stack([neumann(v, f) for f in freqs], axis=2)  # F x R x nf
        d_q.append(torch.from_numpy(np.ascontiguousarray(q.transpose(2, 1, 0))).to(dev))
        d_p.append(torch.empty((len(freqs), v.shape[1], m.num_vertices), dtype=torch.complex128, device=dev))
        R.append(v.shape[1])
    # autotuner: panel width per mesh, lane count on the largest mesh (cached in JSON)
    t0 = time.perf_counter()
    tuned = []
    for i, (c, v) in enumerate(zip(ctxs, vels)):
        fm = float(np.sqrt(freqs[0] * freqs[-1]))
        k = 2 * math.pi * fm / C0
        lanes = autotune.LANES if i == len(ctxs) - 1 else (6,)
        tuned.append(autotune.tune(c, k, 1 / k, neumann(v, fm), _lib.MIXED_FP32_IR, cache=args.tune_cache,
                                   lanes=lanes))
    tune_s = time.perf_counter() - t0
    lanes = tuned[-1]["sweep_lanes"]
    opts = [_lib.Context.opts(_lib.MIXED_FP32_IR, lu_block=t["lu_block"], sweep_lanes=lanes) for t in tuned]
    kl, el = [ks] * len(ctxs), [1 / ks] * len(ctxs)

    def batch():
        return _lib.sweep_batch_device(ctxs, kl, el, [t.data_ptr() for t in d_q], R,
                                       [t.data_ptr() for t in d_p], opts)

    stream = torch.cuda.ExternalStream(ctxs[0].stream_handle(), device=dev)
    for _ in range(max(2, args.warmup - 1)):  # every lane's factorisation captured and replayed once
        batch()
    with ClockSampler(0) as clk:
        ms, diags, _ = timed(stream, batch)
    clocks = clk.summary()
    n_jobs = len(ctxs) * len(freqs)
    p_mixed = [t.cpu().numpy() for t in d_p]
    # end to end from host buffers (pinned inputs)
    q_host = [torch.from_numpy(np.ascontiguousarray(t.cpu().numpy())).pin_memory() for t in d_q]
    qh = [x.numpy().transpose(2, 1, 0) for x in q_host]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _lib.sweep_batch(ctxs, kl, el, qh, opts)
    e2e_s = time.perf_counter() - t0
    # the per-frequency plain FP64 loop
    o64 = _lib.Context.opts(_lib.FP64)
    for c, q, p, r in zip(ctxs, d_q, d_p, R):  # warm: the FP64 workspaces
        c.solve_device(ks[0], 1 / ks[0], q[0].data_ptr(), r, p[0].data_ptr(), o64)

    def loop():
        for c, q, p, r in zip(ctxs, d_q, d_p, R):
            for f in range(len(freqs)):
                c.solve_device(ks[f], 1 / ks[f], q[f].data_ptr(), r, p[f].data_ptr(), o64)

    ms64, _, clocks64 = timed(stream, loop, clocks_device=0)
    err = 0.0
    for pm, t in zip(p_mixed, d_p):
        p64 = t.cpu().numpy()
        err = max(err, float(np.max(np.linalg.norm(pm - p64, axis=2) / np.linalg.norm(p64, axis=2))))
    line = {"metric": "batched sweep: freq-solves/s over 6 enclosures x 64 frequencies, mixed FP32+IR, 1 B200",
            "value": n_jobs / (ms / 1e3), "unit": UNIT, "n_gpus": 1, "steps": 1, "warmup": args.warmup,
            "sweep_wall_s": ms / 1e3, "higher_is_better": True, "dtype": "c64 (fp16x2-split tensor LU) + c128 refinement",
            "data": "synthetic (seeded jittered enclosures and velocities)",
            "config": {"workload": "rounded-box enclosures 0.2x0.3x0.25 m + 0.05 m piston, targets "
                                   f"{list(SWEEP_MESHES)} triangles (F = {[m.num_faces for m in meshes]}, "
                                   f"N = {[m.num_vertices for m in meshes]}), {SWEEP_FREQS} log-spaced "
                                   "frequencies 100 Hz-8 kHz, piston 1 m/s + 4 random RHS (R = 5), order 4/4",
                       "jobs": n_jobs, "lanes": lanes, "lu_block": [t["lu_block"] for t in tuned],
                       "autotune_s": tune_s, "autotune_cached": [t["cached"] for t in tuned]},
            "fp64_loop_value": n_jobs / (ms64 / 1e3), "fp64_loop_wall_s": ms64 / 1e3,
            "speedup_vs_fp64_loop": ms64 / ms,
            "e2e": {"value": n_jobs / e2e_s, "unit": UNIT, "wall_s": e2e_s,
                    "h2d_bytes_per_step": int(sum(t.numel() * 16 for t in d_q)),
                    "d2h_bytes_per_step": int(sum(t.numel() * 16 for t in d_p))},
            "accuracy": {"max_rel_err_mixed_vs_fp64_loop": err, "jobs": n_jobs,
                         "ir_converged": all(d["ir_converged"] == 1 for dm in diags for d in dm)},
            "clocks": clocks, "fp64_clocks": clocks64}
    print(json.dumps(line), flush=True)
    for c in ctxs:
        c.close()
    return 0


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d["bf16_tflops"],
                "bf16_tflops_sustained": d.get("bf16_tflops_sustained", d["bf16_tflops"]), "source": "measured"}
    except (OSError, KeyError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "source": "fallback"}


# DRAM traffic of sym_pairs_kernel<6> (the mixed form's element-pair kernel) measured by ncu on
# the F = 5,120 icosphere: 158.83 MB read + 117.60 MB written per launch, against an algorithmic
# output of A (N^2 c64) + B (N x F c64) = 157.4 MB at N = 2,562.  Traffic grows with the output
# written (the zeroed A and B are read back by the red.global.add flush), so a launch on another
# mesh is scaled by its output bytes.
SYM_TRAFFIC_F5120 = {"bytes": 158.8288e6 + 117.59616e6, "output_bytes": 2562 * 2562 * 8 + 2562 * 5120 * 8}
FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # FP32 FMA lanes x 2 flops x max SM clock


def roofline(args, mesh, stages, peaks):
    """Roofline of the element-pair assembly kernel (sym_pairs_kernel<6>, the
    largest SM-filling kernel of the mixed form; its time is the CUDA-event
    time of its launch, stages_ms.regular_ms).

    The kernel is bound by FP32 instruction issue (FMA + MUFU), not by HBM:
    about 1,300 flops per byte it writes.  So the binding fraction is the
    compute one: achieved = 72 flops per ordered regular point pair (the
    algorithmic count of the combined Burton-Miller integrand) x the point
    pairs of one launch / its duration, against the nominal FP32 FMA rate
    (MEASURED_PEAKS.json holds no FP32 SIMT peak).  The HBM figures beside it:
    algorithmic bytes = A (N^2) + the RHS operator B (N x F), c64; traffic =
    ncu DRAM bytes of the F = 5,120 launch scaled by output bytes."""
    F, N = mesh.num_faces, mesh.num_vertices
    regular_pairs = F * F - (13 * F - 60)
    point_pairs = 36 * regular_pairs
    alg_bytes = N * N * 8 + N * F * 8
    t = stages["regular_ms"] / 1e3
    flops = point_pairs * 72.0
    achieved = flops / t / 1e12 if t > 0 else None
    gbs = alg_bytes / t / 1e9 if t > 0 else None
    traffic = SYM_TRAFFIC_F5120["bytes"] * alg_bytes / SYM_TRAFFIC_F5120["output_bytes"]
    return {"kernel": "sym_pairs_kernel<6> (element-pair Galerkin assembly, both orders per unordered pair)",
            "bound": "fp32_issue", "achieved": achieved, "peak": FP32_NOMINAL_TFLOPS, "unit": "TFLOP/s",
            "frac": (achieved / FP32_NOMINAL_TFLOPS) if achieved else None,
            "peak_source": "nominal FP32 FMA issue: 148 SMs x 128 lanes x 2 flops x 1965 MHz",
            "flops_per_launch": flops, "point_pairs_per_launch": point_pairs, "flops_per_point_pair": 72,
            "traffic": traffic,
            "traffic_basis": "ncu dram read+write of the F=5,120 launch scaled by output bytes",
            "hbm": {"achieved": gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                    "frac": (gbs / peaks["hbm_gbs"]) if gbs else None,
                    "algorithmic_bytes_per_launch": alg_bytes,
                    "peak_source": "measured hbm_gbs (MEASURED_PEAKS.json)" if peaks["source"] == "measured"
                    else "fallback 6.65 TB/s"}}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=24)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--split", type=int, default=3, choices=(1, 3))
    ap.add_argument("--sub", type=int, default=5)
    ap.add_argument("--rhs", type=int, default=16)
    ap.add_argument("--cpu-slices", type=int, default=2,
                    help="assembly slices timed by the cpu_baseline leg (of %d per frequency)" % CPU_SLICES)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 arm")
    ap.add_argument("--config", choices=("headline", "sweep"), default="headline",
                    help="sweep: the batched 6-enclosure x 64-frequency sweep against the FP64 loop")
    ap.add_argument("--tune-cache", default=None, help="autotuner JSON cache (default ~/.cache/beat_b200)")
    ap.add_argument("--lanes", type=int, default=0,
                    help="frequencies in flight in the sweep (0: the library's default); 1 runs them one after "
                         "another on one host thread, as a profiler capture wants")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "b200":
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)
    if args.config == "sweep":
        return run_sweep_config(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
