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

``value``: device-timed throughput with q already in HBM: the K timed steps
(frequencies) run as one beat_b200_sweep_device call, which pipelines them over
up to six solve lanes, four in the FP64 form (one frequency's assembly beside
another's factorisation).
``e2e``: the same through the host C-ABI sweep (beat_b200_sweep) from pinned
host buffers.  ``stages_ms`` are one frequency solved alone.

``--impl reference`` times the CPU restatement of the reference's FP64 path
(oracle/, OpenMP on all host cores + LAPACK LU) on a bounded sample and
extrapolates to freq-solves/s.
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
# CPU baseline: the oracle on a bounded sample
# --------------------------------------------------------------------------
def cpu_sample(mesh, vel, dirs, sample_faces: int, lu_n: int, threads: int):
    """Time the FP64 CPU restatement on a sample and extrapolate one full
    frequency solve: regular+singular assembly of `sample_faces` test faces
    (scaled by F / sample_faces), LAPACK LU + solve at order `lu_n` (scaled by
    (N / lu_n)^3) and the far field of 8 directions (scaled by 541 / 8)."""
    import scipy.linalg as sl

    import oracle
    F, N = mesh.num_faces, mesh.num_vertices
    R = vel.shape[1]
    f = 2000.0
    k = 2 * math.pi * f / C0
    q = neumann(vel, f)
    t0 = time.perf_counter()
    oracle.assemble(mesh, k, 1.0 / k, q, test_range=(0, sample_faces), threads=threads)
    t_asm = (time.perf_counter() - t0) * F / sample_faces
    rng = np.random.default_rng(5)
    A = rng.standard_normal((lu_n, lu_n)) + 1j * rng.standard_normal((lu_n, lu_n)) + lu_n * np.eye(lu_n)
    B = rng.standard_normal((lu_n, R)) + 1j * rng.standard_normal((lu_n, R))
    t0 = time.perf_counter()
    sl.lu_solve(sl.lu_factor(A, overwrite_a=True, check_finite=False), B, check_finite=False)
    t_lu = (time.perf_counter() - t0) * (N / lu_n) ** 3
    p = rng.standard_normal((N, R)) + 1j * rng.standard_normal((N, R))
    t0 = time.perf_counter()
    oracle.farfield(mesh, k, dirs[:8], p, q, threads=threads)
    t_ff = (time.perf_counter() - t0) * dirs.shape[0] / 8
    total = t_asm + t_lu + t_ff
    return 1.0 / total, {"assembly_s": t_asm, "lu_solve_s": t_lu, "farfield_s": t_ff, "total_s": total}


def run_reference(args):
    """--impl reference: the CPU restatement of the reference path on the host."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    mesh, vel, dirs = workload(args.sub, args.rhs)
    vals, parts = [], None
    for i in range(args.warmup + args.steps):
        v, parts = cpu_sample(mesh, vel, dirs, args.ref_sample_faces, args.ref_lu_n, threads)
        if i >= args.warmup:
            vals.append(v)
    value = statistics.median(vals)
    sample = (f"per step: oracle assembly of {args.ref_sample_faces}/{mesh.num_faces} test faces x all trial faces "
              f"(scaled by F/{args.ref_sample_faces}), LAPACK zgetrf+zgetrs at N={args.ref_lu_n} with {args.rhs} RHS "
              f"(scaled by (N/{args.ref_lu_n})^3), far field of 8/541 directions (scaled); extrapolated "
              f"seconds {json.dumps({k: round(v, 2) for k, v in parts.items()})}")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 / value, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": config_dict(args, mesh), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def config_dict(args, mesh):
    return {"workload": f"oscillating sphere: icosphere a=0.1 m subdivided {args.sub} times "
                        f"(F={mesh.num_faces} faces, N={mesh.num_vertices} P1 dofs), R={args.rhs} RHS, "
                        "f cycling 0.5/2/6 kHz, order 4/4, far field at 541 directions",
            "faces": mesh.num_faces, "dofs": mesh.num_vertices, "rhs": args.rhs,
            "precision_form": args.precision, "lu_split_terms": args.split,
            "l2": "inputs larger than L2: every step rewrites A (N^2 complex) and the N x F RHS operator",
            "parallelism": f"frequency replicas x{args.gpus} (no collective); "
                           "up to 6 solve lanes per GPU, 4 in the FP64 form (pipelined frequency sweep)"}


# --------------------------------------------------------------------------
# GPU arm
# --------------------------------------------------------------------------
def count_launches(ctx, fn):
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
    mesh, vel, dirs = workload(args.sub, args.rhs)
    F, N, R, M = mesh.num_faces, mesh.num_vertices, args.rhs, dirs.shape[0]
    prec = _lib.FP64 if args.precision == "fp64" else _lib.MIXED_FP32_IR
    opts = _lib.Context.opts(prec, lu_split_terms=args.split)

    ctx = _lib.Context(local)
    ctx.set_mesh(mesh.vertices, mesh.faces, 4, 4)
    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    # device-resident inputs: q per frequency (F x R column-major = R x F row-major)
    q_dev = {f: torch.from_numpy(np.ascontiguousarray(neumann(vel, f).T)).to(dev) for f in FREQS}
    p_dev = torch.empty((R, N), dtype=torch.complex128, device=dev)
    ff_dev = torch.empty((R, M), dtype=torch.complex128, device=dev)

    # this rank's share of the job's frequency list (round-robin, as
    # beat_engine_b200.sharding splits a multi-GPU sweep); each rank solves
    # its own frequencies, nothing crosses between ranks
    share = sharding.partition(world * (args.steps + args.warmup + args.e2e_steps + 16), world)[rank]

    def freq(i):
        return FREQS[share[i] % len(FREQS)]

    def step(i, diags=None):
        # one frequency on its own (launch count, isolated stage times)
        f = freq(i)
        k = 2 * math.pi * f / C0
        d = ctx.solve_device(k, 1.0 / k, q_dev[f].data_ptr(), R, p_dev.data_ptr(), opts)
        ctx.farfield_device(k, dirs, R, p_dev.data_ptr(), q_dev[f].data_ptr(), ff_dev.data_ptr())
        if diags is not None:
            diags.append(d)

    def sweep_buffers(i0, n):
        fs = [freq(i0 + j) for j in range(n)]
        ks = np.array([2 * math.pi * f / C0 for f in fs])
        qs = torch.stack([q_dev[f] for f in fs])  # n x R x F: frequency-major F x R column-major slices
        ps = torch.empty((n, R, N), dtype=torch.complex128, device=dev)
        ffs = torch.empty((n, R, M), dtype=torch.complex128, device=dev)
        return ks, qs, ps, ffs

    def sweep(bufs):
        ks, qs, ps, ffs = bufs
        return ctx.sweep_device(ks, 1.0 / ks, qs.data_ptr(), R, ps.data_ptr(), opts, dirs, ffs.data_ptr())

    # a step is one frequency solve + far field; the K timed steps run as one
    # pipelined sweep (beat_b200_sweep_device) with their inputs resident
    warm = sweep_buffers(0, max(args.warmup, 2))
    sweep(warm)
    timed = sweep_buffers(args.warmup, args.steps)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        e0.record(stream)
        sweep_diags = sweep(timed)
        # the sweep returns after every lane finished: this event follows all of its work
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    clocks = clk.summary()
    if world > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        if world > 1:
            dist.barrier()
    value = world * args.steps / (ms / 1e3)
    del warm, timed

    # stage times of one frequency solved alone (not timed into value)
    diags = []
    for i in range(3):
        step(i, diags)

    # e2e through the host C-ABI sweep with pinned buffers
    ke = max(2, min(args.steps, args.e2e_steps))
    fs = [freq(i) for i in range(ke)]
    ks = np.array([2 * math.pi * f / C0 for f in fs])
    q_pin = torch.stack([torch.from_numpy(np.ascontiguousarray(neumann(vel, f).T)) for f in fs]).pin_memory()
    qh = q_pin.numpy().transpose(2, 1, 0)  # F x R x ke, column-major view of pinned memory
    ctx.sweep(ks, 1.0 / ks, qh, opts, dirs)  # sizes the lanes' host-staging buffers (untimed)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctx.sweep(ks, 1.0 / ks, qh, opts, dirs)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = world * ke / (e2e_ms / 1e3)
    h2d = F * R * 16 + M * 24
    d2h = N * R * 16 + M * R * 16

    # accuracy of this form against the FP64 form on the same step (not timed)
    acc = None
    if args.check_accuracy and prec != _lib.FP64 and rank == 0:
        f = freq(0)
        k = 2 * math.pi * f / C0
        qh = neumann(vel, f)
        p_mixed, _ = ctx.solve(k, 1.0 / k, qh, opts)
        p64, _ = ctx.solve(k, 1.0 / k, qh, _lib.Context.opts(_lib.FP64))
        err = np.linalg.norm(p_mixed - p64, axis=0) / np.linalg.norm(p64, axis=0)
        acc = {"frequency_hz": f, "max_rel_err_vs_fp64_gpu": float(err.max()),
               "median_rel_err_vs_fp64_gpu": float(np.median(err))}

    launches = None
    if rank == 0:
        try:
            launches = count_launches(ctx, lambda: step(0)) * args.steps
        except Exception as exc:  # profiler unavailable: report the failure, not a guess
            launches = f"unavailable: {exc}"

    if rank == 0:
        def mean(key):
            return float(np.mean([d[key] for d in diags]))
        stages = {k: round(mean(k), 3) for k in ("assembly_ms", "regular_ms", "singular_ms", "lu_ms", "solve_ms",
                                                   "ir_ms")}
        stages["ir_iterations"] = float(np.mean([d["ir_iterations"] for d in diags]))
        peaks = measured_peaks()
        roof = roofline(args, mesh, stages, peaks)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "c64 (tf32 tensor LU) + c128 refinement" if prec != _lib.FP64 else "c128",
                "data": "synthetic (seeded velocities on a generated icosphere)",
                "config": config_dict(args, mesh), "stages_ms": stages,
                "stages_basis": "one frequency solved alone (stage times inside the sweep overlap)",
                "sweep_ir_converged": all(d["ir_converged"] == 1 for d in sweep_diags) if prec != _lib.FP64 else None,
                "roofline": roof,
                "clocks": clocks, "gpu_launches": launches,
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "steps": ke}}
        if acc:
            line["accuracy"] = acc
        if world == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            v, parts = cpu_sample(mesh, vel, dirs, args.cpu_sample_faces, args.cpu_lu_n, threads)
            line["cpu_baseline"] = {
                "value": v, "unit": UNIT, "cores": threads, "kind": "port",
                "sample": (f"oracle (FP64 C/OpenMP restatement) assembly of {args.cpu_sample_faces}/{F} test faces, "
                           f"LAPACK LU at N={args.cpu_lu_n} scaled by (N/{args.cpu_lu_n})^3, far field of 8/541 "
                           f"directions; extrapolated seconds "
                           f"{json.dumps({k: round(x, 2) for k, x in parts.items()})}")}
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
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
# the F = 5,120 icosphere (profiles/sym_pairs_kernel_F5120.md): dram read + write bytes per launch
# and the algorithmic output of that launch (A: N^2 c64, B: N x F c64).  Traffic grows with the
# output written (the zeroed A and B are read back by the red.global.add flush), so a launch on
# another mesh is scaled by its output bytes.
SYM_TRAFFIC_F5120 = {"bytes": 158.986496e6 + 119.639296e6, "output_bytes": 2562 * 2562 * 8 + 2562 * 5120 * 8}


def roofline(args, mesh, stages, peaks):
    """Roofline of the element-pair assembly kernel (the dominant kernel of
    the step: sym_pairs_kernel in the mixed form, regular_pairs_kernel in
    FP64).  achieved = algorithmic bytes per launch / its CUDA-event
    duration; algorithmic bytes = the output it produces, A (N^2) and the RHS
    operator B (N x F), c64 entries in the mixed form, c128 in FP64.  The
    kernel is bound by FP32 FMA/SFU issue, not HBM: the compute fraction
    (72 flops per ordered point pair, the algorithmic count) is reported
    beside it."""
    F, N = mesh.num_faces, mesh.num_vertices
    esz = 16 if args.precision == "fp64" else 8
    regular_pairs = F * F - (13 * F - 60)
    point_pairs = 36 * regular_pairs
    alg_bytes = N * N * esz + N * F * esz
    t = stages["regular_ms"] / 1e3
    achieved = alg_bytes / t / 1e9 if t > 0 else None
    peak = peaks["hbm_gbs"]
    traffic = None
    if esz == 8:
        traffic = SYM_TRAFFIC_F5120["bytes"] * alg_bytes / SYM_TRAFFIC_F5120["output_bytes"]
    flops = point_pairs * 72.0
    fp_peak = 148 * 128 * 2 * 1.965e9 / (2 if args.precision == "fp64" else 1)
    kernel = ("regular_pairs_kernel<double, 6> (element-pair Galerkin assembly)" if esz == 16 else
              "sym_pairs_kernel<6> (element-pair Galerkin assembly, both orders per unordered pair)")
    return {"kernel": kernel, "bound": "hbm",
            "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None, "traffic": traffic,
            "traffic_basis": "ncu dram read+write of the F=5,120 launch scaled by output bytes" if traffic else None,
            "peak_source": f"{peaks['source']} hbm_gbs (MEASURED_PEAKS.json)" if peaks["source"] == "measured"
            else "fallback 6.65 TB/s",
            "algorithmic_bytes_per_launch": alg_bytes,
            "compute": {"point_pairs_per_launch": point_pairs, "flops_per_point_pair": 72,
                        "achieved_tflops": flops / t / 1e12 if t > 0 else None,
                        "peak_tflops": fp_peak / 1e12,
                        "peak_basis": "nominal FP32 (FP64 for the fp64 form) FMA issue, 148 SMs at 1965 MHz",
                        "frac": (flops / t / fp_peak) if t > 0 else None}}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=24)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--precision", choices=("mixed", "fp64"), default="mixed")
    ap.add_argument("--split", type=int, default=3, choices=(1, 3))
    ap.add_argument("--sub", type=int, default=5)
    ap.add_argument("--rhs", type=int, default=16)
    ap.add_argument("--e2e-steps", type=int, default=6)
    ap.add_argument("--cpu-sample-faces", type=int, default=640)
    ap.add_argument("--cpu-lu-n", type=int, default=4096)
    ap.add_argument("--ref-sample-faces", type=int, default=160)
    ap.add_argument("--ref-lu-n", type=int, default=2048)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--check-accuracy", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "b200":
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
