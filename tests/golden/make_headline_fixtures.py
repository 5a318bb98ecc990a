"""Oracle solutions of the headline workload, for the GPU parity tests at full size.

    python tests/golden/make_headline_fixtures.py [--threads T]

Workload (the one bench.py times): icosphere of radius 0.1 m subdivided 5
times (F = 20,480 faces, N = 10,242 P1 unknowns), R = 16 excitations (RHS 0
the rigid translation along z, u_n = n_f . z; RHS 1-15 Re, Im ~ N(0, 1) from
``numpy.random.default_rng(1000 + r)``), c = 343 m/s, rho = 1.21 kg/m^3,
exp(-i omega t), order-4 regular and singular rules, 500 Hz, 2 kHz and 6 kHz.

For each frequency the FP64 oracle assembles A and b (oracle/bem_oracle.c,
the restatement of the reference's fused CPU assembler), LAPACK (scipy)
factors A and solves all 16 columns, and the oracle evaluates the far field
at the 541 directions (360 equator + 181 meridian).  Stored per frequency
(``headline_F20480.npz``, keys suffixed ``_<Hz>``):

* ``p_cols``: the full solution of RHS 0, 1, 2 and 15 (N x 4);
* ``proj``: W^T p for all 16 columns, W = 8 complex Gaussian probe vectors
  (``default_rng(77)``, N x 8): a per-column linear sketch of every column;
* ``pnorm``: ||p_r|| for all 16 columns;
* ``ff``: the far field of all 16 columns (541 x 16);
* ``residual``: max_r ||A p_r - b_r|| / ||b_r|| of the oracle solve;
* ``dipole_err``: relative L2 distance of RHS 0's far field from the analytic
  oscillating-sphere (l = 1) far field.

Timings of the full oracle solve are stored beside them (``seconds_*``,
``threads``).  Nothing at test time runs the oracle at this size; the tests
read this file.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

FREQS = (500.0, 2000.0, 6000.0)
C0, RHO, RADIUS = 343.0, 1.21, 0.1
KEEP = (0, 1, 2, 15)
PROBES, PROBE_SEED = 8, 77


def workload():
    from beat_engine_b200 import mesh as M
    mesh = M.reference_sphere(RADIUS, 5)
    F, R = mesh.num_faces, 16
    vel = np.zeros((F, R), dtype=np.complex128)
    vel[:, 0] = mesh.normals[:, 2]
    for r in range(1, R):
        rng = np.random.default_rng(1000 + r)
        vel[:, r] = rng.standard_normal(F) + 1j * rng.standard_normal(F)
    return mesh, vel, M.equator_meridian_directions(360, 181)


def probes(n):
    rng = np.random.default_rng(PROBE_SEED)
    return rng.standard_normal((n, PROBES)) + 1j * rng.standard_normal((n, PROBES))


def dipole_farfield(dirs, k, omega):
    """Far field lim r e^{-ikr} p(r d) of the rigid sphere oscillating along z
    with unit velocity, exp(-i omega t): p = i rho omega h1(kr) cos(theta) /
    (k h1'(ka)) with h1(z) = -e^{iz}(z + i)/z^2 (tests/axial_source_tests.jl:90-100),
    and r h1(kr) e^{-ikr} -> -1/k."""
    z = k * RADIUS
    dh1 = np.exp(1j * z) * (-1j / z + 2 / z ** 2 + 2j / z ** 3)
    return 1j * RHO * omega * (-1.0 / k) / (k * dh1) * dirs[:, 2]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--out", default=os.path.join(HERE, "headline_F20480.npz"))
    args = ap.parse_args()
    import scipy.linalg as sl

    import oracle
    mesh, vel, dirs = workload()
    W = probes(mesh.num_vertices)
    out = {"keep": np.array(KEEP), "frequencies": np.array(FREQS)}
    meta = {}
    for f in FREQS:
        om = 2 * math.pi * f
        k = om / C0
        q = 1j * RHO * om * vel
        t0 = time.perf_counter()
        A, b = oracle.assemble(mesh, k, 1.0 / k, q, threads=args.threads)
        t1 = time.perf_counter()
        lu = sl.lu_factor(A, check_finite=False)
        p = sl.lu_solve(lu, b, check_finite=False)
        t2 = time.perf_counter()
        ff = oracle.farfield(mesh, k, dirs, p, q, threads=args.threads)
        t3 = time.perf_counter()
        res = np.linalg.norm(A @ p - b, axis=0) / np.linalg.norm(b, axis=0)
        del lu, A
        ana = dipole_farfield(dirs, k, om)
        derr = float(np.linalg.norm(ff[:, 0] - ana) / np.linalg.norm(ana))
        tag = f"_{int(f)}"
        out["p_cols" + tag] = p[:, KEEP]
        out["proj" + tag] = W.T @ p
        out["pnorm" + tag] = np.linalg.norm(p, axis=0)
        out["ff" + tag] = ff
        out["residual" + tag] = np.array(res.max())
        out["dipole_err" + tag] = np.array(derr)
        meta[str(int(f))] = {"assembly_s": t1 - t0, "lu_solve_s": t2 - t1, "farfield_s": t3 - t2,
                             "residual": float(res.max()), "dipole_err": derr}
        print(f"{f:.0f} Hz: assembly {t1 - t0:.1f} s, LU+solve {t2 - t1:.1f} s, far field {t3 - t2:.1f} s, "
              f"residual {res.max():.2e}, dipole far-field error {derr:.3e}", flush=True)
    out["meta"] = np.array(json.dumps({"threads": args.threads or os.cpu_count(), "timings": meta}))
    np.savez(args.out, **out)
    print("wrote", args.out)


if __name__ == "__main__":
    main()
