"""Oracle values for the adjoint-gradient workload at its specified size
(tests/golden/config4_case.py), for tests/test_config4_gradient.py.

    python tests/golden/make_config4_fixtures.py

At the design point without admittance, per frequency, the FP64 oracle
(oracle/ assembly + LAPACK + oracle far field) gives the far field and the
flat target t_f (its mean level).  Along 4 seeded directions (dv, dX) it gives
central differences (h = 1e-6) of J, the reference's own check style for a
CPU solver.  Stored in config4_oracle.npz: targets, pinf (8 x 72), J0,
fd (4), h.  72 oracle solves of a 5,228-face system: minutes on a few cores.
"""
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

import config4_case as case  # noqa: E402

H = 1e-6


def far_fields(m, v):
    import oracle
    from beat_engine_b200.phasor import neumann_scale
    out = []
    dirs = case.directions()
    for f in case.FREQS:
        k = 2 * math.pi * f / case.C0
        q = (neumann_scale(case.RHO, 2 * math.pi * f) * v)[:, None]
        A, b = oracle.assemble(m, k, 1 / k, q)
        p = np.linalg.solve(A, b)
        out.append(oracle.farfield(m, k, dirs, p, q)[:, 0])
    return out


def main():
    from beat_engine_b200 import mesh as M
    t0 = time.perf_counter()
    m = case.mesh()
    v = case.velocity(m)
    w = case.weights(case.directions())
    pinf = far_fields(m, v)
    targets = np.array([case.levels(p).mean() for p in pinf])
    J0 = case.objective_of_far_fields(pinf, targets, w)
    print(f"design point: J0 {J0:.10e} ({time.perf_counter() - t0:.0f} s)", flush=True)
    X0 = np.asarray(m.vertices)
    fd = []
    for i, (dv, dX) in enumerate(case.oracle_directions(m)):
        Jpm = []
        for sgn in (1.0, -1.0):
            mm = M.BoundaryMesh(X0 + sgn * H * dX, np.asarray(m.faces), np.asarray(m.physical_tags))
            Jpm.append(case.objective_of_far_fields(far_fields(mm, v + sgn * H * dv), targets, w))
        fd.append((Jpm[0] - Jpm[1]) / (2 * H))
        print(f"direction {i}: fd {fd[-1]:.10e} ({time.perf_counter() - t0:.0f} s)", flush=True)
    np.savez(os.path.join(HERE, "config4_oracle.npz"), targets=targets, pinf=np.array(pinf), J0=np.array(J0),
             fd=np.array(fd), h=np.array(H), faces=np.array(m.num_faces))
    print("J0", J0, "targets", targets)


if __name__ == "__main__":
    main()
