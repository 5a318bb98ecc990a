"""The adjoint-gradient workload at its specified size, shared by its fixture
generator (make_config4_fixtures.py) and its GPU test (test_config4_gradient.py).

A rounded-box loudspeaker enclosure 0.2 x 0.3 x 0.25 m with a circular piston
of radius 0.05 m on the front face, meshed at a target of 5,120 triangles
(5,228 faces, 2,616 vertices), every vertex moved along its normal by 2 % of
the edge length times a seeded Gaussian.  Eight frequencies log-spaced from
250 Hz to 4 kHz.  Excitation: the piston at 1 m/s plus a seeded complex
velocity of 0.1 m/s on every face (one right-hand side).  Objective over the
72 far-field directions of the horizontal +-90 deg arc:

    J = sum_f sum_d w_d (L_fd - t_f)^2,   L = 10 log10 |p_inf|^2,

with w_d = 2 within 30 deg of the axis and 1 elsewhere, and t_f the flat
target given with the case (the oracle's mean level of the design point
without admittance at that frequency, stored in the fixture).
"""
from __future__ import annotations

import math

import numpy as np

C0, RHO = 343.0, 1.21
DB = 10.0 / math.log(10.0)
FREQS = np.geomspace(250.0, 4000.0, 8)


def mesh():
    from beat_engine_b200 import mesh as M
    base = M.rounded_box_enclosure(5120, seed=31)
    rng = np.random.default_rng(32)
    f = np.asarray(base.faces)
    vn = np.zeros((base.num_vertices, 3))
    for a in range(3):
        np.add.at(vn, f[:, a], base.normals * base.areas[:, None])
    vn /= np.linalg.norm(vn, axis=1)[:, None]
    h = math.sqrt(2.0 * base.areas.sum() / base.num_faces)
    X = np.asarray(base.vertices) + 0.02 * h * rng.standard_normal(base.num_vertices)[:, None] * vn
    return M.BoundaryMesh(X, f, np.asarray(base.physical_tags))


def velocity(m):
    rng = np.random.default_rng(33)
    F = m.num_faces
    return np.where(m.physical_tags == 2, 1.0, 0.0) + 0.1 * (rng.standard_normal(F) + 1j * rng.standard_normal(F))


def admittance(m):
    """The admittance of the GPU check's design point (per face, normal-velocity
    admittance Y, a = neumann_scale Y)."""
    rng = np.random.default_rng(34)
    F = m.num_faces
    return 0.002 * (rng.standard_normal(F) + 1j * rng.standard_normal(F))


def directions():
    th = np.linspace(-math.pi / 2, math.pi / 2, 72)  # +-90 deg about the front axis (+z)
    return np.stack([np.sin(th), np.zeros(72), np.cos(th)], axis=1)


def weights(dirs):
    return np.where(np.abs(dirs[:, 0]) < 0.5, 2.0, 1.0)


def levels(pinf):
    return DB * np.log(np.abs(pinf) ** 2)


def objective_of_far_fields(pinfs, targets, w):
    """J from the far fields of all frequencies (list of 72-vectors)."""
    return float(sum(np.sum(w * (levels(p) - t) ** 2) for p, t in zip(pinfs, targets)))


def gradient_g(pinf, t, w):
    """dJ/d conj(p_inf) of one frequency's term."""
    return 2 * w * (levels(pinf) - t) * DB / np.conj(pinf)


def oracle_directions(m, n=4, seed=35):
    """Directions (dv, dX) of the oracle check (no admittance change)."""
    rng = np.random.default_rng(seed)
    v = velocity(m)
    X0 = np.asarray(m.vertices)
    out = []
    for _ in range(n):
        dv = (rng.standard_normal(m.num_faces) + 1j * rng.standard_normal(m.num_faces)) * np.abs(v).mean()
        dX = rng.standard_normal(X0.shape) * np.abs(X0).mean()
        out.append((dv, dX))
    return out


def gpu_directions(m, n=64, seed=36):
    """Directions (dv, dY, dX) of the check against the GPU forward model."""
    rng = np.random.default_rng(seed)
    v, Y = velocity(m), admittance(m)
    X0 = np.asarray(m.vertices)
    out = []
    for _ in range(n):
        dv = (rng.standard_normal(m.num_faces) + 1j * rng.standard_normal(m.num_faces)) * np.abs(v).mean()
        dY = (rng.standard_normal(m.num_faces) + 1j * rng.standard_normal(m.num_faces)) * np.abs(Y).mean()
        dX = rng.standard_normal(X0.shape) * np.abs(X0).mean()
        out.append((dv, dY, dX))
    return out
