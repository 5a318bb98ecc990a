"""The mixed form's tensor-core LU update on a strongly graded mesh.

The update stages U12 column by column with a power-of-two scale chosen from
each column's largest entry (FP16 high and low parts).  On a sphere whose
elements shrink towards one pole by up to three orders of magnitude in area,
the matrix columns (one per vertex, scaled by the vertex's support) span the
same range, so a single scale for all columns would leave the small columns
with few significant bits.  Per-column scaling keeps the factorisation as
accurate as on a uniform mesh: the FP64 refinement converges in at most two
iterations, and the mixed solution agrees with the FP64 form to 1e-5 per
column (the FP32 assembly's own error on this less well-conditioned system
sets that floor, not the LU).
"""
import math

import numpy as np
import pytest

from beat_engine_b200 import _lib
from beat_engine_b200 import mesh as M

pytestmark = pytest.mark.gpu


def graded_sphere(sub: int, power: float) -> M.BoundaryMesh:
    """Icosphere of radius 0.1 m with each vertex's polar angle t mapped to
    pi (t / pi)^power: elements near the north pole shrink (the map is
    monotone, so the mesh stays valid)."""
    s = M.reference_sphere(0.1, sub)
    d = s.vertices / np.linalg.norm(s.vertices, axis=1, keepdims=True)
    t = np.arccos(np.clip(d[:, 2], -1.0, 1.0))
    ph = np.arctan2(d[:, 1], d[:, 0])
    t2 = math.pi * (t / math.pi) ** power
    v = 0.1 * np.stack([np.sin(t2) * np.cos(ph), np.sin(t2) * np.sin(ph), np.cos(t2)], axis=1)
    return M.BoundaryMesh(v, s.faces, None)


def col_rel(a, b):
    return np.linalg.norm(a - b, axis=0) / np.linalg.norm(b, axis=0)


def test_graded_mesh_mixed_lu():
    m = graded_sphere(4, 2.0)
    area_ratio = m.areas.max() / m.areas.min()
    assert area_ratio > 300.0  # the grading this test is about
    ctx = _lib.Context(0)
    try:
        ctx.set_mesh(m.vertices, m.faces, 4, 4)
        rng = np.random.default_rng(7)
        q = np.zeros((m.num_faces, 3), complex)
        q[:, 0] = m.normals[:, 2]
        q[:, 1:] = rng.standard_normal((m.num_faces, 2)) + 1j * rng.standard_normal((m.num_faces, 2))
        for f in (500.0, 4000.0):
            k = 2 * math.pi * f / 343.0
            p64, d64 = ctx.solve(k, 1 / k, q, _lib.Context.opts(_lib.FP64))
            pmx, dmx = ctx.solve(k, 1 / k, q, _lib.Context.opts(_lib.MIXED_FP32_IR))
            assert dmx["ir_converged"] == 1 and dmx["ir_iterations"] <= 2, (f, dmx)
            assert np.all(col_rel(pmx, p64) <= 1e-5), (f, col_rel(pmx, p64))
    finally:
        ctx.close()
