"""Symmetry images in the oracle (bo_assemble_sym, bo_field_sym), pinned by
physics: a half (quarter) mesh solved with x (xy) symmetry must equal the
full mirrored mesh solved without images, and a body solved with the rigid
ground image must equal the body plus its mirror image.

The two discretisations differ only in how touching pairs that straddle the
symmetry plane are parametrised: mirrored faces have reversed vertex order,
so their Duffy points differ.  Measured agreement is 8e-6 (x, xy) and 1.4e-7
(ground, no touching images).  Tolerances: 3e-5 / 1e-6.
"""
import numpy as np
import pytest

import oracle
from beat_engine_b200 import mesh as M

K = 30.0


def compare(half, full, mode, ncopy, tol):
    rng = np.random.default_rng(2)
    F = half.num_faces
    qh = rng.standard_normal((F, 2)) + 1j * rng.standard_normal((F, 2))
    qf = np.vstack([qh] * ncopy)
    Af, bf = oracle.assemble(full, K, 1 / K, qf)
    pf = np.linalg.solve(Af, bf)
    Ah, bh = oracle.assemble_sym(half, K, 1 / K, qh, mode)
    ph = np.linalg.solve(Ah, bh)
    V = half.num_vertices
    assert np.linalg.norm(ph - pf[:V]) <= tol * np.linalg.norm(pf[:V])
    dirs = M.fibonacci_sphere(15, 1.0)
    ffh = oracle.field_sym(half, K, dirs, ph, qh, mode, far=True)
    fff = oracle.farfield(full, K, dirs, pf, qf)
    assert np.linalg.norm(ffh - fff) <= tol * np.linalg.norm(fff)
    pts = np.array([[0.3, 0.2, 0.1], [-0.25, 0.3, -0.2], [0.1, -0.4, 0.3]])
    fh = oracle.field_sym(half, K, pts, ph, qh, mode)
    ff = oracle.field(full, K, pts, pf, qf)
    assert np.linalg.norm(fh - ff) <= tol * np.linalg.norm(ff)


def test_x_symmetry_equals_the_mirrored_mesh():
    half = M.uv_sphere_patch(0.1, 8, 8, -np.pi / 2, np.pi / 2)
    compare(half, M.mirror(half, 0), "x", 2, 3e-5)


def test_xy_symmetry_equals_the_mirrored_mesh():
    quarter = M.uv_sphere_patch(0.1, 8, 4, 0, np.pi / 2)
    compare(quarter, M.mirror(M.mirror(quarter, 0), 1), "xy", 4, 3e-5)


def test_ground_image_equals_the_mirrored_body():
    body = M.reference_sphere(0.1, 1, centre=(0.0, 0.25, 0.0))
    compare(body, M.mirror(body, 1), "ground", 2, 1e-6)


def test_off_is_the_plain_assembly_and_domain_is_checked():
    s = M.reference_sphere(0.1, 1)
    q = np.ones((s.num_faces, 1), complex)
    A0, b0 = oracle.assemble(s, K, 1 / K, q)
    A1, b1 = oracle.assemble_sym(s, K, 1 / K, q, "off")
    assert np.array_equal(A0, A1) and np.array_equal(b0, b1)
    with pytest.raises(ValueError):
        oracle.symmetry_snap(s.vertices, "x")  # the full sphere is not in x >= 0
