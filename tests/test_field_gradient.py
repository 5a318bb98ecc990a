"""Pressure and gradient at observation points (beat_b200_field_gradient)
through the C ABI against the oracle's restatement of the reference's
pressure_gradient_v1 (oracle.field_gradient; pinned in
tests/test_field_gradient_oracle.py).

Both sides are FP64; the subdivision on the device tracks pieces in face
coordinates rather than by midpoint averaging in space, which moves results
by rounding only.  Tolerance: 1e-10 of the largest entry of each column.
"""
import numpy as np
import pytest

import oracle
from beat_engine_b200 import _lib
from beat_engine_b200 import mesh as M

pytestmark = pytest.mark.gpu
K = 30.0


def close(a, b, tol=1e-10):
    scale = np.abs(b).max(axis=0, keepdims=True)
    return np.all(np.abs(a - b) <= tol * scale)


def random_data(m, R, seed):
    rng = np.random.default_rng(seed)
    p = rng.standard_normal((m.num_vertices, R)) + 1j * rng.standard_normal((m.num_vertices, R))
    q = rng.standard_normal((m.num_faces, R)) + 1j * rng.standard_normal((m.num_faces, R))
    return p, q


def points_around(radius, n, seed):
    """Points from 1.002 to 3 radii out, many of them near the surface."""
    rng = np.random.default_rng(seed)
    d = rng.standard_normal((n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    r = radius * np.concatenate([1.002 + 0.05 * rng.random(n // 2), 1.0 + 2.0 * rng.random(n - n // 2)])
    return d * r[:, None]


@pytest.fixture(scope="module")
def sphere():
    m = M.reference_sphere(0.1, 2)
    c = _lib.Context(0)
    c.set_mesh(m.vertices, m.faces, 4, 4)
    yield m, c
    c.close()


@pytest.mark.parametrize("R", [1, 5])
def test_gradient_matches_oracle(sphere, R):
    m, c = sphere
    p, q = random_data(m, R, 10 + R)
    pts = points_around(0.1, 40, R)
    g = c.field_gradient(K, pts, p, q)
    go = oracle.field_gradient(m, K, pts, p, q)
    assert g.shape == (40, 4, R)
    for r in range(R):
        assert close(g[:, :, r], go[:, :, r])


def test_value_column_matches_the_field_entry(sphere):
    m, c = sphere
    p, q = random_data(m, 3, 7)
    pts = points_around(0.1, 24, 9) * 2.0  # all beyond three face diameters
    g = c.field_gradient(K, pts, p, q)
    assert close(g[:, 0, :], c.field(K, pts, p, q), 1e-12)


def test_negative_wavenumber_and_admittance(sphere):
    m, c = sphere
    p, q = random_data(m, 2, 4)
    pts = points_around(0.1, 16, 5)
    assert close(c.field_gradient(-K, pts, p, q), oracle.field_gradient(m, -K, pts, p, q))
    # with an admittance the Neumann data are q - a (P p), as in the field
    rng = np.random.default_rng(6)
    a = 0.3 * (rng.standard_normal(m.num_faces) + 1j * rng.standard_normal(m.num_faces))
    pface = p[np.asarray(m.faces)].mean(axis=1)
    c.set_admittance(a)
    try:
        g = c.field_gradient(K, pts, p, q)
    finally:
        c.set_admittance(None)
    assert close(g, oracle.field_gradient(m, K, pts, p, q - a[:, None] * pface))


@pytest.mark.parametrize("mode,mesh", [
    ("x", lambda: M.uv_sphere_patch(0.1, 8, 8, -np.pi / 2, np.pi / 2)),
    ("xy", lambda: M.uv_sphere_patch(0.1, 8, 4, 0, np.pi / 2)),
    ("ground", lambda: M.reference_sphere(0.1, 2, centre=(0.0, 0.15, 0.0))),
])
def test_gradient_with_symmetry_matches_oracle(mode, mesh):
    m = mesh()
    p, q = random_data(m, 2, 8)
    # around the whole (mirrored) body: near the mesh and near its images; above
    # the ground plane for "ground", where the lowest points are still within
    # three face diameters of the image sphere
    pts = points_around(0.1, 30, 3)
    if mode == "ground":
        pts = pts + np.array([0.0, 0.15, 0.0])
        pts[:, 1] = np.abs(pts[:, 1])
    with _lib.Context(0) as c:
        c.set_mesh(m.vertices, m.faces, 4, 4)
        c.set_symmetry(mode)
        g = c.field_gradient(K, pts, p, q)
    go = oracle.field_gradient(m, K, pts, p, q, mode=mode)
    for r in range(2):
        assert close(g[:, :, r], go[:, :, r])


def test_point_on_the_boundary_is_an_error_and_the_context_survives(sphere):
    m, c = sphere
    p, q = random_data(m, 1, 2)
    with pytest.raises(_lib.BeatB200Error) as e:
        c.field_gradient(K, m.vertices[:1], p, q)
    assert e.value.status == _lib.INVALID_ARG
    assert "too close" in str(e.value)
    pts = points_around(0.1, 8, 1)
    assert close(c.field_gradient(K, pts, p, q), oracle.field_gradient(m, K, pts, p, q))


def test_empty_point_set(sphere):
    m, c = sphere
    p, q = random_data(m, 2, 3)
    assert c.field_gradient(K, np.zeros((0, 3)), p, q).shape == (0, 4, 2)
