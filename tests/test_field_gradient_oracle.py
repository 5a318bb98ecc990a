"""The pressure-gradient restatement (oracle.field_gradient, after
BeatEngineFieldGradient.jl:1-88) pinned on the CPU:

* away from the boundary its value column is the oracle's pressure field
  (bo_field_sym, itself pinned against the reference's field formula);
* its gradient columns are the derivatives of its value column (central
  differences, near the boundary too, where the adaptive correction acts);
* with the exact boundary data of a point source inside a sphere, the
  corrected value and gradient near the surface keep the mesh's own error,
  which the plain quadrature sum does not;
* x symmetry on a half sphere equals the full mirrored sphere.
"""
import numpy as np
import pytest

import oracle
from beat_engine_b200 import mesh as M

K = 30.0


def random_data(m, R, seed):
    rng = np.random.default_rng(seed)
    p = rng.standard_normal((m.num_vertices, R)) + 1j * rng.standard_normal((m.num_vertices, R))
    q = rng.standard_normal((m.num_faces, R)) + 1j * rng.standard_normal((m.num_faces, R))
    return p, q


def test_value_column_is_the_pressure_field_away_from_the_boundary():
    m = M.reference_sphere(0.1, 2)
    p, q = random_data(m, 2, 1)
    pts = np.array([[0.3, 0.1, -0.2], [0.0, 0.25, 0.1], [-0.4, -0.3, 0.5]])
    g = oracle.field_gradient(m, K, pts, p, q)
    v = oracle.field_sym(m, K, pts, p, q, "off")
    assert np.abs(g[:, 0, :] - v).max() <= 1e-13 * np.abs(v).max()


@pytest.mark.parametrize("x,h,tol", [((0.3, 0.1, -0.2), 1e-5, 1e-7), ((0.104, 0.0, 0.0), 1e-6, 1e-6),
                                     ((0.0, 0.02, 0.1003), 1e-7, 1e-5)])
def test_gradient_is_the_derivative_of_the_value(x, h, tol):
    m = M.reference_sphere(0.1, 2)
    p, q = random_data(m, 1, 2)
    x = np.asarray(x)
    g = oracle.field_gradient(m, K, x[None], p, q)[0, :, 0]
    for d in range(3):
        e = np.zeros(3)
        e[d] = h
        fd = (oracle.field_gradient(m, K, (x + e)[None], p, q)[0, 0, 0]
              - oracle.field_gradient(m, K, (x - e)[None], p, q)[0, 0, 0]) / (2 * h)
        assert abs(fd - g[1 + d]) <= tol * np.abs(g[1:]).max(), (d, fd, g[1 + d])


def monopole_data(m, k):
    v = m.vertices
    r = np.linalg.norm(v, axis=1)
    p = np.exp(1j * k * r) / (4 * np.pi * r)
    tri = v[m.faces]
    c = tri.mean(axis=1)
    rc = np.linalg.norm(c, axis=1)
    n = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    n /= np.linalg.norm(n, axis=1)[:, None]
    q = (1j * k - 1 / rc) * np.exp(1j * k * rc) / (4 * np.pi * rc) * np.einsum("ij,ij->i", c, n) / rc
    return p, q


def test_near_boundary_correction_keeps_the_mesh_error():
    m = M.reference_sphere(0.1, 3)
    p, q = monopole_data(m, K)
    far_err = None
    for dist in (0.2, 0.105, 0.1005):
        x = np.array([dist, 0.013, 0.007])
        g = oracle.field_gradient(m, K, x[None], p, q)[0, :, 0]
        plain = oracle.field_sym(m, K, x[None], p, q, "off")[0, 0]
        rr = np.linalg.norm(x)
        pe = np.exp(1j * K * rr) / (4 * np.pi * rr)
        ge = pe * (1j * K - 1 / rr) * x / rr
        err_v = abs(g[0] - pe) / abs(pe)
        err_g = np.linalg.norm(g[1:] - ge) / np.linalg.norm(ge)
        if far_err is None:
            far_err = err_v
        # the gradient also carries the piecewise-constant Neumann data's O(h) error
        assert err_v <= 1.5 * far_err and err_g <= 3.0 * far_err, (dist, err_v, err_g, far_err)
        if dist < 0.101:  # the plain sum is three times worse there
            assert abs(plain - pe) / abs(pe) >= 3 * err_v


def test_x_symmetry_equals_the_mirrored_mesh():
    half = M.uv_sphere_patch(0.1, 8, 8, -np.pi / 2, np.pi / 2)
    full = M.mirror(half, 0)
    p, q = random_data(half, 1, 3)
    # mirrored copies keep vertex and face order; vertices on the plane are shared
    on = np.abs(np.asarray(half.vertices)[:, 0]) <= 1e-12
    pf = np.concatenate([p, p[~on]])
    qf = np.concatenate([q, q])
    assert pf.shape[0] == full.num_vertices and qf.shape[0] == full.num_faces
    pts = np.array([[0.03, 0.05, 0.104], [0.3, -0.1, 0.2], [0.001, 0.101, 0.0]])
    gs = oracle.field_gradient(half, K, pts, p, q, mode="x")
    gf = oracle.field_gradient(full, K, pts, pf, qf)
    assert np.abs(gs - gf).max() <= 1e-10 * np.abs(gf).max()


def test_point_on_the_boundary_is_an_error():
    m = M.reference_sphere(0.1, 1)
    p, q = random_data(m, 1, 4)
    with pytest.raises(RuntimeError, match="too close"):
        oracle.field_gradient(m, K, m.vertices[:1], p, q)
