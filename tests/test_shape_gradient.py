"""Gradient of a far-field functional with respect to the vertex positions
(beat_b200_adjoint_shape) against central differences of the oracle's own
forward model (oracle assembly and far field, oracle/adjoint.py), on a
perturbed icosphere.  No reference counterpart: the reference computes no
gradients, so this is the pin.

J = sum |p_inf - t|^2 over M directions and R columns; g = p_inf - t.
Tolerances: FP64 form, 1e-6 of the largest gradient entry against step-1e-6
central differences (their error is O(h^2) of J's curvature plus rounding of
J / h); the mixed form within 1e-5 of the FP64 form (its adjoint solve runs on
the FP32 operator).
"""
import numpy as np
import pytest

from oracle import adjoint as adj
from beat_engine_b200 import _lib
from beat_engine_b200 import mesh as M

pytestmark = pytest.mark.gpu
K = 30.0
H = 1e-6


def perturbed_sphere(seed):
    m = M.reference_sphere(0.1, 1)
    rng = np.random.default_rng(seed)
    v = np.asarray(m.vertices) * (1.0 + 0.02 * rng.standard_normal((m.num_vertices, 1)))
    return M.BoundaryMesh(v, np.asarray(m.faces), np.asarray(m.physical_tags))


def objective(mesh, q0, a, t, dirs):
    A, B = adj.operators(mesh, K, 1.0 / K)
    P = adj.face_average(mesh)
    Fp, Fq = adj.farfield_operators(mesh, K, dirs)
    p, q = adj.forward(A, B, P, a, q0)
    return float(np.sum(np.abs(Fp @ p + Fq @ q - t) ** 2))


@pytest.fixture(scope="module")
def problem():
    mesh = perturbed_sphere(1)
    rng = np.random.default_rng(2)
    F, R = mesh.num_faces, 2
    dirs = M.fibonacci_sphere(9, 1.0)
    q0 = rng.standard_normal((F, R)) + 1j * rng.standard_normal((F, R))
    a = 0.3 * (rng.standard_normal(F) + 1j * rng.standard_normal(F))
    t = rng.standard_normal((dirs.shape[0], R)) + 1j * rng.standard_normal((dirs.shape[0], R))
    return dict(mesh=mesh, q0=q0, a=a, t=t, dirs=dirs)


def device_gradient(pr, precision, with_admittance):
    m = pr["mesh"]
    with _lib.Context(0) as c:
        c.set_mesh(m.vertices, m.faces, 4, 4)
        if with_admittance:
            c.set_admittance(pr["a"])
        opts = _lib.Context.opts(precision, flags=_lib.FLAG_RHS_CACHED)
        p, _ = c.solve(K, 1.0 / K, pr["q0"], opts)
        g = c.farfield(K, pr["dirs"], p, pr["q0"]) - pr["t"]
        w, ga, gx = c.adjoint_shape(K, pr["dirs"], p, pr["q0"], g, opts)
        w1, ga1 = c.adjoint(K, pr["dirs"], p, g, opts)
    return w, ga, gx, w1, ga1


@pytest.mark.parametrize("with_admittance", [False, True])
def test_vertex_gradient_matches_central_differences(problem, with_admittance):
    pr = problem
    m = pr["mesh"]
    a = pr["a"] if with_admittance else np.zeros(m.num_faces, complex)
    w, ga, gx, w1, ga1 = device_gradient(pr, _lib.FP64, with_admittance)
    # the Neumann-data and admittance gradients are beat_b200_adjoint's
    assert np.allclose(w, w1, rtol=0, atol=1e-12 * np.abs(w1).max())
    assert np.allclose(ga, ga1, rtol=0, atol=1e-12 * np.abs(ga1).max())
    scale = np.abs(gx).max()
    rng = np.random.default_rng(5)
    v0 = np.asarray(m.vertices)
    for v, d in zip(rng.integers(0, m.num_vertices, 10), rng.integers(0, 3, 10)):
        js = []
        for sgn in (1.0, -1.0):
            vv = v0.copy()
            vv[v, d] += sgn * H
            js.append(objective(M.BoundaryMesh(vv, np.asarray(m.faces), np.asarray(m.physical_tags)), pr["q0"], a,
                                pr["t"], pr["dirs"]))
        fd = (js[0] - js[1]) / (2 * H)
        assert abs(fd - gx[v, d]) <= 1e-6 * scale, (v, d, fd, gx[v, d], scale)


def test_mixed_form_agrees_with_fp64(problem):
    pr = problem
    _, _, g64, _, _ = device_gradient(pr, _lib.FP64, False)
    _, _, g32, _, _ = device_gradient(pr, _lib.MIXED_FP32_IR, False)
    assert np.abs(g32 - g64).max() <= 1e-5 * np.abs(g64).max()


def test_symmetry_is_refused():
    m = M.uv_sphere_patch(0.1, 6, 6, -np.pi / 2, np.pi / 2)
    dirs = M.fibonacci_sphere(5, 1.0)
    q = np.ones((m.num_faces, 1), complex)
    with _lib.Context(0) as c:
        c.set_mesh(m.vertices, m.faces, 4, 4)
        c.set_symmetry("x")
        p, _ = c.solve(K, 1.0 / K, q, _lib.Context.opts(_lib.FP64, flags=_lib.FLAG_RHS_CACHED))
        with pytest.raises(_lib.BeatB200Error) as e:
            c.adjoint_shape(K, dirs, p, q, np.ones((dirs.shape[0], 1), complex))
        assert e.value.status == _lib.STATE
