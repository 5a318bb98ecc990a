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


def _symmetric_problem(mode, seed):
    """A fundamental-domain mesh of the given symmetry (x >= 0, x, y >= 0 or
    y >= 0 sphere patches), its vertices perturbed off the sphere while those
    on a symmetry plane stay on it, with seeded data."""
    patch = {"x": (-np.pi / 2, np.pi / 2, 8), "xy": (0.0, np.pi / 2, 4), "ground": (0.0, np.pi, 8)}[mode]
    m = M.uv_sphere_patch(0.1, 6, patch[2], patch[0], patch[1])
    rng = np.random.default_rng(seed)
    v = np.asarray(m.vertices) * (1.0 + 0.02 * rng.standard_normal((m.num_vertices, 1)))
    planes = {"x": (0,), "xy": (0, 1), "ground": (1,)}[mode]
    for ax in planes:
        v[np.asarray(m.vertices)[:, ax] == 0.0, ax] = 0.0
    mesh = M.BoundaryMesh(v, np.asarray(m.faces), np.asarray(m.physical_tags))
    F, R = mesh.num_faces, 2
    dirs = M.fibonacci_sphere(7, 1.0)
    q0 = rng.standard_normal((F, R)) + 1j * rng.standard_normal((F, R))
    a = 0.3 * (rng.standard_normal(F) + 1j * rng.standard_normal(F))
    t = rng.standard_normal((dirs.shape[0], R)) + 1j * rng.standard_normal((dirs.shape[0], R))
    return mesh, planes, q0, a, t, dirs


def _gpu_objective(c, verts, faces, q0, a, t, dirs, with_admittance):
    c.set_mesh(verts, faces, 4, 4)  # the context's symmetry mode applies
    if with_admittance:
        c.set_admittance(a)
    p, _ = c.solve(K, 1.0 / K, q0, _lib.Context.opts(_lib.FP64, flags=_lib.FLAG_RHS_CACHED))
    return float(np.sum(np.abs(c.farfield(K, dirs, p, q0) - t) ** 2))


@pytest.mark.parametrize("mode,with_admittance", [("x", False), ("x", True), ("xy", False), ("ground", False)])
def test_symmetry_images_gradient_matches_central_differences(mode, with_admittance):
    """With symmetry images the vertex gradient and the Neumann-data gradient
    match central differences (h = 1e-6) of the FP64 forward model with the
    same images (the GPU's, whose images are pinned to mirrored full meshes
    and to the oracle by the symmetry tests), within 1e-6 of the largest
    entry.  In the x and xy modes a vertex on a symmetry plane stays on it, so
    its gradient's component normal to the plane is zero.  The ground mode has
    no such constraint (as in the reference, its plane has no orbit weights);
    there the hemisphere rests on the plane, so its touching image pairs are
    exercised, and moving a vertex off the plane would end that contact, so
    the differences move plane vertices within the plane only."""
    mesh, planes, q0, a, t, dirs = _symmetric_problem(mode, 11)
    faces = np.asarray(mesh.faces)
    v0 = np.asarray(mesh.vertices)
    with _lib.Context(0) as c:
        c.set_mesh(v0, faces, 4, 4)
        c.set_symmetry(mode)
        if with_admittance:
            c.set_admittance(a)
        opts = _lib.Context.opts(_lib.FP64, flags=_lib.FLAG_RHS_CACHED)
        p, _ = c.solve(K, 1.0 / K, q0, opts)
        g = c.farfield(K, dirs, p, q0) - t
        w, _, gx = c.adjoint_shape(K, dirs, p, q0, g, opts)
        on_plane = np.zeros(v0.shape, dtype=bool)
        for ax in planes:
            on_plane[v0[:, ax] == 0.0, ax] = True
        assert on_plane.any()
        if mode != "ground":
            assert np.all(gx[on_plane] == 0.0)
        scale = np.abs(gx).max()
        rng = np.random.default_rng(5)
        free = np.argwhere(~on_plane)
        # plane vertices (in-plane components) and others
        plane_rows = np.argwhere(on_plane.any(axis=1)[:, None] & ~on_plane)
        picks = [tuple(free[i]) for i in rng.choice(len(free), 8, replace=False)]
        picks += [tuple(plane_rows[i]) for i in rng.choice(len(plane_rows), 4, replace=False)]
        for v, d in picks:
            js = []
            for sgn in (1.0, -1.0):
                vv = v0.copy()
                vv[v, d] += sgn * H
                js.append(_gpu_objective(c, vv, faces, q0, a, t, dirs, with_admittance))
            fd = (js[0] - js[1]) / (2 * H)
            assert abs(fd - gx[v, d]) <= 1e-6 * scale, (mode, v, d, fd, gx[v, d], scale)
        # the Neumann-data gradient: dJ = 2 Re sum conj(w) dq0 along a seeded
        # direction; J is quadratic in q0, so a central difference is exact at
        # any step, and a step of 1e-3 keeps J's rounding out of it
        dq = rng.standard_normal(q0.shape) + 1j * rng.standard_normal(q0.shape)
        hq = 1e-3
        jp = _gpu_objective(c, v0, faces, q0 + hq * dq, a, t, dirs, with_admittance)
        jm = _gpu_objective(c, v0, faces, q0 - hq * dq, a, t, dirs, with_admittance)
        fdq = (jp - jm) / (2 * hq)
        dj = 2.0 * np.real(np.sum(np.conj(w) * dq))
        assert abs(fdq - dj) <= 1e-6 * abs(dj), (mode, fdq, dj)


@pytest.mark.parametrize("mode", ["x", "xy"])
def test_symmetry_images_mixed_form_agrees_with_fp64(mode):
    """With symmetry images, the mixed form's gradients (adjoint solve on the
    FP32 factors with FP64 refinement) agree with the FP64 form's within
    1e-5 of the largest entry."""
    mesh, _, q0, _, t, dirs = _symmetric_problem(mode, 12)
    out = {}
    for precision in (_lib.FP64, _lib.MIXED_FP32_IR):
        with _lib.Context(0) as c:
            c.set_mesh(mesh.vertices, mesh.faces, 4, 4)
            c.set_symmetry(mode)
            opts = _lib.Context.opts(precision, flags=_lib.FLAG_RHS_CACHED)
            p, _ = c.solve(K, 1.0 / K, q0, opts)
            g = c.farfield(K, dirs, p, q0) - t
            out[precision] = c.adjoint_shape(K, dirs, p, q0, g, opts)
    (w64, _, gx64), (w32, _, gx32) = out[_lib.FP64], out[_lib.MIXED_FP32_IR]
    assert np.abs(gx32 - gx64).max() <= 1e-5 * np.abs(gx64).max()
    assert np.abs(w32 - w64).max() <= 1e-5 * np.abs(w64).max()
