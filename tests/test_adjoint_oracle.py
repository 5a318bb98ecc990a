"""The admittance / adjoint restatement (oracle/adjoint.py) pinned by central
finite differences of its own forward model, on a small icosphere (CPU).

J = sum |p_inf - t|^2 over M directions and R columns, so
g = dJ/d conj(p_inf) = p_inf - t, and for any complex parameter z with
gradient G = dJ/d conj(z):  dJ/d Re z = 2 Re G,  dJ/d Im z = 2 Im G.
Tolerance: relative 1e-6 against step-2e-4 central differences (their
truncation error is O(h^2) of the curvature of J).
"""
import numpy as np

import oracle
from oracle import adjoint as adj
from beat_engine_b200 import mesh as M


def setup():
    mesh = M.reference_sphere(0.1, 1)
    k = 41.0
    A, B = adj.operators(mesh, k, 1.0 / k)
    P = adj.face_average(mesh)
    dirs = M.fibonacci_sphere(9, 1.0)
    Fp, Fq = adj.farfield_operators(mesh, k, dirs)
    rng = np.random.default_rng(4)
    F, R = mesh.num_faces, 2
    q0 = rng.standard_normal((F, R)) + 1j * rng.standard_normal((F, R))
    a = 0.3 * (rng.standard_normal(F) + 1j * rng.standard_normal(F))
    t = rng.standard_normal((dirs.shape[0], R)) + 1j * rng.standard_normal((dirs.shape[0], R))
    return mesh, k, A, B, P, Fp, Fq, q0, a, t, dirs


def J(A, B, P, Fp, Fq, q0, a, t):
    p, q = adj.forward(A, B, P, a, q0)
    return float(np.sum(np.abs(Fp @ p + Fq @ q - t) ** 2))


def test_forward_far_field_operators_match_oracle_far_field():
    mesh, k, A, B, P, Fp, Fq, q0, a, t, dirs = setup()
    p, q = adj.forward(A, B, P, a, q0)
    direct = oracle.farfield(mesh, k, dirs, p, q)
    assert np.linalg.norm(Fp @ p + Fq @ q - direct) <= 1e-12 * np.linalg.norm(direct)


def test_zero_admittance_is_the_plain_solve():
    mesh, k, A, B, P, Fp, Fq, q0, a, t, dirs = setup()
    p, q = adj.forward(A, B, P, np.zeros_like(a), q0)
    _, b = oracle.assemble(mesh, k, 1.0 / k, q0)
    assert np.allclose(p, oracle.lu_solve(A, b), rtol=0, atol=1e-12 * np.abs(p).max())
    assert np.array_equal(q, q0)


def test_adjoint_gradients_match_central_differences():
    mesh, k, A, B, P, Fp, Fq, q0, a, t, dirs = setup()
    p, q = adj.forward(A, B, P, a, q0)
    g = Fp @ p + Fq @ q - t
    w, ga = adj.adjoint(A, B, P, a, Fp, Fq, p, g)
    h = 2e-4
    rng = np.random.default_rng(7)
    for f, r in zip(rng.integers(0, mesh.num_faces, 6), rng.integers(0, 2, 6)):
        for unit, part in ((1.0, np.real), (1j, np.imag)):
            dq = np.zeros_like(q0)
            dq[f, r] = unit * h
            fd = (J(A, B, P, Fp, Fq, q0 + dq, a, t) - J(A, B, P, Fp, Fq, q0 - dq, a, t)) / (2 * h)
            assert abs(fd - 2 * part(w[f, r])) <= 1e-6 * max(1.0, abs(fd)), (f, r, fd, w[f, r])
    for f in rng.integers(0, mesh.num_faces, 6):
        for unit, part in ((1.0, np.real), (1j, np.imag)):
            da = np.zeros_like(a)
            da[f] = unit * h
            fd = (J(A, B, P, Fp, Fq, q0, a + da, t) - J(A, B, P, Fp, Fq, q0, a - da, t)) / (2 * h)
            assert abs(fd - 2 * part(ga[f])) <= 1e-6 * max(1.0, abs(fd)), (f, fd, ga[f])
