"""Admittance boundary condition and adjoint gradients through the C ABI
against the numpy restatement (oracle/adjoint.py, itself pinned by central
finite differences in tests/test_adjoint_oracle.py).

Tolerances (relative L2): FP64 form 1e-9; mixed form (FP32 operator and
factors, FP64 refinement of both the solve and the adjoint solve) 2e-6.
"""
import numpy as np
import pytest

import oracle
from oracle import adjoint as adj
from beat_engine_b200 import _lib
from beat_engine_b200 import mesh as M

pytestmark = pytest.mark.gpu

K = 52.0


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def problem():
    mesh = M.reference_sphere(0.1, 2)
    A, B = adj.operators(mesh, K, 1.0 / K)
    P = adj.face_average(mesh)
    dirs = M.fibonacci_sphere(13, 1.0)
    Fp, Fq = adj.farfield_operators(mesh, K, dirs)
    rng = np.random.default_rng(11)
    F, R = mesh.num_faces, 3
    q0 = rng.standard_normal((F, R)) + 1j * rng.standard_normal((F, R))
    a = 0.4 * (rng.standard_normal(F) + 1j * rng.standard_normal(F))
    t = rng.standard_normal((dirs.shape[0], R)) + 1j * rng.standard_normal((dirs.shape[0], R))
    return dict(mesh=mesh, A=A, B=B, P=P, dirs=dirs, Fp=Fp, Fq=Fq, q0=q0, a=a, t=t)


@pytest.fixture(scope="module")
def ctx(problem):
    m = problem["mesh"]
    c = _lib.Context(0)
    c.set_mesh(m.vertices, m.faces, 4, 4)
    yield c
    c.close()


@pytest.mark.parametrize("precision,tol", [(_lib.FP64, 1e-9), (_lib.MIXED_FP32_IR, 2e-6)])
@pytest.mark.parametrize("with_admittance", [True, False])
def test_admittance_solve_far_field_and_adjoint(ctx, problem, precision, tol, with_admittance):
    pr = problem
    a = pr["a"] if with_admittance else np.zeros(pr["mesh"].num_faces, complex)
    ctx.set_admittance(pr["a"] if with_admittance else None)
    opts = _lib.Context.opts(precision)
    p, d = ctx.solve(K, 1.0 / K, pr["q0"], opts)
    po, qo = adj.forward(pr["A"], pr["B"], pr["P"], a, pr["q0"])
    assert rel(p, po) <= tol
    # the far field applies the same boundary condition
    ff = ctx.farfield(K, pr["dirs"], p, pr["q0"])
    ffo = pr["Fp"] @ po + pr["Fq"] @ qo
    assert rel(ff, ffo) <= tol
    g = ffo - pr["t"]
    w, ga = ctx.adjoint(K, pr["dirs"], p, g, opts)
    wo, gao = adj.adjoint(pr["A"], pr["B"], pr["P"], a, pr["Fp"], pr["Fq"], po, g)
    assert rel(w, wo) <= tol, rel(w, wo)
    assert rel(ga, gao) <= tol, rel(ga, gao)
    ctx.set_admittance(None)


def test_zero_admittance_reproduces_the_plain_solve(ctx, problem):
    pr = problem
    opts = _lib.Context.opts(_lib.FP64)
    ctx.set_admittance(None)
    p0, _ = ctx.solve(K, 1.0 / K, pr["q0"], opts)
    ctx.set_admittance(np.zeros(pr["mesh"].num_faces, complex))
    p1, _ = ctx.solve(K, 1.0 / K, pr["q0"], opts)
    ctx.set_admittance(None)
    assert rel(p1, p0) <= 1e-13


def test_sweep_with_admittance_matches_single_solves(ctx, problem):
    pr = problem
    ctx.set_admittance(pr["a"])
    ks = np.array([K, 30.0, 70.0])
    q = np.asfortranarray(np.stack([pr["q0"]] * 3, axis=2))
    opts = _lib.Context.opts(_lib.FP64)
    p, ff, _ = ctx.sweep(ks, 1.0 / ks, q, opts, pr["dirs"])
    for f in range(3):
        pf, _ = ctx.solve(ks[f], 1.0 / ks[f], pr["q0"], opts)
        assert rel(p[:, :, f], pf) <= 1e-10
        assert rel(ff[:, :, f], ctx.farfield(ks[f], pr["dirs"], pf, pr["q0"])) <= 1e-10
    ctx.set_admittance(None)


def test_adjoint_state_errors(problem):
    m = problem["mesh"]
    with _lib.Context(0) as c:
        c.set_mesh(m.vertices, m.faces, 4, 4)
        g = np.ones((problem["dirs"].shape[0], 1), complex)
        p = np.ones((m.num_vertices, 1), complex)
        with pytest.raises(_lib.BeatB200Error) as e:
            c.adjoint(K, problem["dirs"], p, g)
        assert e.value.status == _lib.STATE
        c.solve(K, 1.0 / K, problem["q0"][:, :1], _lib.Context.opts(_lib.FP64))
        with pytest.raises(_lib.BeatB200Error) as e:
            c.adjoint(K + 1.0, problem["dirs"], p, g)
        assert e.value.status == _lib.STATE
        with pytest.raises(ValueError):
            c.set_admittance(np.ones(3))
