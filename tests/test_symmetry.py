"""Symmetry images (x, xy, ground) through the C ABI against the oracle's
restatement of the reference's image method (bo_assemble_sym, bo_field_sym;
pinned against full mirrored meshes in tests/test_symmetry_oracle.py).

Tolerances: FP64 assembly entrywise 1e-12 of max |A|; FP64 solve, field and
far field 1e-10; mixed solve 1e-6; adjoint (FP64) 1e-9.
"""
import numpy as np
import pytest

import oracle
from oracle import adjoint as adj
from beat_engine_b200 import _lib
from beat_engine_b200 import mesh as M

pytestmark = pytest.mark.gpu
K = 30.0


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def meshes():
    return {
        "x": M.uv_sphere_patch(0.1, 10, 10, -np.pi / 2, np.pi / 2),
        "xy": M.uv_sphere_patch(0.1, 10, 5, 0, np.pi / 2),
        "ground": M.reference_sphere(0.1, 2, centre=(0.0, 0.22, 0.0)),
    }


@pytest.fixture(scope="module")
def cases():
    out = {}
    for mode, m in meshes().items():
        c = _lib.Context(0)
        c.set_mesh(m.vertices, m.faces, 4, 4)
        c.set_symmetry(mode)
        rng = np.random.default_rng(5)
        q = rng.standard_normal((m.num_faces, 3)) + 1j * rng.standard_normal((m.num_faces, 3))
        Ao, bo = oracle.assemble_sym(m, K, 1 / K, q, mode)
        out[mode] = dict(ctx=c, mesh=m, q=q, Ao=Ao, bo=bo, po=np.linalg.solve(Ao, bo))
    yield out
    for v in out.values():
        v["ctx"].close()


@pytest.mark.parametrize("mode", ["x", "xy", "ground"])
def test_assembly_matches_oracle(cases, mode):
    cs = cases[mode]
    A, b = cs["ctx"].assemble(K, 1 / K, cs["q"], precision=_lib.FP64)
    scale = np.abs(cs["Ao"]).max()
    assert np.abs(A - cs["Ao"]).max() <= 1e-12 * scale
    assert rel(b, cs["bo"]) <= 1e-12


@pytest.mark.parametrize("mode", ["x", "xy", "ground"])
def test_solve_field_and_far_field_match_oracle(cases, mode):
    cs = cases[mode]
    c, m, q = cs["ctx"], cs["mesh"], cs["q"]
    p, _ = c.solve(K, 1 / K, q, _lib.Context.opts(_lib.FP64))
    assert rel(p, cs["po"]) <= 1e-10
    dirs = M.fibonacci_sphere(17, 1.0)
    assert rel(c.farfield(K, dirs, p, q), oracle.field_sym(m, K, dirs, cs["po"], q, mode, far=True)) <= 1e-10
    pts = np.array([[0.35, 0.3, 0.1], [0.2, 0.45, -0.3], [0.4, 0.25, 0.35]])
    assert rel(c.field(K, pts, p, q), oracle.field_sym(m, K, pts, cs["po"], q, mode)) <= 1e-10
    pm, d = c.solve(K, 1 / K, q, _lib.Context.opts(_lib.MIXED_FP32_IR))
    assert d["ir_converged"] == 1 and rel(pm, cs["po"]) <= 1e-6


def test_adjoint_with_x_symmetry(cases):
    cs = cases["x"]
    c, m, q = cs["ctx"], cs["mesh"], cs["q"]
    F, N = m.num_faces, m.num_vertices
    _, B = oracle.assemble_sym(m, K, 1 / K, np.eye(F, dtype=complex), "x")
    dirs = M.fibonacci_sphere(11, 1.0)
    Fp = oracle.field_sym(m, K, dirs, np.eye(N, dtype=complex), np.zeros((F, N), complex), "x", far=True)
    Fq = oracle.field_sym(m, K, dirs, np.zeros((N, F), complex), np.eye(F, dtype=complex), "x", far=True)
    P = adj.face_average(m)
    a = np.zeros(F, complex)
    p, _ = c.solve(K, 1 / K, q, _lib.Context.opts(_lib.FP64))
    g = Fp @ p + Fq @ q - 1.0
    w, ga = c.adjoint(K, dirs, p, g, _lib.Context.opts(_lib.FP64))
    wo, gao = adj.adjoint(cs["Ao"], B, P, a, Fp, Fq, cs["po"], g)
    assert rel(w, wo) <= 1e-9 and rel(ga, gao) <= 1e-9


def test_sweep_with_symmetry_matches_single_solves(cases):
    cs = cases["xy"]
    c, q = cs["ctx"], cs["q"]
    ks = np.array([K, 45.0])
    qq = np.asfortranarray(np.stack([q, q], axis=2))
    p, _, _ = c.sweep(ks, 1 / ks, qq, _lib.Context.opts(_lib.FP64))
    for f in range(2):
        pf, _ = c.solve(ks[f], 1 / ks[f], q, _lib.Context.opts(_lib.FP64))
        assert rel(p[:, :, f], pf) <= 1e-10


def test_mode_changes_and_domain_errors():
    full = M.reference_sphere(0.1, 1)
    with _lib.Context(0) as c:
        c.set_mesh(full.vertices, full.faces, 4, 4)
        with pytest.raises(_lib.BeatB200Error) as e:
            c.set_symmetry("x")  # a full sphere is not in x >= 0
        assert e.value.status == _lib.INVALID_ARG
        q = np.ones((full.num_faces, 1), complex)
        p0, _ = c.solve(K, 1 / K, q, _lib.Context.opts(_lib.FP64))  # still the plain set-up
        c.set_symmetry("ground")
        c.set_symmetry("off")
        p1, _ = c.solve(K, 1 / K, q, _lib.Context.opts(_lib.FP64))
        assert rel(p1, p0) <= 1e-13
        with pytest.raises(_lib.BeatB200Error):
            c.set_symmetry(7)
