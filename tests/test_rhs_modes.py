"""Right-hand-side modes on the GPU: the matrix-free path (B-tile x q inside
the element-pair kernels, no N x F array) against the cached mapping
(b = B q), as the reference's CUDA tests compare its two column modes
(runtests.jl:1817-1839, agreement 2e-5 in FP32).

Tolerances (relative L2): FP64 form 1e-12 (both modes are FP64 throughout;
only the summation order differs); mixed form 1e-6 between the modes (b is
summed from FP32 element-pair blocks either way, in a different order).
"""
import numpy as np
import pytest

import oracle
from beat_engine_b200 import _lib
from beat_engine_b200 import mesh as M

pytestmark = pytest.mark.gpu
K = 40.0
MF, CA = _lib.FLAG_RHS_MATRIX_FREE, _lib.FLAG_RHS_CACHED


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def neumann(m, R, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((m.num_faces, R)) + 1j * rng.standard_normal((m.num_faces, R))


@pytest.fixture(scope="module")
def sphere():
    m = M.reference_sphere(0.1, 3)
    c = _lib.Context(0)
    c.set_mesh(m.vertices, m.faces, 4, 4)
    yield m, c
    c.close()


@pytest.mark.parametrize("precision,tol", [(_lib.FP64, 1e-12), (_lib.MIXED_FP32_IR, 1e-6)])
@pytest.mark.parametrize("R", [1, 3, 17])
def test_matrix_free_matches_cached(sphere, precision, tol, R):
    m, c = sphere
    q = neumann(m, R, R)
    pc, dc = c.solve(K, 1 / K, q, _lib.Context.opts(precision, flags=CA))
    pm, dm = c.solve(K, 1 / K, q, _lib.Context.opts(precision, flags=MF))
    assert dc["rhs_mode"] == _lib.RHS_CACHED and dm["rhs_mode"] == _lib.RHS_MATRIX_FREE
    assert rel(pm, pc) <= tol
    if precision == _lib.MIXED_FP32_IR:
        assert dm["ir_converged"] == 1


def test_matrix_free_matches_the_oracle(sphere):
    m, c = sphere
    q = neumann(m, 5, 9)
    A, b = oracle.assemble(m, K, 1 / K, q)
    p, _ = c.solve(K, 1 / K, q, _lib.Context.opts(_lib.FP64, flags=MF))
    assert rel(p, np.linalg.solve(A, b)) <= 1e-10


def test_auto_follows_the_policy_and_frees_the_mapping(sphere):
    m, c = sphere
    _, d1 = c.solve(K, 1 / K, neumann(m, 1, 1), _lib.Context.opts(_lib.FP64))
    assert d1["rhs_mode"] == _lib.RHS_MATRIX_FREE  # one excitation: nothing to save
    held_mf = c.device_bytes()
    _, d2 = c.solve(K, 1 / K, neumann(m, 2, 2), _lib.Context.opts(_lib.FP64))
    assert d2["rhs_mode"] == _lib.RHS_CACHED
    held_ca = c.device_bytes()
    assert held_ca - held_mf >= m.num_vertices * m.num_faces * 16  # B is resident
    _, d3 = c.solve(K, 1 / K, neumann(m, 2, 2), _lib.Context.opts(_lib.FP64, flags=MF))
    assert d3["rhs_mode"] == _lib.RHS_MATRIX_FREE
    assert c.device_bytes() <= held_ca - m.num_vertices * m.num_faces * 16
    with pytest.raises(_lib.BeatB200Error) as e:
        c.solve(K, 1 / K, neumann(m, 2, 2), _lib.Context.opts(_lib.FP64, flags=MF | CA))
    assert e.value.status == _lib.INVALID_ARG


@pytest.mark.parametrize("precision,tol", [(_lib.FP64, 1e-12), (_lib.MIXED_FP32_IR, 1e-6)])
def test_symmetry_images_in_both_modes(precision, tol):
    m = M.uv_sphere_patch(0.1, 10, 5, 0, np.pi / 2)
    q = neumann(m, 4, 3)
    with _lib.Context(0) as c:
        c.set_mesh(m.vertices, m.faces, 4, 4)
        c.set_symmetry("xy")
        pc, _ = c.solve(K, 1 / K, q, _lib.Context.opts(precision, flags=CA))
        pm, dm = c.solve(K, 1 / K, q, _lib.Context.opts(precision, flags=MF))
    assert dm["rhs_mode"] == _lib.RHS_MATRIX_FREE
    assert rel(pm, pc) <= tol
    if precision == _lib.FP64:
        Ao, bo = oracle.assemble_sym(m, K, 1 / K, q, "xy")
        assert rel(pm, np.linalg.solve(Ao, bo)) <= 1e-10


def test_sweep_matrix_free_matches_single_solves(sphere):
    m, c = sphere
    ks = np.array([K, 25.0, 55.0])
    q = np.asfortranarray(np.stack([neumann(m, 3, 20 + f) for f in range(3)], axis=2))
    opts = _lib.Context.opts(_lib.FP64, flags=MF)
    p, _, diags = c.sweep(ks, 1 / ks, q, opts)
    for f in range(3):
        assert diags[f]["rhs_mode"] == _lib.RHS_MATRIX_FREE
        pf, _ = c.solve(ks[f], 1 / ks[f], q[:, :, f], _lib.Context.opts(_lib.FP64, flags=CA))
        assert rel(p[:, :, f], pf) <= 1e-12


def test_admittance_needs_the_mapping_and_the_adjoint_needs_it_resident():
    m = M.reference_sphere(0.1, 2)
    q = neumann(m, 1, 5)
    rng = np.random.default_rng(6)
    a = 0.3 * (rng.standard_normal(m.num_faces) + 1j * rng.standard_normal(m.num_faces))
    dirs = M.fibonacci_sphere(7, 1.0)
    with _lib.Context(0) as c:
        c.set_mesh(m.vertices, m.faces, 4, 4)
        # matrix-free solve, then an adjoint: B is not resident
        p, d = c.solve(K, 1 / K, q, _lib.Context.opts(_lib.FP64))
        assert d["rhs_mode"] == _lib.RHS_MATRIX_FREE
        g = np.ones((dirs.shape[0], 1), complex)
        with pytest.raises(_lib.BeatB200Error) as e:
            c.adjoint(K, dirs, p, g)
        assert e.value.status == _lib.STATE
        # after a cached solve the adjoint runs
        p, d = c.solve(K, 1 / K, q, _lib.Context.opts(_lib.FP64, flags=CA))
        w, ga = c.adjoint(K, dirs, p, g)
        assert np.all(np.isfinite(w)) and np.all(np.isfinite(ga))
        # an admittance makes auto take the mapping even for one excitation ...
        c.set_admittance(a)
        _, d = c.solve(K, 1 / K, q, _lib.Context.opts(_lib.FP64))
        assert d["rhs_mode"] == _lib.RHS_CACHED
        # ... and refuses the matrix-free mode
        with pytest.raises(_lib.BeatB200Error) as e:
            c.solve(K, 1 / K, q, _lib.Context.opts(_lib.FP64, flags=MF))
        assert e.value.status == _lib.INVALID_ARG
        c.set_admittance(None)
