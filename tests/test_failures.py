"""Failure paths, provoked on the host (no GPU fault, trap or hang):

* refinement that misses its tolerance (a one-iteration budget at an
  unreachable 1e-15) falls back to the FP64 form and reports it, or returns
  BEAT_B200_NOT_CONVERGED with BEAT_B200_FLAG_NO_FALLBACK;
* out-of-memory injected with BEAT_B200_FAULT_OOM_BYTES: the right-hand-side
  mapping falls back to the matrix-free mode, an admittance (which needs the
  mapping) and the system matrix itself report BEAT_B200_OOM, and the context
  solves normally once the hook is cleared.
"""
import os

import numpy as np
import pytest

import oracle
from beat_engine_b200 import _lib
from beat_engine_b200 import mesh as M

pytestmark = pytest.mark.gpu
K = 30.0


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def problem():
    m = M.reference_sphere(0.1, 2)
    rng = np.random.default_rng(3)
    q = rng.standard_normal((m.num_faces, 2)) + 1j * rng.standard_normal((m.num_faces, 2))
    A, b = oracle.assemble(m, K, 1 / K, q)
    return m, q, np.linalg.solve(A, b)


def test_refinement_failure_falls_back_to_fp64(problem):
    m, q, po = problem
    with _lib.Context(0) as c:
        c.set_mesh(m.vertices, m.faces, 4, 4)
        hopeless = dict(ir_max_iters=1, ir_restart=1, ir_rtol=1e-15)
        p, d = c.solve(K, 1 / K, q, _lib.Context.opts(_lib.MIXED_FP32_IR, **hopeless))
        assert d["precision"] == _lib.FP64 and d["ir_converged"] == 0 and d["ir_iterations"] >= 1
        assert rel(p, po) <= 1e-10
        with pytest.raises(_lib.BeatB200Error) as e:
            c.solve(K, 1 / K, q, _lib.Context.opts(_lib.MIXED_FP32_IR, flags=_lib.FLAG_NO_FALLBACK, **hopeless))
        assert e.value.status == _lib.NOT_CONVERGED
        p, d = c.solve(K, 1 / K, q, _lib.Context.opts(_lib.MIXED_FP32_IR))  # the context carries on
        assert d["precision"] == _lib.MIXED_FP32_IR and d["ir_converged"] == 1 and rel(p, po) <= 1e-6


@pytest.fixture
def oom_hook():
    def set_limit(nbytes):
        os.environ["BEAT_B200_FAULT_OOM_BYTES"] = str(int(nbytes))
    yield set_limit
    os.environ.pop("BEAT_B200_FAULT_OOM_BYTES", None)


def test_injected_oom_paths(oom_hook):
    # large enough that A and the N x F mapping are the two largest buffers
    m = M.reference_sphere(0.1, 3)
    rng = np.random.default_rng(4)
    q = rng.standard_normal((m.num_faces, 2)) + 1j * rng.standard_normal((m.num_faces, 2))
    A, b = oracle.assemble(m, K, 1 / K, q)
    po = np.linalg.solve(A, b)
    N, F = m.num_vertices, m.num_faces
    ld = (N + 127) // 128 * 128
    a_bytes, b_bytes = N * ld * 16, N * F * 16  # FP64 form: A and the N x F mapping
    inverse_blocks = 6 * ((N + 63) // 64) * 64 * 64 * 16  # the triangular solves' block inverses
    assert inverse_blocks < a_bytes < b_bytes
    with _lib.Context(0) as c:
        c.set_mesh(m.vertices, m.faces, 4, 4)
        opts = _lib.Context.opts(_lib.FP64)
        # the mapping cannot be allocated: matrix-free right-hand sides instead
        oom_hook(b_bytes)
        p, d = c.solve(K, 1 / K, q, opts)
        assert d["rhs_mode"] == _lib.RHS_MATRIX_FREE and rel(p, po) <= 1e-10
        # an admittance needs the mapping: out of memory
        c.set_admittance(np.full(F, 0.1 + 0.05j))
        with pytest.raises(_lib.BeatB200Error) as e:
            c.solve(K, 1 / K, q, opts)
        assert e.value.status == _lib.OOM and "BEAT_B200_FAULT_OOM_BYTES" in str(e.value)
        c.set_admittance(None)
        # the system matrix itself
        c.release_workspace()
        oom_hook(a_bytes)
        with pytest.raises(_lib.BeatB200Error) as e:
            c.solve(K, 1 / K, q, opts)
        assert e.value.status == _lib.OOM
        # hook cleared: the cached mapping again, same answer
        os.environ.pop("BEAT_B200_FAULT_OOM_BYTES")
        p, d = c.solve(K, 1 / K, q, opts)
        assert d["rhs_mode"] == _lib.RHS_CACHED and rel(p, po) <= 1e-10
