"""beat_b200_resolve_noalloc against beat_b200_solve, on a B200.

The no-allocation entry point serves callers that cannot let the library
allocate device memory: a caller whose device memory belongs to its own pool
(a library-side cudaMalloc would bypass that pool's accounting) or that cannot
afford cudaMalloc/cudaFree on their thread.  It re-applies the factors of the
last beat_b200_solve to right-hand sides already in device memory.

These tests call it through the C ABI, two calls in a row, and compare each
result with the corresponding columns of beat_b200_solve's own answer, within
the tolerances of the other GPU tests (1e-11 for the FP64 form; 2e-5 for the
mixed form's direct FP32-LU solution, whose right-hand side is re-assembled
with FP32 atomics in each call).  They also check the property the entry
point is named for: while it runs, every library allocation is made to fail
(BEAT_B200_FAULT_OOM_BYTES=1) and the context's device memory stays the
same.  R = 20 spans two 16-column chunks of the block substitution, which
reuse one set of block flags.  The file is collected last and needs nothing
from the other tests.
"""
import math
import os

import numpy as np
import pytest

from beat_engine_b200 import _lib
from beat_engine_b200 import mesh as M

pytestmark = pytest.mark.gpu
K = 2 * math.pi * 1500.0 / 343.0


def _q(F, R, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((F, R)) + 1j * rng.standard_normal((F, R))


class _NoAllocation:
    """Makes every library allocation fail while active (the host-side
    out-of-memory hook), and records the context's device bytes around it."""

    def __init__(self, ctx):
        self.ctx = ctx

    def __enter__(self):
        self.before = self.ctx.device_bytes()
        os.environ["BEAT_B200_FAULT_OOM_BYTES"] = "1"
        return self

    def __exit__(self, *exc):
        os.environ.pop("BEAT_B200_FAULT_OOM_BYTES", None)
        self.after = self.ctx.device_bytes()


@pytest.mark.parametrize("precision,flags,tol,R,cols_per_call",
                         [(_lib.FP64, 0, 1e-11, 2, 1), (_lib.MIXED_FP32_IR, 1, 2e-5, 2, 1),
                          (_lib.FP64, 0, 1e-11, 20, 20)])
def test_resolve_noalloc_matches_solve(precision, flags, tol, R, cols_per_call):
    torch = pytest.importorskip("torch")
    mesh = M.reference_sphere(0.1, 3)
    q = _q(mesh.num_faces, R, 77)
    with _lib.Context(0) as c:
        c.set_mesh(mesh.vertices, mesh.faces, 4, 4)
        _, b = c.assemble(K, 1.0 / K, q, precision=precision, want_matrix=False)
        p, _ = c.solve(K, 1.0 / K, q, _lib.Context.opts(precision, flags=flags))
        n = mesh.num_vertices
        dev = torch.device("cuda", 0)
        for call in range(2):  # two calls in a row
            cols = slice(0, cols_per_call) if cols_per_call == R else slice(call, call + 1)
            d_b = torch.from_numpy(np.asfortranarray(b[:, cols]).T.copy()).to(dev)  # R x N rows = N x R col-major
            d_x = torch.zeros_like(d_b)
            torch.cuda.synchronize()
            with _NoAllocation(c) as na:
                c.resolve_noalloc(cols_per_call, d_b.data_ptr(), d_x.data_ptr())
            assert na.after == na.before
            torch.cuda.synchronize()
            x = d_x.cpu().numpy().T
            err = np.linalg.norm(x - p[:, cols], axis=0) / np.linalg.norm(p[:, cols], axis=0)
            assert err.max() <= tol, (call, err)


def test_resolve_noalloc_refuses_stale_factors_and_overlap():
    torch = pytest.importorskip("torch")
    mesh = M.reference_sphere(0.1, 2)
    q = _q(mesh.num_faces, 2, 5)
    dev = torch.device("cuda", 0)
    n = mesh.num_vertices
    with _lib.Context(0) as c:
        c.set_mesh(mesh.vertices, mesh.faces, 4, 4)
        d_b = torch.ones((2, n), dtype=torch.complex128, device=dev)
        d_x = torch.zeros((2, n), dtype=torch.complex128, device=dev)
        with pytest.raises(_lib.BeatB200Error) as e:  # nothing factored yet
            c.resolve_noalloc(1, d_b.data_ptr(), d_x.data_ptr())
        assert e.value.status == _lib.STATE
        c.solve(K, 1.0 / K, q, _lib.Context.opts(_lib.FP64))
        c.resolve_noalloc(2, d_b.data_ptr(), d_x.data_ptr())
        # b and x overlapping by one column
        with pytest.raises(_lib.BeatB200Error) as e:
            c.resolve_noalloc(2, d_b.data_ptr(), d_b[1].data_ptr())
        assert e.value.status == _lib.INVALID_ARG
        # a solve that fails (out of memory on its new workspace) leaves no factors
        os.environ["BEAT_B200_FAULT_OOM_BYTES"] = "1"
        try:
            with pytest.raises(_lib.BeatB200Error):
                c.solve(K, 1.0 / K, q, _lib.Context.opts(_lib.MIXED_FP32_IR))
        finally:
            os.environ.pop("BEAT_B200_FAULT_OOM_BYTES", None)
        with pytest.raises(_lib.BeatB200Error) as e:
            c.resolve_noalloc(1, d_b.data_ptr(), d_x.data_ptr())
        assert e.value.status == _lib.STATE
        # a sweep leaves no factors the caller can name
        c.solve(K, 1.0 / K, q, _lib.Context.opts(_lib.FP64))
        ks = np.array([K, 1.3 * K])
        c.sweep(ks, 1.0 / ks, np.stack([q, q], axis=2), _lib.Context.opts(_lib.FP64))
        with pytest.raises(_lib.BeatB200Error) as e:
            c.resolve_noalloc(1, d_b.data_ptr(), d_x.data_ptr())
        assert e.value.status == _lib.STATE
