"""beat_b200_resolve_noalloc against beat_b200_solve, on a B200.

The no-allocation entry point serves callers that cannot let the library
allocate device memory: a caller whose device memory belongs to its own pool
(a library-side cudaMalloc would bypass that pool's accounting) or that cannot
afford cudaMalloc/cudaFree on its thread.  It re-applies the factors of the
last beat_b200_solve to right-hand sides already in device memory.  This test
calls it twice in a row through the C ABI and compares each result with the
corresponding column of beat_b200_solve's own answer, within the tolerances
of the other GPU tests (1e-11 for the FP64 form; 2e-5 for the mixed form's
direct FP32-LU solution, whose right-hand side is re-assembled with FP32
atomics in each call).  It sits in its own file, collected last, and needs
nothing from the other tests.
"""
import math

import numpy as np
import pytest

from beat_engine_b200 import _lib
from beat_engine_b200 import mesh as M

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,flags,tol", [(_lib.FP64, 0, 1e-11), (_lib.MIXED_FP32_IR, 1, 2e-5)])
def test_resolve_noalloc_matches_solve(precision, flags, tol):
    torch = pytest.importorskip("torch")
    mesh = M.reference_sphere(0.1, 3)
    k = 2 * math.pi * 1500.0 / 343.0
    rng = np.random.default_rng(77)
    q = rng.standard_normal((mesh.num_faces, 2)) + 1j * rng.standard_normal((mesh.num_faces, 2))
    with _lib.Context(0) as c:
        c.set_mesh(mesh.vertices, mesh.faces, 4, 4)
        _, b = c.assemble(k, 1.0 / k, q, precision=precision, want_matrix=False)
        p, _ = c.solve(k, 1.0 / k, q, _lib.Context.opts(precision, flags=flags))
        n = mesh.num_vertices
        dev = torch.device("cuda", 0)
        for col in range(2):  # two calls in a row, one right-hand side each
            d_b = torch.from_numpy(np.ascontiguousarray(b[:, col])).to(dev)
            d_x = torch.zeros(n, dtype=torch.complex128, device=dev)
            c.resolve_noalloc(1, d_b.data_ptr(), d_x.data_ptr())
            torch.cuda.synchronize()
            x = d_x.cpu().numpy()
            err = np.linalg.norm(x - p[:, col]) / np.linalg.norm(p[:, col])
            assert err <= tol, (col, err)
