"""The LU's grid-wide panel kernel, on a B200.

A sub-panel is factored by one 16-CTA thread-block cluster while its rows fit
the cluster's shared memory: about 721 rows of 32 complex columns per CTA, so
N - k <= ~11,540 rows.  Past that, the first sub-panels of a larger system go
to the cooperative grid-wide panel kernel instead.  Smaller test systems never
reach it.

Here a closed rounded-box enclosure of 28,060 faces (N = 14,032) takes that
path in both forms.  The FP32 tensor-core LU with FP64 refinement and the FP64
LU are independent factorisations, so their agreement checks both:

* per column, the relative L2 difference is <= 1e-6 (the mixed form's target
  against FP64);
* the refinement converges to its 1e-10 residual.

A dense FP64 CPU solve of this size would take minutes, so the FP64 form is
the reference here.
"""
import math

import numpy as np
import pytest

from beat_engine_b200 import _lib
from beat_engine_b200 import mesh as M

pytestmark = pytest.mark.gpu


def col_rel(a, b):
    return np.linalg.norm(a - b, axis=0) / np.linalg.norm(b, axis=0)


def test_both_forms_agree_past_the_cluster_rows():
    mesh = M.rounded_box_enclosure(28000, seed=3)
    assert mesh.num_vertices > 13000  # the first sub-panels exceed one cluster's rows
    k = 2 * math.pi * 500.0 / 343.0
    rng = np.random.default_rng(21)
    q = rng.standard_normal((mesh.num_faces, 2)) + 1j * rng.standard_normal((mesh.num_faces, 2))
    with _lib.Context(0) as c:
        c.set_mesh(mesh.vertices, mesh.faces, 4, 4)
        p64, d64 = c.solve(k, 1.0 / k, q, _lib.Context.opts(_lib.FP64))
        pmx, dmx = c.solve(k, 1.0 / k, q, _lib.Context.opts(_lib.MIXED_FP32_IR))
    assert d64["precision"] == _lib.FP64 and np.all(np.isfinite(p64))
    assert dmx["ir_converged"] == 1 and dmx["ir_residual"] <= 1e-10
    err = col_rel(pmx, p64)
    assert np.all(err <= 1e-6), err
