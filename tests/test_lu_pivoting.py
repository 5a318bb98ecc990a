"""The mixed form's two pivoting rules for its FP32 LU (the preconditioner of
the FP64 refinement): tournament pivoting (default: each 32-column
sub-panel's pivots chosen among every CTA's local pivot rows) and partial
pivoting as LAPACK does (BEAT_B200_FLAG_PARTIAL_PIVOT).  Both must give the
FP64 oracle's solution within 1e-6 per column with the refinement converged
in at most two iterations, for every panel width, on a mesh whose LU runs on
the cluster panels (F = 5,120, N = 2,562) and on an enclosure whose last
sub-panel is partial (F = 1,184, N = 594 = 18 x 32 + 18)."""
import math

import numpy as np
import pytest

import oracle
from beat_engine_b200 import _lib
from beat_engine_b200 import mesh as M

pytestmark = pytest.mark.gpu


def col_rel(a, b):
    return np.linalg.norm(a - b, axis=0) / np.linalg.norm(b, axis=0)


@pytest.fixture(scope="module", params=[("sphere4", None), ("enclosure", 1200)])
def case(request):
    name, target = request.param
    m = M.reference_sphere(0.1, 4) if name == "sphere4" else M.rounded_box_enclosure(target, seed=5)
    k = 2 * math.pi * 3000.0 / 343.0
    rng = np.random.default_rng(9)
    q = rng.standard_normal((m.num_faces, 3)) + 1j * rng.standard_normal((m.num_faces, 3))
    A, b = oracle.assemble(m, k, 1 / k, q)
    po = np.linalg.solve(A, b)
    ctx = _lib.Context(0)
    ctx.set_mesh(m.vertices, m.faces, 4, 4)
    yield m, k, q, po, ctx
    ctx.close()


@pytest.mark.parametrize("lu_block", [32, 64, 128, 256])
@pytest.mark.parametrize("flags", [0, _lib.FLAG_PARTIAL_PIVOT])
def test_mixed_lu_pivoting_rules(case, lu_block, flags):
    m, k, q, po, ctx = case
    p, d = ctx.solve(k, 1 / k, q, _lib.Context.opts(_lib.MIXED_FP32_IR, lu_block=lu_block, flags=flags))
    assert d["precision"] == _lib.MIXED_FP32_IR and d["ir_converged"] == 1
    assert d["ir_iterations"] <= 2
    assert col_rel(p, po).max() <= 1e-6


def test_tournament_factors_precondition_alone(case):
    """Without refinement the tournament-pivoted FP32 factors alone solve the
    system to FP32-LU accuracy (as partial pivoting does)."""
    m, k, q, po, ctx = case
    errs = []
    for flags in (_lib.FLAG_NO_REFINE, _lib.FLAG_NO_REFINE | _lib.FLAG_PARTIAL_PIVOT):
        p, _ = ctx.solve(k, 1 / k, q, _lib.Context.opts(_lib.MIXED_FP32_IR, flags=flags))
        errs.append(col_rel(p, po).max())
    assert errs[0] <= 1e-4 and errs[1] <= 1e-4
    assert errs[0] <= 5 * errs[1] + 1e-6, errs
