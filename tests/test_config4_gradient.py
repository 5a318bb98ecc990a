"""The adjoint-gradient workload at its specified size (tests/golden/config4_case.py):
a 5,228-face perturbed loudspeaker enclosure, 8 frequencies from 250 Hz to
4 kHz, a dB objective over 72 far-field directions.  Gradients with respect
to the per-face complex normal velocity, the per-face admittance and the
vertex positions come from beat_b200_adjoint_shape (one adjoint solve per
frequency on the forward solve's factors, FP64 form).

* Against the FP64 oracle (tests/golden/config4_oracle.npz): at the design
  point without admittance the GPU far fields equal the oracle's (1e-10),
  and the adjoint directional derivatives along 4 seeded (velocity, vertex)
  directions equal the oracle's central differences (h = 1e-6) within 1e-5.
* Against the GPU's own FP64 forward model: at a design point with an
  admittance, the directional derivatives along 64 seeded (velocity,
  admittance, vertex) directions equal central differences (h = 1e-6)
  within 1e-5.
"""
import math
import os
import sys

import numpy as np
import pytest

from beat_engine_b200 import _lib
from beat_engine_b200.phasor import neumann_scale

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import config4_case as case  # noqa: E402

pytestmark = pytest.mark.gpu
GOLD = os.path.join(HERE, "golden", "config4_oracle.npz")
H = 1e-6


@pytest.fixture(scope="module")
def setup():
    if not os.path.exists(GOLD):
        pytest.fail("tests/golden/config4_oracle.npz is missing: run tests/golden/make_config4_fixtures.py")
    gold = dict(np.load(GOLD))
    m = case.mesh()
    assert m.num_faces == int(gold["faces"])
    ctx = _lib.Context(0)
    ctx.set_mesh(m.vertices, m.faces, 4, 4)
    yield m, gold, ctx
    ctx.close()


def _forward(ctx, v, Y):
    """Far fields of all frequencies (FP64 form) with admittance Y (or None)."""
    dirs = case.directions()
    opts = _lib.Context.opts(_lib.FP64, flags=_lib.FLAG_RHS_CACHED)
    out = []
    for f in case.FREQS:
        k = 2 * math.pi * f / case.C0
        s = neumann_scale(case.RHO, 2 * math.pi * f)
        ctx.set_admittance(None if Y is None else s * Y)
        q0 = (s * v)[:, None]
        p, _ = ctx.solve(k, 1 / k, q0, opts)
        out.append(ctx.farfield(k, dirs, p, q0)[:, 0])
    ctx.set_admittance(None)
    return out


def _gradients(ctx, v, Y, targets):
    """(J, dJ/d conj(v), dJ/d conj(Y), dJ/dX) by the adjoint."""
    dirs = case.directions()
    w = case.weights(dirs)
    opts = _lib.Context.opts(_lib.FP64, flags=_lib.FLAG_RHS_CACHED)
    F = v.size
    gv, gY, gX, J = np.zeros(F, complex), np.zeros(F, complex), None, 0.0
    for f, t in zip(case.FREQS, targets):
        k = 2 * math.pi * f / case.C0
        s = neumann_scale(case.RHO, 2 * math.pi * f)
        ctx.set_admittance(None if Y is None else s * Y)
        q0 = (s * v)[:, None]
        p, _ = ctx.solve(k, 1 / k, q0, opts)
        pinf = ctx.farfield(k, dirs, p, q0)[:, 0]
        J += float(np.sum(w * (case.levels(pinf) - t) ** 2))
        g = case.gradient_g(pinf, t, w)[:, None]
        wq, ga, gx = ctx.adjoint_shape(k, dirs, p, q0, g, opts)
        gv += np.conj(s) * wq[:, 0]  # q0 = s v
        gY += np.conj(s) * ga  # a = s Y
        gX = gx if gX is None else gX + gx
    ctx.set_admittance(None)
    return J, gv, gY, gX


def _objective(ctx, m, X, v, Y, targets):
    ctx.set_mesh(X, m.faces, 4, 4)
    return case.objective_of_far_fields(_forward(ctx, v, Y), targets, case.weights(case.directions()))


def test_forward_and_gradient_against_oracle(setup):
    m, gold, ctx = setup
    ctx.set_mesh(m.vertices, m.faces, 4, 4)
    v = case.velocity(m)
    pinf = _forward(ctx, v, None)
    for i in range(len(case.FREQS)):
        e = np.linalg.norm(pinf[i] - gold["pinf"][i]) / np.linalg.norm(gold["pinf"][i])
        assert e <= 1e-10, (case.FREQS[i], e)
    J, gv, _, gX = _gradients(ctx, v, None, gold["targets"])
    assert J == pytest.approx(float(gold["J0"]), rel=1e-9)
    for i, (dv, dX) in enumerate(case.oracle_directions(m)):
        pred = 2 * np.real(np.vdot(gv, dv)) + float(np.sum(gX * dX))
        fd = float(gold["fd"][i])
        assert abs(pred - fd) <= 1e-5 * abs(fd), (i, pred, fd)


def test_gradient_against_gpu_central_differences(setup):
    m, gold, ctx = setup
    ctx.set_mesh(m.vertices, m.faces, 4, 4)
    v, Y = case.velocity(m), case.admittance(m)
    targets = gold["targets"]
    J0, gv, gY, gX = _gradients(ctx, v, Y, targets)
    X0 = np.asarray(m.vertices)
    worst = 0.0
    for i, (dv, dY, dX) in enumerate(case.gpu_directions(m)):
        pred = 2 * np.real(np.vdot(gv, dv)) + 2 * np.real(np.vdot(gY, dY)) + float(np.sum(gX * dX))
        jp = _objective(ctx, m, X0 + H * dX, v + H * dv, Y + H * dY, targets)
        jm = _objective(ctx, m, X0 - H * dX, v - H * dv, Y - H * dY, targets)
        fd = (jp - jm) / (2 * H)
        worst = max(worst, abs(pred - fd) / abs(fd))
        assert abs(pred - fd) <= 1e-5 * abs(fd), (i, pred, fd)
    print(f"64 directions: worst relative difference {worst:.2e}")
