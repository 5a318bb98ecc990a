"""The torch.autograd.Function over the adjoint (beat_engine_b200.autodiff),
the Python counterpart of the ChainRulesCore.rrule a Julia caller puts over
the same C entry points.

J = sum_r sum_d w_d |p_inf(d, r)|^2 on a perturbed icosphere (F = 320) with an
admittance, FP64 form.  torch's gradients with respect to the Neumann data,
the admittance and the vertices must match central differences (h = 1e-6
relative) of the GPU forward solve along seeded random directions within
1e-6 of the directional derivative; the mixed form's gradients match the
FP64 form's within 1e-5.  A second forward call between forward and backward
(which replaces the context's factors) must not change the gradient.
"""
import math

import numpy as np
import pytest

from beat_engine_b200 import _lib
from beat_engine_b200 import mesh as M

pytestmark = pytest.mark.gpu
K = 2 * math.pi * 1200.0 / 343.0


@pytest.fixture(scope="module")
def case():
    base = M.reference_sphere(0.1, 2)
    rng = np.random.default_rng(41)
    X = np.asarray(base.vertices) * (1 + 0.02 * rng.standard_normal(base.num_vertices))[:, None]
    F = base.num_faces
    q = rng.standard_normal((F, 2)) + 1j * rng.standard_normal((F, 2))
    a = 0.05 * (rng.standard_normal(F) + 1j * rng.standard_normal(F))
    dirs = M.equator_meridian_directions(24, 13)
    w = 1.0 + np.abs(dirs[:, 2])
    return dict(faces=np.asarray(base.faces), X=X, q=q, a=a, dirs=dirs, w=w)


def _loss(torch, pinf, w):
    return (torch.from_numpy(w)[:, None] * pinf.abs() ** 2).sum()


def _grads(torch, c, cs, precision, perturb_between=False):
    from beat_engine_b200.autodiff import farfield_solve
    q = torch.tensor(cs["q"], requires_grad=True)
    a = torch.tensor(cs["a"], requires_grad=True)
    X = torch.tensor(cs["X"], requires_grad=True)
    pinf = farfield_solve(c, cs["faces"], K, 1 / K, cs["dirs"], q, a, X, precision=precision)
    J = _loss(torch, pinf, cs["w"])
    if perturb_between:  # another forward replaces the context's factors
        farfield_solve(c, cs["faces"], K, 1 / K, cs["dirs"], q.detach() * 1.7, a.detach(), X.detach() * 1.01,
                       precision=precision)
    J.backward()
    return float(J), q.grad.numpy(), a.grad.numpy(), X.grad.numpy()


def test_autograd_matches_central_differences(case):
    torch = pytest.importorskip("torch")
    from beat_engine_b200.autodiff import farfield_solve
    cs = case
    with _lib.Context(0) as c:
        c.set_mesh(cs["X"], cs["faces"], 4, 4)
        _, gq, ga, gX = _grads(torch, c, cs, _lib.FP64)

        def J(q, a, X):
            with torch.no_grad():
                p = farfield_solve(c, cs["faces"], K, 1 / K, cs["dirs"], torch.tensor(q), torch.tensor(a),
                                   torch.tensor(X), precision=_lib.FP64)
                return float(_loss(torch, p, cs["w"]))

        rng = np.random.default_rng(42)
        h = 1e-6
        for _ in range(3):
            dq = rng.standard_normal(cs["q"].shape) + 1j * rng.standard_normal(cs["q"].shape)
            da = 0.05 * (rng.standard_normal(cs["a"].shape) + 1j * rng.standard_normal(cs["a"].shape))
            dX = 0.1 * rng.standard_normal(cs["X"].shape)
            # torch's complex gradient is 2 dJ/d conj(z): dJ = Re <grad, dz>
            pred = (np.real(np.vdot(gq, dq)) + np.real(np.vdot(ga, da)) + float(np.sum(gX * dX)))
            fd = (J(cs["q"] + h * dq, cs["a"] + h * da, cs["X"] + h * dX) -
                  J(cs["q"] - h * dq, cs["a"] - h * da, cs["X"] - h * dX)) / (2 * h)
            assert abs(fd - pred) <= 1e-6 * abs(fd), (fd, pred)
        # each input alone, so no term can hide behind another (J moves little with
        # the admittance: a direction 100 times larger keeps the difference well
        # above the rounding of J, and h times it still small against a)
        for dq, da, dX in ((rng.standard_normal(cs["q"].shape) + 0j, 0 * cs["a"], 0 * cs["X"]),
                           (0 * cs["q"], 5.0 * rng.standard_normal(cs["a"].shape) + 0j, 0 * cs["X"]),
                           (0 * cs["q"], 0 * cs["a"], 0.1 * rng.standard_normal(cs["X"].shape))):
            pred = np.real(np.vdot(gq, dq)) + np.real(np.vdot(ga, da)) + float(np.sum(gX * dX))
            fd = (J(cs["q"] + h * dq, cs["a"] + h * da, cs["X"] + h * dX) -
                  J(cs["q"] - h * dq, cs["a"] - h * da, cs["X"] - h * dX)) / (2 * h)
            assert abs(fd - pred) <= 1e-6 * abs(fd), (fd, pred)


def test_autograd_backward_after_another_solve_and_mixed_form(case):
    torch = pytest.importorskip("torch")
    cs = case
    with _lib.Context(0) as c:
        c.set_mesh(cs["X"], cs["faces"], 4, 4)
        J0, gq0, ga0, gX0 = _grads(torch, c, cs, _lib.FP64)
        J1, gq1, ga1, gX1 = _grads(torch, c, cs, _lib.FP64, perturb_between=True)
        assert J1 == pytest.approx(J0, rel=1e-13)
        for g0, g1 in ((gq0, gq1), (ga0, ga1), (gX0, gX1)):
            assert np.linalg.norm(g1 - g0) <= 1e-10 * np.linalg.norm(g0)
        Jm, gqm, gam, gXm = _grads(torch, c, cs, _lib.MIXED_FP32_IR)
        assert Jm == pytest.approx(J0, rel=1e-5)
        for g0, g1 in ((gq0, gqm), (ga0, gam), (gX0, gXm)):
            assert np.linalg.norm(g1 - g0) <= 1e-5 * np.linalg.norm(g0)
