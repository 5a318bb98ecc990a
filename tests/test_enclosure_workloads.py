"""The batched-sweep and adjoint-gradient workloads on a rounded-box
loudspeaker enclosure with a front piston, at sizes the FP64 oracle runs in
seconds:

* sweep: a 2k-face enclosure, log-spaced frequencies from 100 Hz to 8 kHz, the
  piston at 1 m/s plus 4 seeded random-velocity columns, mixed form with
  refinement through beat_b200_sweep against the oracle's FP64 solve (1e-6)
  and the plain FP64 loop (1e-10);
* adjoint: the enclosure with a 2 % seeded Gaussian normal perturbation, a dB
  objective over 72 far-field directions on the horizontal +-90 deg arc
  weighted toward a flat target, summed over two frequencies.  Its gradients
  with respect to the element normal velocity (complex), the element
  admittance (complex) and the vertex positions come from beat_b200_adjoint_shape
  and are checked along seeded random directions against central differences
  (h = 1e-6 relative) of the oracle's FP64 forward model, within 1e-5.
"""
import math

import numpy as np
import pytest

import oracle
from oracle import adjoint as adj
from beat_engine_b200 import _lib
from beat_engine_b200 import mesh as M
from beat_engine_b200.phasor import neumann_scale

pytestmark = pytest.mark.gpu
C0, RHO = 343.0, 1.21


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def velocities(m, seed):
    """Piston at 1 m/s (rest rigid) plus 4 seeded random complex columns."""
    rng = np.random.default_rng(seed)
    v = np.zeros((m.num_faces, 5), complex)
    v[m.physical_tags == 2, 0] = 1.0
    v[:, 1:] = rng.standard_normal((m.num_faces, 4)) + 1j * rng.standard_normal((m.num_faces, 4))
    return v


def test_batched_sweep_on_the_enclosure():
    m = M.rounded_box_enclosure(2000, seed=11)
    v = velocities(m, 12)
    freqs = np.geomspace(100.0, 8000.0, 4)
    ks = 2 * math.pi * freqs / C0
    q = np.stack([neumann_scale(RHO, 2 * math.pi * f) * v for f in freqs], axis=2)
    dirs = M.fibonacci_sphere(32, 1.0)
    with _lib.Context(0) as c:
        c.set_mesh(m.vertices, m.faces, 4, 4)
        p, ff, diags = c.sweep(ks, 1 / ks, q, _lib.Context.opts(_lib.MIXED_FP32_IR), dirs)
        p64, _, _ = c.sweep(ks, 1 / ks, q, _lib.Context.opts(_lib.FP64), dirs)
    for i, k in enumerate(ks):
        assert diags[i]["ir_converged"] == 1
        A, b = oracle.assemble(m, k, 1 / k, q[:, :, i])
        po = np.linalg.solve(A, b)
        assert rel(p64[:, :, i], po) <= 1e-10
        assert rel(p[:, :, i], po) <= 1e-6
    fo = oracle.farfield(m, ks[-1], dirs, p64[:, :, -1], q[:, :, -1])
    assert rel(ff[:, :, -1], fo) <= 1e-6


def horizontal_arc(n=72):
    th = np.linspace(-math.pi / 2, math.pi / 2, n)  # +-90 deg about the front axis (+z)
    return np.stack([np.sin(th), np.zeros(n), np.cos(th)], axis=1)


DB = 10.0 / math.log(10.0)


def levels(pinf):
    return DB * np.log(np.abs(pinf) ** 2)


@pytest.fixture(scope="module")
def adjoint_case():
    base = M.rounded_box_enclosure(300, seed=21)
    rng = np.random.default_rng(22)
    f = np.asarray(base.faces)
    vn = np.zeros((base.num_vertices, 3))
    for a in range(3):
        np.add.at(vn, f[:, a], base.normals * base.areas[:, None])
    vn /= np.linalg.norm(vn, axis=1)[:, None]
    h = math.sqrt(2.0 * base.areas.sum() / base.num_faces)
    X = np.asarray(base.vertices) + 0.02 * h * rng.standard_normal(base.num_vertices)[:, None] * vn
    m = M.BoundaryMesh(X, f, np.asarray(base.physical_tags))
    F = m.num_faces
    v = np.where(m.physical_tags == 2, 1.0, 0.0) + 0.1 * (rng.standard_normal(F) + 1j * rng.standard_normal(F))
    Y = 0.002 * (rng.standard_normal(F) + 1j * rng.standard_normal(F))
    freqs = np.array([250.0, 4000.0])
    dirs = horizontal_arc()
    w = np.where(np.abs(dirs[:, 0]) < 0.5, 2.0, 1.0)  # on-axis directions weigh more
    targets = []
    for fr in freqs:
        pinf = forward_far_field(m, fr, v, Y, dirs)
        targets.append(levels(pinf).mean())  # the flat target: the design's mean level
    return dict(mesh=m, v=v, Y=Y, freqs=freqs, dirs=dirs, w=w, targets=np.array(targets))


def forward_far_field(m, fr, v, Y, dirs):
    k = 2 * math.pi * fr / C0
    s = neumann_scale(RHO, 2 * math.pi * fr)
    A, B = adj.operators(m, k, 1 / k)
    Fp, Fq = adj.farfield_operators(m, k, dirs)
    p, q = adj.forward(A, B, adj.face_average(m), s * Y, (s * v)[:, None])
    return (Fp @ p + Fq @ q)[:, 0]


def objective(case, X=None, v=None, Y=None):
    m = case["mesh"]
    if X is not None:
        m = M.BoundaryMesh(X, np.asarray(m.faces), np.asarray(m.physical_tags))
    v = case["v"] if v is None else v
    Y = case["Y"] if Y is None else Y
    J = 0.0
    for fr, t in zip(case["freqs"], case["targets"]):
        L = levels(forward_far_field(m, fr, v, Y, case["dirs"]))
        J += float(np.sum(case["w"] * (L - t) ** 2))
    return J


def test_adjoint_gradients_on_the_perturbed_enclosure(adjoint_case):
    cs = adjoint_case
    m, dirs = cs["mesh"], cs["dirs"]
    F = m.num_faces
    gv = np.zeros(F, complex)
    gY = np.zeros(F, complex)
    gX = np.zeros((m.num_vertices, 3))
    with _lib.Context(0) as c:
        c.set_mesh(m.vertices, m.faces, 4, 4)
        opts = _lib.Context.opts(_lib.FP64, flags=_lib.FLAG_RHS_CACHED)
        for fr, t in zip(cs["freqs"], cs["targets"]):
            k = 2 * math.pi * fr / C0
            s = neumann_scale(RHO, 2 * math.pi * fr)
            c.set_admittance(s * cs["Y"])
            q0 = (s * cs["v"])[:, None]
            p, _ = c.solve(k, 1 / k, q0, opts)
            pinf = c.farfield(k, dirs, p, q0)[:, 0]
            g = (2 * cs["w"] * (levels(pinf) - t) * DB / np.conj(pinf))[:, None]  # dJ/d conj(p_inf)
            w, ga, gx = c.adjoint_shape(k, dirs, p, q0, g, opts)
            gv += np.conj(s) * w[:, 0]  # q0 = s v
            gY += np.conj(s) * ga  # a = s Y
            gX += gx
        c.set_admittance(None)
    rng = np.random.default_rng(23)
    h = 1e-6
    X0 = np.asarray(m.vertices)
    for _ in range(3):
        dv = (rng.standard_normal(F) + 1j * rng.standard_normal(F)) * np.abs(cs["v"]).mean()
        dY = (rng.standard_normal(F) + 1j * rng.standard_normal(F)) * np.abs(cs["Y"]).mean()
        dX = rng.standard_normal(X0.shape) * np.abs(X0).mean()
        predicted = 2 * np.real(np.vdot(gv, dv)) + 2 * np.real(np.vdot(gY, dY)) + float(np.sum(gX * dX))
        jp = objective(cs, X0 + h * dX, cs["v"] + h * dv, cs["Y"] + h * dY)
        jm = objective(cs, X0 - h * dX, cs["v"] - h * dv, cs["Y"] - h * dY)
        fd = (jp - jm) / (2 * h)
        assert abs(fd - predicted) <= 1e-5 * abs(fd), (fd, predicted)
