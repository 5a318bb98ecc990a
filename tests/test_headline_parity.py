"""Parity at the headline size: F = 20,480 faces, N = 10,242 unknowns, R = 16.

The workload bench.py times (icosphere a = 0.1 m subdivided 5 times; RHS 0 the
rigid translation along z, u_n = n_f . z; RHS 1-15 seeded complex velocities
from default_rng(1000 + r); order 4/4; exp(-i omega t)) at 500 Hz, 2 kHz and
6 kHz, through the C ABI, against the FP64 oracle's solution of the same
system (oracle assembly + LAPACK LU), stored by
tests/golden/make_headline_fixtures.py in tests/golden/headline_F20480.npz:

* full solution columns 0, 1, 2 and 15, per column relative L2 error;
* all 16 columns through 8 seeded Gaussian probes W^T p (a linear sketch whose
  mean square estimates ||p_r||^2; its relative error estimates each column's);
* the far field of all 16 columns at 541 directions.

Tolerances: FP64 form 1e-10 per column (the oracle's own LU residual is
~1e-15); mixed form (FP32 assembly, TF32 3-split tensor-core LU, FP64 GMRES
refinement) 1e-6 per column, the headline metric's bound.  RHS 0's far field
is also checked against the analytic oscillating sphere (dipole): within the
discretisation error the oracle itself shows on this mesh, plus 1e-6.
"""
import math
import os

import numpy as np
import pytest

from beat_engine_b200 import _lib
from beat_engine_b200 import mesh as M

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "headline_F20480.npz")
C0, RHO = 343.0, 1.21
FREQS = (500.0, 2000.0, 6000.0)
PROBE_SEED, PROBES = 77, 8


@pytest.fixture(scope="module")
def gold():
    if not os.path.exists(GOLD):
        pytest.fail("tests/golden/headline_F20480.npz is missing: run tests/golden/make_headline_fixtures.py")
    return dict(np.load(GOLD))


@pytest.fixture(scope="module")
def setup():
    mesh = M.reference_sphere(0.1, 5)
    F, R = mesh.num_faces, 16
    vel = np.zeros((F, R), dtype=np.complex128)
    vel[:, 0] = mesh.normals[:, 2]
    for r in range(1, R):
        rng = np.random.default_rng(1000 + r)
        vel[:, r] = rng.standard_normal(F) + 1j * rng.standard_normal(F)
    rng = np.random.default_rng(PROBE_SEED)
    W = rng.standard_normal((mesh.num_vertices, PROBES)) + 1j * rng.standard_normal((mesh.num_vertices, PROBES))
    dirs = M.equator_meridian_directions(360, 181)
    ctx = _lib.Context(0)
    ctx.set_mesh(mesh.vertices, mesh.faces, 4, 4)
    yield mesh, vel, W, dirs, ctx
    ctx.close()


def dipole_farfield(dirs, k, omega, radius=0.1):
    z = k * radius
    dh1 = np.exp(1j * z) * (-1j / z + 2 / z ** 2 + 2j / z ** 3)
    return 1j * RHO * omega * (-1.0 / k) / (k * dh1) * dirs[:, 2]


@pytest.mark.parametrize("precision,tol", [(_lib.FP64, 1e-10), (_lib.MIXED_FP32_IR, 1e-6)])
@pytest.mark.parametrize("f", FREQS)
def test_headline_against_oracle(gold, setup, precision, tol, f):
    mesh, vel, W, dirs, ctx = setup
    om = 2 * math.pi * f
    k = om / C0
    q = 1j * RHO * om * vel
    p, diag = ctx.solve(k, 1.0 / k, q, _lib.Context.opts(precision))
    assert diag["precision"] == precision  # no FP64 fallback in the mixed form
    tag = f"_{int(f)}"
    keep = list(gold["keep"])
    ref = gold["p_cols" + tag]
    err_cols = np.linalg.norm(p[:, keep] - ref, axis=0) / np.linalg.norm(ref, axis=0)
    assert err_cols.max() <= tol, err_cols
    # every column through the probe sketch
    proj = W.T @ p
    err_proj = np.sqrt(np.mean(np.abs(proj - gold["proj" + tag]) ** 2, axis=0)) / gold["pnorm" + tag]
    assert err_proj.max() <= tol, err_proj
    ff = ctx.farfield(k, dirs, p, q)
    fref = gold["ff" + tag]
    err_ff = np.linalg.norm(ff - fref, axis=0) / np.linalg.norm(fref, axis=0)
    assert err_ff.max() <= tol, err_ff
    # RHS 0: the analytic oscillating sphere, within the oracle's own mesh error
    ana = dipole_farfield(dirs, k, om)
    dip = np.linalg.norm(ff[:, 0] - ana) / np.linalg.norm(ana)
    assert dip <= float(gold["dipole_err" + tag]) + 1e-6, (dip, float(gold["dipole_err" + tag]))
    assert dip <= 0.02


def test_headline_sweep_against_oracle(gold, setup):
    """The three frequencies as one pipelined sweep (the bench's path), mixed
    form, against the oracle."""
    mesh, vel, W, dirs, ctx = setup
    ks = np.array([2 * math.pi * f / C0 for f in FREQS])
    q = np.stack([1j * RHO * 2 * math.pi * f * vel for f in FREQS], axis=2)
    p, ff, diags = ctx.sweep(ks, 1.0 / ks, q, _lib.Context.opts(_lib.MIXED_FP32_IR), dirs)
    for i, f in enumerate(FREQS):
        tag = f"_{int(f)}"
        assert diags[i]["ir_converged"] == 1
        proj = W.T @ p[:, :, i]
        err_proj = np.sqrt(np.mean(np.abs(proj - gold["proj" + tag]) ** 2, axis=0)) / gold["pnorm" + tag]
        assert err_proj.max() <= 1e-6, (f, err_proj)
        fref = gold["ff" + tag]
        err_ff = np.linalg.norm(ff[:, :, i] - fref, axis=0) / np.linalg.norm(fref, axis=0)
        assert err_ff.max() <= 1e-6, (f, err_ff)
