"""Frequency sweep (beat_b200_sweep / beat_b200_sweep_device) against one
solve per frequency on the same context, through the C ABI.

A sweep runs the same kernels as beat_b200_solve, pipelined over up to six
solve lanes (four in FP64); only the order of the floating-point atomic sums
in the assembly can differ between the two runs.  Tolerances: mixed form relative L2 per column
<= 1e-6 (the target of the form), FP64 <= 1e-10, far field the same.
"""
import numpy as np
import pytest
import torch

from beat_engine_b200 import _lib
from beat_engine_b200 import mesh as M

pytestmark = pytest.mark.gpu


def col_rel(a, b):
    return np.linalg.norm(a - b, axis=0) / np.linalg.norm(b, axis=0)


@pytest.fixture(scope="module")
def sphere3():
    return M.reference_sphere(0.1, 3)


@pytest.fixture(scope="module")
def ctx(sphere3):
    c = _lib.Context(0)
    c.set_mesh(sphere3.vertices, sphere3.faces, 4, 4)
    yield c
    c.close()


def sweep_inputs(F, R, ks, seed):
    rng = np.random.default_rng(seed)
    q = rng.standard_normal((F, R, len(ks))) + 1j * rng.standard_normal((F, R, len(ks)))
    return np.asarray(ks, float), 1.0 / np.asarray(ks, float), np.asfortranarray(q)


@pytest.mark.parametrize("precision,tol", [(_lib.MIXED_FP32_IR, 1e-6), (_lib.FP64, 1e-10)])
def test_sweep_matches_one_solve_per_frequency(ctx, sphere3, precision, tol):
    ks = [7.0, 36.6, -52.0, 110.0, 20.0]  # both phasor signs, one frequency per lane
    k, eta, q = sweep_inputs(sphere3.num_faces, 3, ks, 5)
    dirs = M.fibonacci_sphere(17, 1.0)
    opts = _lib.Context.opts(precision)
    p, ff, diags = ctx.sweep(k, eta, q, opts, dirs)
    assert p.shape == (sphere3.num_vertices, 3, len(ks)) and ff.shape == (17, 3, len(ks))
    for f in range(len(ks)):
        pf, d = ctx.solve(k[f], eta[f], q[:, :, f], opts)
        assert np.all(col_rel(p[:, :, f], pf) <= tol), (f, col_rel(p[:, :, f], pf))
        fff = ctx.farfield(k[f], dirs, pf, q[:, :, f])
        assert np.all(col_rel(ff[:, :, f], fff) <= tol)
        assert diags[f]["precision"] == precision and diags[f]["lu_ms"] > 0
        if precision == _lib.MIXED_FP32_IR:
            assert diags[f]["ir_converged"] == 1


def test_lanes_reused_across_frequencies(ctx, sphere3):
    # more frequencies than lanes in both forms: each lane solves several in turn
    ks = [7.0, 20.0, 36.6, -52.0, 64.0, 80.0, 95.0, 110.0, 12.0, 44.0]
    k, eta, q = sweep_inputs(sphere3.num_faces, 2, ks, 7)
    for precision, tol in ((_lib.MIXED_FP32_IR, 1e-6), (_lib.FP64, 1e-10)):
        opts = _lib.Context.opts(precision)
        p, _, diags = ctx.sweep(k, eta, q, opts)
        for f in range(len(ks)):
            pf, _ = ctx.solve(k[f], eta[f], q[:, :, f], opts)
            assert np.all(col_rel(p[:, :, f], pf) <= tol), (precision, f, col_rel(p[:, :, f], pf))
            assert diags[f]["precision"] == precision


def test_sweep_device_matches_host_sweep(ctx, sphere3):
    ks = [36.6, 80.0, 12.0]
    k, eta, q = sweep_inputs(sphere3.num_faces, 4, ks, 9)
    dirs = M.fibonacci_sphere(11, 1.0)
    opts = _lib.Context.opts(_lib.MIXED_FP32_IR)
    p, ff, _ = ctx.sweep(k, eta, q, opts, dirs)
    N, F, R, nf, Md = sphere3.num_vertices, sphere3.num_faces, 4, len(ks), 11
    dev = torch.device("cuda", 0)
    # device slices: frequency-major, each F x R (N x R, M x R) column-major
    dq = torch.from_numpy(np.ascontiguousarray(np.transpose(q, (2, 1, 0)))).to(dev)
    dp = torch.zeros((nf, R, N), dtype=torch.complex128, device=dev)
    dff = torch.zeros((nf, R, Md), dtype=torch.complex128, device=dev)
    torch.cuda.synchronize()
    diags = ctx.sweep_device(k, eta, dq.data_ptr(), R, dp.data_ptr(), opts, dirs, dff.data_ptr())
    pd = np.transpose(dp.cpu().numpy(), (2, 1, 0))
    ffd = np.transpose(dff.cpu().numpy(), (2, 1, 0))
    for f in range(nf):
        assert np.all(col_rel(pd[:, :, f], p[:, :, f]) <= 1e-6)
        assert np.all(col_rel(ffd[:, :, f], ff[:, :, f]) <= 1e-6)
        assert diags[f]["ir_converged"] == 1


def test_sweep_single_frequency_and_lanes_memory(ctx, sphere3):
    k, eta, q = sweep_inputs(sphere3.num_faces, 2, [36.6], 3)
    p, ff, diags = ctx.sweep(k, eta, q, _lib.Context.opts(_lib.FP64))
    assert ff is None and len(diags) == 1
    pf, _ = ctx.solve(k[0], eta[0], q[:, :, 0], _lib.Context.opts(_lib.FP64))
    assert np.all(col_rel(p[:, :, 0], pf) <= 1e-10)
    # the second lane (created by the earlier sweeps) holds its own workspace
    before = ctx.device_bytes()
    ctx.release_workspace()
    assert ctx.device_bytes() < before


def test_sweep_errors_are_status_codes(ctx, sphere3):
    lib = _lib.load()
    k = np.array([36.6, 40.0])
    eta = 1.0 / k
    q = np.zeros((sphere3.num_faces, 2, 2), dtype=np.complex128, order="F")
    st = lib.beat_b200_sweep(ctx.handle, 2, _lib._dp(k), _lib._dp(eta), 0, _lib._dp(q), None,
                             _lib._dp(np.zeros((sphere3.num_vertices, 2, 2), dtype=np.complex128)), 0, None, None,
                             None)
    assert st == _lib.INVALID_ARG
    with pytest.raises(ValueError):
        ctx.sweep(k, eta[:1], q)
    # a zero wavenumber is rejected per frequency, with its index in the message
    with pytest.raises(_lib.BeatB200Error) as e:
        ctx.sweep(np.array([36.6, 0.0]), np.array([1 / 36.6, 1.0]), q)
    assert "frequency 1" in str(e.value)
