"""Batched sweep over meshes of uneven size (beat_b200_sweep_batch and
beat_b200_sweep_batch_device) against one FP64 solve per (mesh, frequency),
and the smallest mesh against the FP64 oracle.

Three rounded-box enclosures with a piston (about 300, 700 and 1,200 faces),
log-spaced frequencies from 100 Hz to 8 kHz, the piston at 1 m/s plus 4
seeded random columns, mixed form with refinement: every job within 1e-6 of
the FP64 form (relative L2 over the columns), the far fields within 1e-6, the
device variant equal to the host one.  Bad batches (a context twice, a null
pointer, a lane count out of range) are status codes.
"""
import ctypes
import math

import numpy as np
import pytest

import oracle
from beat_engine_b200 import _lib
from beat_engine_b200 import mesh as M
from beat_engine_b200.phasor import neumann_scale

pytestmark = pytest.mark.gpu
C0, RHO = 343.0, 1.21


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def velocities(m, seed):
    rng = np.random.default_rng(seed)
    v = np.zeros((m.num_faces, 5), complex)
    v[m.physical_tags == 2, 0] = 1.0
    v[:, 1:] = rng.standard_normal((m.num_faces, 4)) + 1j * rng.standard_normal((m.num_faces, 4))
    return v


@pytest.fixture(scope="module")
def batch():
    meshes = [M.rounded_box_enclosure(n, seed=40 + i) for i, n in enumerate((1200, 300, 700))]
    nf = (5, 3, 4)
    ctxs, ks, qs = [], [], []
    for i, m in enumerate(meshes):
        c = _lib.Context(0)
        c.set_mesh(m.vertices, m.faces, 4, 4)
        ctxs.append(c)
        f = np.geomspace(100.0, 8000.0, nf[i])
        ks.append(2 * math.pi * f / C0)
        v = velocities(m, 50 + i)
        qs.append(np.stack([neumann_scale(RHO, 2 * math.pi * x) * v for x in f], axis=2))
    yield meshes, ctxs, ks, qs
    for c in ctxs:
        c.close()


def test_batch_matches_single_solves(batch):
    meshes, ctxs, ks, qs = batch
    dirs = M.fibonacci_sphere(24, 1.0)
    opts = [_lib.Context.opts(_lib.MIXED_FP32_IR, sweep_lanes=4) for _ in ctxs]
    out = _lib.sweep_batch(ctxs, ks, [1 / k for k in ks], qs, opts, dirs)
    for m, (p, ff, diags) in enumerate(out):
        for f in range(ks[m].size):
            assert diags[f]["ir_converged"] == 1
            p64, _ = ctxs[m].solve(ks[m][f], 1 / ks[m][f], qs[m][:, :, f], _lib.Context.opts(_lib.FP64))
            assert rel(p[:, :, f], p64) <= 1e-6, (m, f)
            f64 = ctxs[m].farfield(ks[m][f], dirs, p64, qs[m][:, :, f])
            assert rel(ff[:, :, f], f64) <= 1e-6, (m, f)
    # the smallest mesh against the oracle at its highest frequency
    m, f = 1, ks[1].size - 1
    A, b = oracle.assemble(meshes[m], ks[m][f], 1 / ks[m][f], qs[m][:, :, f])
    assert rel(out[m][0][:, :, f], np.linalg.solve(A, b)) <= 1e-6


def test_batch_device_matches_host(batch):
    torch = pytest.importorskip("torch")
    meshes, ctxs, ks, qs = batch
    dev = torch.device("cuda", 0)
    dirs = M.fibonacci_sphere(12, 1.0)
    host = _lib.sweep_batch(ctxs, ks, [1 / k for k in ks], qs, None, dirs)
    d_q, d_p, d_ff, R = [], [], [], []
    for m, c in enumerate(ctxs):
        nf = ks[m].size
        q = torch.from_numpy(np.ascontiguousarray(qs[m].transpose(2, 1, 0))).to(dev)  # nf x R x F
        d_q.append(q)
        d_p.append(torch.zeros((nf, q.shape[1], c.V), dtype=torch.complex128, device=dev))
        d_ff.append(torch.zeros((nf, q.shape[1], dirs.shape[0]), dtype=torch.complex128, device=dev))
        R.append(q.shape[1])
    diags = _lib.sweep_batch_device(ctxs, ks, [1 / k for k in ks], [t.data_ptr() for t in d_q], R,
                                    [t.data_ptr() for t in d_p], None, dirs, [t.data_ptr() for t in d_ff])
    torch.cuda.synchronize()
    for m in range(len(ctxs)):
        assert all(d["ir_converged"] == 1 for d in diags[m])
        p = d_p[m].cpu().numpy().transpose(2, 1, 0)
        ff = d_ff[m].cpu().numpy().transpose(2, 1, 0)
        assert rel(p, host[m][0]) <= 1e-6
        assert rel(ff, host[m][1]) <= 1e-6


def test_batch_errors_are_status_codes(batch):
    meshes, ctxs, ks, qs = batch
    with pytest.raises(_lib.BeatB200Error) as e:
        _lib.sweep_batch([ctxs[0], ctxs[0]], [ks[0], ks[0]], [1 / ks[0]] * 2, [qs[0], qs[0]])
    assert e.value.status == _lib.INVALID_ARG
    L = ctxs[0].lib
    st = L.beat_b200_sweep_batch(1, (ctypes.c_void_p * 1)(ctxs[0].handle.value), (ctypes.c_int32 * 1)(2), None,
                                 None, (ctypes.c_int32 * 1)(5), None, None, None, 0, None, None, None)
    assert st == _lib.INVALID_ARG
    # a bad lane count is refused, and the contexts carry on
    with pytest.raises(_lib.BeatB200Error) as e:
        _lib.sweep_batch(ctxs[:1], ks[:1], [1 / ks[0]], qs[:1], [_lib.Context.opts(sweep_lanes=99)])
    assert e.value.status == _lib.INVALID_ARG
    p, _, _ = _lib.sweep_batch(ctxs[1:2], ks[1:2], [1 / ks[1]], qs[1:2])[0]
    assert np.all(np.isfinite(p))


def test_sweep_config_subset_against_oracle():
    """The benchmark's batched-sweep workload (bench.py --config sweep): its two
    smallest enclosures at the first, middle and last of the 64 frequencies,
    as one batch in the mixed form, against the FP64 oracle (1e-6)."""
    from bench import neumann, sweep_workload
    meshes, vels, freqs = sweep_workload()
    sel = freqs[[0, 32, 63]]
    ks = 2 * math.pi * sel / C0
    ctxs = []
    try:
        for m in meshes[:2]:
            c = _lib.Context(0)
            c.set_mesh(m.vertices, m.faces, 4, 4)
            ctxs.append(c)
        qs = [np.stack([neumann(v, f) for f in sel], axis=2) for v in vels[:2]]
        out = _lib.sweep_batch(ctxs, [ks, ks], [1 / ks, 1 / ks], qs)
        for m, f in ((0, 0), (0, 1), (0, 2), (1, 2)):
            A, b = oracle.assemble(meshes[m], ks[f], 1 / ks[f], qs[m][:, :, f])
            assert rel(out[m][0][:, :, f], np.linalg.solve(A, b)) <= 1e-6, (m, f)
            assert out[m][2][f]["ir_converged"] == 1
    finally:
        for c in ctxs:
            c.close()
