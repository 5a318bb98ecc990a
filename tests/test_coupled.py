"""Coupled FEM-BEM combined operators (beat_b200_assemble_coupled_device) and
their block products (beat_b200_coupled_blocks_device) against the oracle,
as the reference's tests/coupled_bem_cuda_tests.jl:4-53 checks its CUDA
combined A/C against the four operators:
    A = 1/2 M - D + alpha H,  C = S + alpha (K' + 1/2 M_p1dp0),  alpha = i/k,
which are the oracle's direct system at eta = i/k with C = -B.

Tolerances: FP64 form 1e-12 of the largest entry; mixed form (FP32 regular
quadrature) 2e-5 of the largest entry, the reference's atol scale (rtol 2e-4,
atol 2e-5 in FP32).
"""
import numpy as np
import pytest
import torch

import oracle
from beat_engine_b200 import _lib
from beat_engine_b200 import mesh as M

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)

MESHES = {
    "off": lambda: M.reference_sphere(0.1, 2),
    "x": lambda: M.uv_sphere_patch(0.1, 8, 8, -np.pi / 2, np.pi / 2),
    "xy": lambda: M.uv_sphere_patch(0.1, 8, 4, 0, np.pi / 2),
    "ground": lambda: M.reference_sphere(0.1, 2, centre=(0.0, 0.15, 0.0)),
}


def reference_operators(m, k, mode):
    F = m.num_faces
    eye = np.eye(F, dtype=complex)
    if mode == "off":
        A, B = oracle.assemble(m, k, 1.0 / k, eye)
    else:
        A, B = oracle.assemble_sym(m, k, 1.0 / k, eye, mode)
    return A, -B


def device_operators(c, m, k, precision):
    N, F = m.num_vertices, m.num_faces
    dt = torch.complex128 if precision == _lib.FP64 else torch.complex64
    # column-major N x N / N x F == row-major (cols, rows)
    dA = torch.zeros((N, N), dtype=dt, device=DEV)
    dC = torch.zeros((F, N), dtype=dt, device=DEV)
    torch.cuda.synchronize()
    c.assemble_coupled_device(k, precision, dA.data_ptr(), dC.data_ptr())
    return dA, dC


@pytest.mark.parametrize("precision,tol", [(_lib.FP64, 1e-12), (_lib.MIXED_FP32_IR, 2e-5)])
@pytest.mark.parametrize("mode", ["off", "x", "xy", "ground"])
@pytest.mark.parametrize("k", [7.0, -70.0])
def test_combined_operators_match_oracle(mode, precision, tol, k):
    m = MESHES[mode]()
    Ao, Co = reference_operators(m, k, mode)
    with _lib.Context(0) as c:
        c.set_mesh(m.vertices, m.faces, 4, 4)
        if mode != "off":
            c.set_symmetry(mode)
        dA, dC = device_operators(c, m, k, precision)
    A = dA.cpu().numpy().T
    C = dC.cpu().numpy().T
    assert np.abs(A - Ao).max() <= tol * np.abs(Ao).max()
    assert np.abs(C - Co).max() <= tol * np.abs(Co).max()


def csc(F, ncols, seed):
    """A random F x ncols sparse map, CSC with 1-based indices (Julia's)."""
    rng = np.random.default_rng(seed)
    colptr, rowval, nz = [1], [], []
    dense = np.zeros((F, ncols), complex)
    for j in range(ncols):
        rows = np.sort(rng.choice(F, size=rng.integers(0, 4), replace=False))
        for r in rows:
            v = rng.standard_normal() + 1j * rng.standard_normal()
            rowval.append(r + 1)
            nz.append(v)
            dense[r, j] = v
        colptr.append(len(rowval) + 1)
    return np.array(colptr, np.int32), np.array(rowval, np.int32), np.array(nz), dense


@pytest.mark.parametrize("precision,tol", [(_lib.FP64, 1e-12), (_lib.MIXED_FP32_IR, 1e-5)])
def test_block_products(precision, tol):
    m = MESHES["off"]()
    N, F = m.num_vertices, m.num_faces
    dt = torch.complex128 if precision == _lib.FP64 else torch.complex64
    rng = np.random.default_rng(3)
    colptr, rowval, nz, Q = csc(F, 7, 1)
    motion = rng.standard_normal((F, 3)) + 1j * rng.standard_normal((F, 3))
    prescribed = rng.standard_normal((F, 10)) + 1j * rng.standard_normal((F, 10))  # two column passes
    with _lib.Context(0) as c:
        c.set_mesh(m.vertices, m.faces, 4, 4)
        _, dC = device_operators(c, m, 25.0, precision)
        C = dC.cpu().numpy().T.astype(complex)
        d_colptr = torch.from_numpy(colptr).to(DEV)
        d_rowval = torch.from_numpy(rowval).to(DEV)
        d_nz = torch.from_numpy(nz).to(dt).to(DEV)
        d_mot = torch.from_numpy(np.ascontiguousarray(motion.T)).to(dt).to(DEV)
        d_pre = torch.from_numpy(np.ascontiguousarray(prescribed.T)).to(dt).to(DEV)
        d_int = torch.zeros((7, N), dtype=dt, device=DEV)
        d_mo = torch.zeros((3, N), dtype=dt, device=DEV)
        d_po = torch.zeros((10, N), dtype=dt, device=DEV)
        torch.cuda.synchronize()
        c.coupled_blocks_device(precision, dC.data_ptr(), 7, d_colptr.data_ptr(), d_rowval.data_ptr(),
                                d_nz.data_ptr(), len(nz), d_int.data_ptr(), 3, d_mot.data_ptr(), d_mo.data_ptr(),
                                10, d_pre.data_ptr(), d_po.data_ptr())
        for got, want in ((d_int, C @ Q), (d_mo, C @ motion), (d_po, -C @ prescribed)):
            g = got.cpu().numpy().T
            assert np.abs(g - want).max() <= tol * np.abs(want).max()
        # an out-of-range row index is an argument error, the context stays usable
        bad = rowval.copy()
        bad[0] = F + 1
        d_bad = torch.from_numpy(bad).to(DEV)
        with pytest.raises(_lib.BeatB200Error) as e:
            c.coupled_blocks_device(precision, dC.data_ptr(), 7, d_colptr.data_ptr(), d_bad.data_ptr(),
                                    d_nz.data_ptr(), len(nz), d_int.data_ptr())
        assert e.value.status == _lib.INVALID_ARG
        p, _ = c.solve(25.0, 1 / 25.0, motion, _lib.Context.opts(_lib.FP64))
        assert np.all(np.isfinite(p))
