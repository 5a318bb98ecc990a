"""FP64 CPU oracle for the exterior Burton-Miller path.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` as the checker.  The product package
``beat_engine_b200`` never imports it.

``bem_oracle.c`` restates the reference's fused CPU assembly, dense LU and
field evaluator (citations in that file); this module is its ctypes binding.
Matrices use Julia's column-major layout: ``A[i + j*N]``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libbemoracle.so")
_lib = None

SKIP_REGULAR, SKIP_SINGULAR, SKIP_IDENTITY, NO_CLEAR = 1, 2, 4, 8


def build(force: bool = False) -> str:
    """Compile ``bem_oracle.c`` with the committed Makefile (gcc + OpenMP)."""
    src = os.path.join(_HERE, "bem_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
        c_int, c_double = ctypes.c_int, ctypes.c_double
        L.bo_assemble_range.argtypes = [c_int, dp, c_int, ip, c_int, c_int, c_double, c_double,
                                        c_int, dp, dp, dp, c_int, c_int, c_int, c_int]
        L.bo_lu_factor.argtypes = [c_int, dp, ip, c_int]
        L.bo_lu_solve.argtypes = [c_int, dp, ip, c_int, dp]
        L.bo_field.argtypes = [c_int, dp, c_int, ip, c_int, c_double, c_int, dp, c_int, dp, dp, dp, c_int]
        L.bo_farfield.argtypes = L.bo_field.argtypes
        L.bo_triangle_rule.argtypes = [c_int, dp, dp]
        L.bo_gauss_rule_1d.argtypes = [c_int, dp, dp]
        L.bo_duffy_rule.argtypes = [c_int, c_int, dp, dp, dp]
        L.bo_singular_pairs.argtypes = [c_int, dp, c_int, ip, c_int, c_int, ip, ip, ip, ip, ip]
        L.bo_mesh_geometry.argtypes = [c_int, dp, c_int, ip, dp, dp, dp]
        L.bo_symmetry_snap.argtypes = [c_int, dp, c_int]
        L.bo_assemble_sym.argtypes = [c_int, dp, c_int, ip, c_int, c_int, c_double, c_double,
                                      c_int, dp, dp, dp, c_int, c_int]
        L.bo_field_sym.argtypes = [c_int, dp, c_int, ip, c_int, c_double, c_int, dp, c_int, dp, dp, dp, c_int,
                                   c_int, c_int]
        L.bo_field_gradient.argtypes = [c_int, dp, c_int, ip, c_int, c_double, c_int, dp, c_int, dp, dp, dp,
                                        c_int, c_int]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _mesh_args(mesh):
    v = np.ascontiguousarray(mesh.vertices, dtype=np.float64)
    f = np.ascontiguousarray(mesh.faces, dtype=np.int32)
    return v, f


def assemble(mesh, k_signed, eta, q=None, quad_order=4, sing_order=4, threads=0, flags=0,
             test_range=None, out=None):
    """Fused Burton-Miller system ``(A, b)``: ``A`` is ``N x N`` complex128,
    ``b`` ``N x R``.  ``q`` is ``F x R`` (or ``F``) complex Neumann data,
    ``k_signed`` the outgoing wavenumber, ``eta`` the imaginary part of the
    coupling (``burton_miller_coupling``).  ``test_range`` restricts the
    element pairs to test faces [t0, t1); ``out = (A, b)`` (Fortran-ordered
    complex128, ``b`` with max(R, 1) columns) reuses buffers, and with
    ``flags & NO_CLEAR`` the slice accumulates into them."""
    v, f = _mesh_args(mesh)
    N, F = mesh.num_vertices, mesh.num_faces
    if q is None:
        q = np.zeros((F, 0), dtype=np.complex128)
    q = np.asarray(q, dtype=np.complex128)
    if q.ndim == 1:
        q = q[:, None]
    R = q.shape[1]
    qf = np.asfortranarray(q)
    if out is None:
        A = np.zeros((N, N), dtype=np.complex128, order="F")
        b = np.zeros((N, max(R, 1)), dtype=np.complex128, order="F")
    else:
        A, b = out
        if (A.shape != (N, N) or b.shape != (N, max(R, 1)) or A.dtype != np.complex128 or b.dtype != np.complex128
                or not A.flags.f_contiguous or not b.flags.f_contiguous):
            raise ValueError("out must be Fortran-ordered complex128 (N x N, N x max(R, 1)) buffers")
    t0, t1 = (0, F) if test_range is None else test_range
    st = lib().bo_assemble_range(N, _dp(v), F, _ip(f), quad_order, sing_order, float(k_signed), float(eta),
                                 R, qf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                 A.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                 b.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), threads, flags, t0, t1)
    if st != 0:
        raise RuntimeError(f"oracle assembly failed with status {st}")
    return A, b[:, :R]


def lu_solve(A, b, threads=0):
    """Partial-pivot complex LU (izamax pivoting) and solve for all columns."""
    N = A.shape[0]
    LU = np.array(A, dtype=np.complex128, order="F", copy=True)
    piv = np.zeros(N, dtype=np.int32)
    st = lib().bo_lu_factor(N, LU.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _ip(piv), threads)
    if st != 0:
        raise RuntimeError("oracle LU: singular matrix")
    B = np.array(b, dtype=np.complex128, order="F", copy=True)
    if B.ndim == 1:
        B = B[:, None]
    lib().bo_lu_solve(N, LU.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _ip(piv), B.shape[1],
                      B.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return B


def _field_common(fn, mesh, k_signed, pts, p, q, quad_order, threads):
    v, f = _mesh_args(mesh)
    pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    p = np.asarray(p, dtype=np.complex128)
    q = np.asarray(q, dtype=np.complex128)
    if p.ndim == 1:
        p, q = p[:, None], q[:, None]
    R, M = p.shape[1], pts.shape[0]
    pf, qf = np.asfortranarray(p), np.asfortranarray(q)
    out = np.zeros((M, R), dtype=np.complex128, order="F")
    st = fn(mesh.num_vertices, _dp(v), mesh.num_faces, _ip(f), quad_order, float(k_signed), M, _dp(pts), R,
            pf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), qf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), threads)
    if st != 0:
        raise RuntimeError(f"oracle field failed with status {st}")
    return out


def field(mesh, k_signed, points, p, q, quad_order=4, threads=0):
    """Pressure at observation points (``M x R``)."""
    return _field_common(lib().bo_field, mesh, k_signed, points, p, q, quad_order, threads)


def farfield(mesh, k_signed, dirs, p, q, quad_order=4, threads=0):
    """Far-field pattern ``lim r exp(-i k r) p(r d)`` (``M x R``)."""
    return _field_common(lib().bo_farfield, mesh, k_signed, dirs, p, q, quad_order, threads)


def triangle_rule(order):
    pts, w = np.zeros(2 * 16), np.zeros(16)
    n = lib().bo_triangle_rule(order, _dp(pts), _dp(w))
    return pts[:2 * n].reshape(n, 2), w[:n]


def duffy_rule(order, kind):
    cap = order ** 4 * 6
    tp, sp, w = np.zeros(2 * cap), np.zeros(2 * cap), np.zeros(cap)
    n = lib().bo_duffy_rule(order, kind, _dp(tp), _dp(sp), _dp(w))
    return tp[:2 * n].reshape(n, 2), sp[:2 * n].reshape(n, 2), w[:n]


def singular_pairs(mesh, order=4):
    v, f = _mesh_args(mesh)
    cap = 32 * mesh.num_faces
    t, s, r = (np.zeros(cap, dtype=np.int32) for _ in range(3))
    nr, npts = np.zeros(1, dtype=np.int32), np.zeros(1, dtype=np.int32)
    n = lib().bo_singular_pairs(mesh.num_vertices, _dp(v), mesh.num_faces, _ip(f), order, cap,
                                _ip(t), _ip(s), _ip(r), _ip(nr), _ip(npts))
    if n < 0:
        raise RuntimeError("invalid mesh")
    return t[:n], s[:n], r[:n], int(nr[0]), int(npts[0])


def mesh_geometry(mesh):
    v, f = _mesh_args(mesh)
    F = mesh.num_faces
    n, a, c = np.zeros(3 * F), np.zeros(F), np.zeros(9 * F)
    st = lib().bo_mesh_geometry(mesh.num_vertices, _dp(v), F, _ip(f), _dp(n), _dp(a), _dp(c))
    if st != 0:
        raise RuntimeError("invalid mesh")
    return n.reshape(F, 3), a, c.reshape(F, 3, 3)


# symmetry modes (normalized_symmetry_mode, BeatEngineCore.jl:448-454)
SYMMETRY_MODES = {"off": 0, "x": 1, "xy": 2, "ground": 3}


def symmetry_snap(vertices, mode):
    """Vertices snapped onto the active symmetry planes (a copy); raises when a
    vertex lies outside the positive fundamental domain."""
    v = np.ascontiguousarray(vertices, dtype=np.float64).copy()
    st = lib().bo_symmetry_snap(v.shape[0], _dp(v), SYMMETRY_MODES[mode])
    if st != 0:
        raise ValueError(f"mesh is not in the fundamental domain of symmetry {mode}")
    return v


def assemble_sym(mesh, k_signed, eta, q, mode, quad_order=4, sing_order=4, threads=0):
    """``(A, b)`` of the fundamental-domain mesh with symmetry images (mode
    ``off``, ``x``, ``xy`` or ``ground``); the mesh's vertices are snapped first."""
    v = symmetry_snap(mesh.vertices, mode)
    f = np.ascontiguousarray(mesh.faces, dtype=np.int32)
    N, F = mesh.num_vertices, mesh.num_faces
    q = np.asarray(q, dtype=np.complex128)
    if q.ndim == 1:
        q = q[:, None]
    R = q.shape[1]
    qf = np.asfortranarray(q)
    A = np.zeros((N, N), dtype=np.complex128, order="F")
    b = np.zeros((N, max(R, 1)), dtype=np.complex128, order="F")
    st = lib().bo_assemble_sym(N, _dp(v), F, _ip(f), quad_order, sing_order, float(k_signed), float(eta), R,
                               qf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                               A.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                               b.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), threads, SYMMETRY_MODES[mode])
    if st != 0:
        raise RuntimeError(f"oracle symmetric assembly failed with status {st}")
    return A, b[:, :R]


def field_sym(mesh, k_signed, pts, p, q, mode, far=False, quad_order=4, threads=0):
    """Field (or far field) of the fundamental-domain solution with its images."""
    v = symmetry_snap(mesh.vertices, mode)
    f = np.ascontiguousarray(mesh.faces, dtype=np.int32)
    pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    p = np.asarray(p, dtype=np.complex128)
    q = np.asarray(q, dtype=np.complex128)
    if p.ndim == 1:
        p, q = p[:, None], q[:, None]
    R, M = p.shape[1], pts.shape[0]
    pf, qf = np.asfortranarray(p), np.asfortranarray(q)
    out = np.zeros((M, R), dtype=np.complex128, order="F")
    st = lib().bo_field_sym(mesh.num_vertices, _dp(v), mesh.num_faces, _ip(f), quad_order, float(k_signed), M,
                            _dp(pts), R, pf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                            qf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), threads, SYMMETRY_MODES[mode],
                            1 if far else 0)
    if st != 0:
        raise RuntimeError(f"oracle field failed with status {st}")
    return out


def field_gradient(mesh, k_signed, points, p, q, mode="off", quad_order=4, threads=0):
    """Pressure and its gradient at observation points (pressure_gradient_v1):
    ``M x 4 x R`` complex (value, d/dx, d/dy, d/dz), with the reference's
    adaptive near-panel correction."""
    v = symmetry_snap(mesh.vertices, mode) if mode != "off" else np.ascontiguousarray(mesh.vertices, np.float64)
    f = np.ascontiguousarray(mesh.faces, dtype=np.int32)
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
    p = np.asarray(p, dtype=np.complex128)
    q = np.asarray(q, dtype=np.complex128)
    if p.ndim == 1:
        p, q = p[:, None], q[:, None]
    R, M = p.shape[1], pts.shape[0]
    pf, qf = np.asfortranarray(p), np.asfortranarray(q)
    out = np.zeros((M, 4, R), dtype=np.complex128, order="F")
    st = lib().bo_field_gradient(mesh.num_vertices, _dp(v), mesh.num_faces, _ip(f), quad_order, float(k_signed), M,
                                 _dp(pts), R, pf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                 qf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), threads, SYMMETRY_MODES[mode])
    if st != 0:
        raise RuntimeError("oracle field gradient failed: a point is too close to the boundary"
                           if st == 4 else f"oracle field gradient failed with status {st}")
    return out
