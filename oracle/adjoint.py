"""CPU restatement (numpy, FP64) of the admittance boundary condition and of
the adjoint gradients of a far-field functional.  Test infrastructure only:
the tests compare the library against it, nothing ships it.

Neither exists in the reference's exterior path (its admittance is a
coupled-FEM wall model, BeatEngineCoupled.jl:594-623; it computes no
gradients), so parity is unpinned by the reference.  The restatement is
pinned by central finite differences of its own forward model
(tests/test_adjoint_oracle.py).  With a = 0 the forward model is the
reference's solve (the oracle's assembly and far field):

    q      = q0 - diag(a) P p,   P = face average of the P1 pressure
    p      = (A + B diag(a) P)^-1 B q0
    p_inf  = Fp p + Fq q
    g      = dJ/d conj(p_inf) for a real functional J
    w      = B^H (A'^H)^-1 E^H g + Fq^H g,   E = Fp - Fq diag(a) P
    dJ/d conj(q0) = w,   dJ/d conj(a_f) = -sum_r w[f, r] conj((P p)[f, r])
"""
import numpy as np

from . import assemble, farfield


def face_average(mesh):
    """P (F x N): (P p)_f = mean of p over the face's three vertices."""
    F, N = mesh.num_faces, mesh.num_vertices
    P = np.zeros((F, N))
    for f, tri in enumerate(np.asarray(mesh.faces)):
        for v in tri:
            P[f, v] += 1.0 / 3.0
    return P


def operators(mesh, k_signed, eta, quad_order=4, sing_order=4):
    """The assembled A (N x N) and the RHS operator B (N x F), b = B q."""
    F = mesh.num_faces
    A, B = assemble(mesh, k_signed, eta, np.eye(F, dtype=np.complex128), quad_order, sing_order)
    return A, B


def farfield_operators(mesh, k_signed, dirs, quad_order=4):
    """Fp (M x N) and Fq (M x F) with p_inf = Fp p + Fq q."""
    N, F = mesh.num_vertices, mesh.num_faces
    Fp = farfield(mesh, k_signed, dirs, np.eye(N, dtype=np.complex128), np.zeros((F, N), np.complex128), quad_order)
    Fq = farfield(mesh, k_signed, dirs, np.zeros((N, F), np.complex128), np.eye(F, dtype=np.complex128), quad_order)
    return Fp, Fq


def forward(A, B, P, a, q0):
    """Pressures p (N x R) and the boundary Neumann data q (F x R)."""
    Ap = A + B @ (a[:, None] * P)
    p = np.linalg.solve(Ap, B @ q0)
    return p, q0 - a[:, None] * (P @ p)


def adjoint(A, B, P, a, Fp, Fq, p, g):
    """(dJ/d conj(q0): F x R, dJ/d conj(a): F) for g = dJ/d conj(p_inf)."""
    Ap = A + B @ (a[:, None] * P)
    E = Fp - Fq @ (a[:, None] * P)
    z = np.linalg.solve(Ap.conj().T, E.conj().T @ g)
    w = B.conj().T @ z + Fq.conj().T @ g
    ga = -np.sum(w * np.conj(P @ p), axis=1)
    return w, ga
