"""ctypes binding of libbeatb200.so (C ABI in include/beat_b200.h).

The library is built in-tree (``beat_engine_b200/libbeatb200.so``).  Loading
fails loudly when it is missing: there is no CPU fallback for the solver.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbeatb200.so")

OK, INVALID_ARG, OOM, CUDA_ERROR, NOT_CONVERGED, TIMEOUT, NO_DEVICE, STATE, SINGULAR = range(9)
FP64, MIXED_FP32_IR = 0, 1
FLAG_NO_REFINE, FLAG_RHS_MATRIX_FREE, FLAG_RHS_CACHED, FLAG_NO_FALLBACK = 1, 2, 4, 8
RHS_AUTO, RHS_MATRIX_FREE, RHS_CACHED = 0, 1, 2
RHS_MODES = {"auto": RHS_AUTO, "matrix_free": RHS_MATRIX_FREE, "cached_operator": RHS_CACHED}
STATUS_NAMES = {OK: "OK", INVALID_ARG: "INVALID_ARG", OOM: "OOM", CUDA_ERROR: "CUDA_ERROR",
                NOT_CONVERGED: "NOT_CONVERGED", TIMEOUT: "TIMEOUT", NO_DEVICE: "NO_DEVICE", STATE: "STATE",
                SINGULAR: "SINGULAR"}

# every symbol include/beat_b200.h declares
EXPORTS = (
    "beat_b200_abi_version", "beat_b200_default_opts", "beat_b200_create", "beat_b200_destroy",
    "beat_b200_last_error", "beat_b200_set_mesh", "beat_b200_solve", "beat_b200_solve_device",
    "beat_b200_field", "beat_b200_farfield", "beat_b200_farfield_device", "beat_b200_assemble",
    "beat_b200_release_workspace", "beat_b200_device_bytes", "beat_b200_stream", "beat_b200_resolve_noalloc",
    "beat_b200_sweep_batch", "beat_b200_sweep_batch_device",
    "beat_b200_sweep", "beat_b200_sweep_device", "beat_b200_set_admittance", "beat_b200_adjoint",
    "beat_b200_set_symmetry", "beat_b200_field_gradient", "beat_b200_field_gradient_device",
    "beat_b200_rhs_use_operator", "beat_b200_assemble_coupled_device", "beat_b200_coupled_blocks_device",
    "beat_b200_adjoint_shape",
)

SYMMETRY_MODES = {"off": 0, "x": 1, "xy": 2, "ground": 3}


def symmetry_mode(mode) -> int:
    """A symmetry mode name, trimmed and case-insensitive as the reference
    normalises it (``normalized_symmetry_mode``, src/BeatEngineCore.jl:448-454),
    or its number 0..3, as the C ABI's mode number.  An unknown name raises
    ``ValueError`` with the reference's message; numbers are checked by the
    library."""
    if isinstance(mode, str):
        key = mode.strip().lower()
        if key not in SYMMETRY_MODES:
            raise ValueError(f"Unsupported image mode: {mode}. Expected off, x, xy, or ground.")
        return SYMMETRY_MODES[key]
    return int(mode)


class Opts(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int32), ("ir_restart", ctypes.c_int32), ("ir_max_iters", ctypes.c_int32),
                ("lu_split_terms", ctypes.c_int32), ("ir_rtol", ctypes.c_double), ("lu_block", ctypes.c_int32),
                ("flags", ctypes.c_int32), ("sweep_lanes", ctypes.c_int32)]


class Diag(ctypes.Structure):
    _fields_ = [("assembly_ms", ctypes.c_double), ("singular_ms", ctypes.c_double),
                ("regular_ms", ctypes.c_double), ("lu_ms", ctypes.c_double),
                ("solve_ms", ctypes.c_double), ("ir_ms", ctypes.c_double), ("field_ms", ctypes.c_double),
                ("ir_iterations", ctypes.c_int32), ("ir_converged", ctypes.c_int32),
                ("ir_residual", ctypes.c_double), ("regular_pairs", ctypes.c_int64),
                ("singular_pairs", ctypes.c_int64), ("precision", ctypes.c_int32), ("lu_block", ctypes.c_int32),
                ("lu_split_terms", ctypes.c_int32), ("rhs_mode", ctypes.c_int32)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class BeatB200Error(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_lib = None


def rhs_mode(value) -> str:
    """exterior_rhs_mode (exterior_rhs_policy.jl:17-23): the normalised mode name."""
    mode = str(value).strip().lower()
    if mode not in RHS_MODES:
        raise ValueError(f"Unknown exterior right-hand-side mode: {value}. "
                         "Expected auto, matrix_free or cached_operator.")
    return mode


def use_rhs_operator(mode, excitations: int, matrix_bytes: int, operator_bytes: int, available_bytes: int) -> bool:
    """exterior_use_rhs_operator (exterior_rhs_policy.jl:38-44), evaluated by
    the library's own policy (beat_b200_rhs_use_operator)."""
    r = load().beat_b200_rhs_use_operator(RHS_MODES[rhs_mode(mode)], int(excitations), int(matrix_bytes),
                                          int(operator_bytes), int(available_bytes))
    return r == 1


def rhs_flags(mode) -> int:
    """opts.flags bits requesting a right-hand-side mode."""
    return {RHS_AUTO: 0, RHS_MATRIX_FREE: FLAG_RHS_MATRIX_FREE, RHS_CACHED: FLAG_RHS_CACHED}[RHS_MODES[rhs_mode(mode)]]


def load(path: str = LIB_PATH):
    """Load the shared library and declare its prototypes."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with `python -m beat_engine_b200.build` (nvcc, sm_100a). "
            "The exterior solver has no CPU fallback.")
    L = ctypes.CDLL(path)
    vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int32)
    i32, f64 = ctypes.c_int32, ctypes.c_double
    L.beat_b200_abi_version.restype = i32
    L.beat_b200_default_opts.argtypes = [ctypes.POINTER(Opts)]
    L.beat_b200_default_opts.restype = None
    L.beat_b200_create.argtypes = [i32, ctypes.POINTER(vp)]
    L.beat_b200_create.restype = i32
    L.beat_b200_destroy.argtypes = [vp]
    L.beat_b200_destroy.restype = i32
    L.beat_b200_last_error.argtypes = [vp]
    L.beat_b200_last_error.restype = ctypes.c_char_p
    L.beat_b200_set_mesh.argtypes = [vp, i32, dp, i32, ip, i32, i32]
    L.beat_b200_set_mesh.restype = i32
    L.beat_b200_solve.argtypes = [vp, f64, f64, i32, dp, ctypes.POINTER(Opts), dp, ctypes.POINTER(Diag)]
    L.beat_b200_solve.restype = i32
    L.beat_b200_solve_device.argtypes = [vp, f64, f64, i32, vp, ctypes.POINTER(Opts), vp, ctypes.POINTER(Diag)]
    L.beat_b200_solve_device.restype = i32
    L.beat_b200_field.argtypes = [vp, f64, i32, dp, i32, dp, dp, dp]
    L.beat_b200_field.restype = i32
    L.beat_b200_farfield.argtypes = [vp, f64, i32, dp, i32, dp, dp, dp]
    L.beat_b200_farfield.restype = i32
    L.beat_b200_farfield_device.argtypes = [vp, f64, i32, dp, i32, vp, vp, vp]
    L.beat_b200_farfield_device.restype = i32
    L.beat_b200_rhs_use_operator.argtypes = [i32, i32, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64]
    L.beat_b200_rhs_use_operator.restype = i32
    L.beat_b200_adjoint_shape.argtypes = [vp, f64, i32, dp, i32, dp, dp, dp, ctypes.POINTER(Opts), dp, dp, dp]
    L.beat_b200_adjoint_shape.restype = i32
    L.beat_b200_assemble_coupled_device.argtypes = [vp, f64, i32, vp, vp]
    L.beat_b200_assemble_coupled_device.restype = i32
    L.beat_b200_coupled_blocks_device.argtypes = [vp, i32, vp, i32, vp, vp, vp, ctypes.c_int64, vp, i32, vp, vp,
                                                  i32, vp, vp]
    L.beat_b200_coupled_blocks_device.restype = i32
    L.beat_b200_field_gradient.argtypes = [vp, f64, i32, dp, i32, dp, dp, dp]
    L.beat_b200_field_gradient.restype = i32
    L.beat_b200_field_gradient_device.argtypes = [vp, f64, i32, dp, i32, vp, vp, vp]
    L.beat_b200_field_gradient_device.restype = i32
    L.beat_b200_assemble.argtypes = [vp, f64, f64, i32, dp, i32, dp, dp]
    L.beat_b200_assemble.restype = i32
    L.beat_b200_release_workspace.argtypes = [vp]
    L.beat_b200_release_workspace.restype = i32
    L.beat_b200_device_bytes.argtypes = [vp]
    L.beat_b200_device_bytes.restype = ctypes.c_int64
    L.beat_b200_stream.argtypes = [vp]
    L.beat_b200_stream.restype = vp
    L.beat_b200_resolve_noalloc.argtypes = [vp, i32, vp, vp]
    L.beat_b200_resolve_noalloc.restype = i32
    L.beat_b200_sweep.argtypes = [vp, i32, dp, dp, i32, dp, ctypes.POINTER(Opts), dp, i32, dp, dp,
                                  ctypes.POINTER(Diag)]
    L.beat_b200_sweep.restype = i32
    L.beat_b200_sweep_device.argtypes = [vp, i32, dp, dp, i32, vp, ctypes.POINTER(Opts), vp, i32, dp, vp,
                                         ctypes.POINTER(Diag)]
    L.beat_b200_sweep_device.restype = i32
    pp = ctypes.POINTER(vp)
    L.beat_b200_sweep_batch.argtypes = [i32, pp, ip, pp, pp, ip, pp, ctypes.POINTER(Opts), pp, i32, dp, pp, pp]
    L.beat_b200_sweep_batch.restype = i32
    L.beat_b200_sweep_batch_device.argtypes = [i32, pp, ip, pp, pp, ip, pp, ctypes.POINTER(Opts), pp, i32, dp, pp,
                                               pp]
    L.beat_b200_sweep_batch_device.restype = i32
    L.beat_b200_set_symmetry.argtypes = [vp, i32]
    L.beat_b200_set_symmetry.restype = i32
    L.beat_b200_set_admittance.argtypes = [vp, dp]
    L.beat_b200_set_admittance.restype = i32
    L.beat_b200_adjoint.argtypes = [vp, f64, i32, dp, i32, dp, dp, ctypes.POINTER(Opts), dp, dp]
    L.beat_b200_adjoint.restype = i32
    _lib = L
    return L


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _c128_f(a, rows: int) -> np.ndarray:
    """Column-major complex128 view with ``rows`` rows (1-d input -> 1 column)."""
    a = np.asarray(a, dtype=np.complex128)
    if a.ndim == 1:
        a = a[:, None]
    if a.shape[0] != rows:
        raise ValueError(f"expected {rows} rows, got {a.shape[0]}")
    return np.asfortranarray(a)


class Context:
    """One device context per mesh (``beat_b200_create`` .. ``beat_b200_destroy``)."""

    generation = 0  # library calls made through this object (see _check)
    quad_order = singular_order = 4

    def __init__(self, device: int = 0):
        self.lib = load()
        h = ctypes.c_void_p()
        st = self.lib.beat_b200_create(device, ctypes.byref(h))
        if st != OK:
            raise BeatB200Error(st, "beat_b200_create failed")
        self.handle = h
        self.V = self.F = 0

    def close(self):
        if getattr(self, "handle", None):
            self.lib.beat_b200_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int):
        # every library call on this context counts: a caller that must know
        # whether the context still holds the state it left (autodiff's
        # backward) compares this counter
        self.generation += 1
        if st != OK:
            raise BeatB200Error(st, self.lib.beat_b200_last_error(self.handle).decode(errors="replace"))

    def set_mesh(self, vertices, faces0, quad_order: int = 4, singular_order: int = 4):
        v = np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1, 3)
        f = np.ascontiguousarray(np.asarray(faces0, dtype=np.int32).reshape(-1, 3) + 1, dtype=np.int32)
        self._check(self.lib.beat_b200_set_mesh(self.handle, v.shape[0], _dp(v), f.shape[0],
                                                f.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                                quad_order, singular_order))
        self.V, self.F = v.shape[0], f.shape[0]
        self.quad_order, self.singular_order = quad_order, singular_order

    @staticmethod
    def opts(precision: int = MIXED_FP32_IR, **kw) -> Opts:
        o = Opts()
        load().beat_b200_default_opts(ctypes.byref(o))
        o.precision = precision
        for k, v in kw.items():
            setattr(o, k, v)
        return o

    def solve(self, k_signed: float, eta: float, q, opts: Opts | None = None):
        qf = _c128_f(q, self.F)
        R = qf.shape[1]
        p = np.zeros((self.V, R), dtype=np.complex128, order="F")
        d = Diag()
        self._check(self.lib.beat_b200_solve(self.handle, float(k_signed), float(eta), R, _dp(qf),
                                             ctypes.byref(opts) if opts is not None else None,
                                             _dp(p), ctypes.byref(d)))
        return p, d.as_dict()

    def solve_device(self, k_signed: float, eta: float, d_q_ptr: int, R: int, d_p_ptr: int,
                     opts: Opts | None = None) -> dict:
        d = Diag()
        self._check(self.lib.beat_b200_solve_device(self.handle, float(k_signed), float(eta), R,
                                                    ctypes.c_void_p(d_q_ptr),
                                                    ctypes.byref(opts) if opts is not None else None,
                                                    ctypes.c_void_p(d_p_ptr), ctypes.byref(d)))
        return d.as_dict()

    def assemble(self, k_signed: float, eta: float, q=None, precision: int = FP64, want_matrix: bool = True):
        if q is None:
            qf = np.zeros((self.F, 0), dtype=np.complex128, order="F")
        else:
            qf = _c128_f(q, self.F)
        R = qf.shape[1]
        A = np.zeros((self.V, self.V), dtype=np.complex128, order="F") if want_matrix else None
        b = np.zeros((self.V, max(R, 1)), dtype=np.complex128, order="F")
        self._check(self.lib.beat_b200_assemble(self.handle, float(k_signed), float(eta), R,
                                                _dp(qf) if R else None, precision,
                                                _dp(A) if A is not None else None,
                                                _dp(b)))
        return A, b[:, :R]

    def _eval(self, fn, k_signed, pts, p, q):
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        pf, qf = _c128_f(p, self.V), _c128_f(q, self.F)
        if pf.shape[1] != qf.shape[1]:
            raise ValueError("p and q need the same number of columns")
        out = np.zeros((pts.shape[0], pf.shape[1]), dtype=np.complex128, order="F")
        self._check(fn(self.handle, float(k_signed), pts.shape[0], _dp(pts), pf.shape[1], _dp(pf),
                       _dp(qf), _dp(out)))
        return out

    def field(self, k_signed, points, p, q):
        return self._eval(self.lib.beat_b200_field, k_signed, points, p, q)

    def assemble_coupled_device(self, k_signed: float, precision: int, d_a_ptr: int, d_c_ptr: int):
        """beat_b200_assemble_coupled_device: A (N x N) and C (N x F), column-major,
        into device buffers (complex64 in the mixed form, complex128 in FP64)."""
        self._check(self.lib.beat_b200_assemble_coupled_device(self.handle, float(k_signed), precision,
                                                               ctypes.c_void_p(d_a_ptr), ctypes.c_void_p(d_c_ptr)))

    def coupled_blocks_device(self, precision: int, d_c_ptr: int, ncols: int, d_colptr: int, d_rowval: int,
                              d_nzval: int, nnz: int, d_interface: int, nmotion: int = 0, d_motion: int = 0,
                              d_motion_out: int = 0, nprescribed: int = 0, d_prescribed: int = 0,
                              d_prescribed_out: int = 0):
        """beat_b200_coupled_blocks_device: C Q (CSC, 1-based), C motion, -C prescribed."""
        v = ctypes.c_void_p
        self._check(self.lib.beat_b200_coupled_blocks_device(
            self.handle, precision, v(d_c_ptr), ncols, v(d_colptr), v(d_rowval), v(d_nzval), int(nnz),
            v(d_interface), nmotion, v(d_motion), v(d_motion_out), nprescribed, v(d_prescribed),
            v(d_prescribed_out)))

    def field_gradient(self, k_signed, points, p, q):
        """Pressure and gradient at points: M x 4 x R complex128 (value, d/dx,
        d/dy, d/dz per column)."""
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        pf, qf = _c128_f(p, self.V), _c128_f(q, self.F)
        if pf.shape[1] != qf.shape[1]:
            raise ValueError("p and q need the same number of columns")
        out = np.zeros((pts.shape[0], 4, pf.shape[1]), dtype=np.complex128, order="F")
        self._check(self.lib.beat_b200_field_gradient(self.handle, float(k_signed), pts.shape[0], _dp(pts),
                                                      pf.shape[1], _dp(pf), _dp(qf), _dp(out)))
        return out

    def farfield(self, k_signed, dirs, p, q):
        return self._eval(self.lib.beat_b200_farfield, k_signed, dirs, p, q)

    def farfield_device(self, k_signed, dirs, R, d_p_ptr, d_q_ptr, d_out_ptr):
        dirs = np.ascontiguousarray(dirs, dtype=np.float64).reshape(-1, 3)
        self._check(self.lib.beat_b200_farfield_device(self.handle, float(k_signed), dirs.shape[0], _dp(dirs), R,
                                                       ctypes.c_void_p(d_p_ptr), ctypes.c_void_p(d_q_ptr),
                                                       ctypes.c_void_p(d_out_ptr)))

    def sweep(self, k_signed, eta, q, opts: Opts | None = None, dirs=None):
        """Frequency sweep through beat_b200_sweep: q is F x R x nfreq complex128
        (frequency f's Neumann data in q[:, :, f]).  Returns (p: N x R x nfreq,
        far field: M x R x nfreq or None, per-frequency diagnostics)."""
        k_signed = np.ascontiguousarray(k_signed, dtype=np.float64).ravel()
        eta = np.ascontiguousarray(eta, dtype=np.float64).ravel()
        nf = k_signed.size
        if eta.size != nf:
            raise ValueError("k_signed and eta must have one entry per frequency")
        q = np.asfortranarray(np.asarray(q, dtype=np.complex128).reshape(self.F, -1, nf))
        R = q.shape[1]
        p = np.zeros((self.V, R, nf), dtype=np.complex128, order="F")
        M = 0
        dd = None
        ff = None
        if dirs is not None:
            dd = np.ascontiguousarray(dirs, dtype=np.float64).reshape(-1, 3)
            M = dd.shape[0]
            ff = np.zeros((M, R, nf), dtype=np.complex128, order="F")
        diags = (Diag * max(nf, 1))()
        self._check(self.lib.beat_b200_sweep(
            self.handle, nf, _dp(k_signed), _dp(eta), R, _dp(q), ctypes.byref(opts) if opts is not None else None,
            _dp(p), M, _dp(dd) if dd is not None else None, _dp(ff) if ff is not None else None, diags))
        return p, ff, [diags[i].as_dict() for i in range(nf)]

    def sweep_device(self, k_signed, eta, d_q_ptr: int, R: int, d_p_ptr: int, opts: Opts | None = None,
                     dirs=None, d_ff_ptr: int = 0) -> list:
        """beat_b200_sweep_device: q, p and the far field in device memory
        (F x R, N x R and M x R complex128 slices, one per frequency)."""
        k_signed = np.ascontiguousarray(k_signed, dtype=np.float64).ravel()
        eta = np.ascontiguousarray(eta, dtype=np.float64).ravel()
        nf = k_signed.size
        dd = np.ascontiguousarray(dirs, dtype=np.float64).reshape(-1, 3) if dirs is not None else None
        M = 0 if dd is None else dd.shape[0]
        diags = (Diag * max(nf, 1))()
        self._check(self.lib.beat_b200_sweep_device(
            self.handle, nf, _dp(k_signed), _dp(eta), R, ctypes.c_void_p(d_q_ptr),
            ctypes.byref(opts) if opts is not None else None, ctypes.c_void_p(d_p_ptr), M,
            _dp(dd) if dd is not None else None, ctypes.c_void_p(d_ff_ptr), diags))
        return [diags[i].as_dict() for i in range(nf)]

    def set_symmetry(self, mode):
        """Symmetry images: "off", "x", "xy" or "ground" (or 0..3)."""
        self._check(self.lib.beat_b200_set_symmetry(self.handle, symmetry_mode(mode)))

    def set_admittance(self, a=None):
        """Per-face admittance coefficients a (F complex): later solves use
        q = q0 - a (P p).  None clears them."""
        if a is None:
            self._check(self.lib.beat_b200_set_admittance(self.handle, None))
            return
        a = np.ascontiguousarray(np.asarray(a, dtype=np.complex128).ravel())
        if a.size != self.F:
            raise ValueError(f"expected {self.F} coefficients, got {a.size}")
        self._check(self.lib.beat_b200_set_admittance(self.handle, _dp(a)))

    def adjoint(self, k_signed: float, dirs, p, g, opts: Opts | None = None, want_admittance: bool = True):
        """Gradients of a real far-field functional after a solve at k_signed:
        g = dJ/d conj(p_inf) (M x R).  Returns (dJ/d conj(q0): F x R,
        dJ/d conj(a): F or None)."""
        dd = np.ascontiguousarray(dirs, dtype=np.float64).reshape(-1, 3)
        M = dd.shape[0]
        pf = _c128_f(p, self.V)
        R = pf.shape[1]
        gf = _c128_f(g, M)
        if gf.shape[1] != R:
            raise ValueError("p and g need the same number of columns")
        w = np.zeros((self.F, R), dtype=np.complex128, order="F")
        ga = np.zeros(self.F, dtype=np.complex128) if want_admittance else None
        self._check(self.lib.beat_b200_adjoint(self.handle, float(k_signed), M, _dp(dd), R, _dp(pf), _dp(gf),
                                               ctypes.byref(opts) if opts is not None else None, _dp(w),
                                               _dp(ga) if ga is not None else None))
        return w, ga

    def adjoint_shape(self, k_signed: float, dirs, p, q, g, opts: Opts | None = None):
        """beat_b200_adjoint_shape: (dJ/d conj(q0): F x R, dJ/d conj(a): F,
        dJ/dX: V x 3) after a solve at k_signed with Neumann data q."""
        dd = np.ascontiguousarray(dirs, dtype=np.float64).reshape(-1, 3)
        M = dd.shape[0]
        pf, qf = _c128_f(p, self.V), _c128_f(q, self.F)
        R = pf.shape[1]
        gf = _c128_f(g, M)
        if gf.shape[1] != R or qf.shape[1] != R:
            raise ValueError("p, q and g need the same number of columns")
        w = np.zeros((self.F, R), dtype=np.complex128, order="F")
        ga = np.zeros(self.F, dtype=np.complex128)
        gx = np.zeros((self.V, 3), dtype=np.float64)
        self._check(self.lib.beat_b200_adjoint_shape(self.handle, float(k_signed), M, _dp(dd), R, _dp(pf), _dp(qf),
                                                     _dp(gf), ctypes.byref(opts) if opts is not None else None,
                                                     _dp(w), _dp(ga), _dp(gx)))
        return w, ga, gx

    def release_workspace(self):
        self._check(self.lib.beat_b200_release_workspace(self.handle))

    def device_bytes(self) -> int:
        return int(self.lib.beat_b200_device_bytes(self.handle))

    def resolve_noalloc(self, R: int, d_b_ptr: int, d_x_ptr: int) -> None:
        """Solve R more right-hand sides (device N x R complex128, column-major)
        with the current factors, allocating nothing (beat_b200_resolve_noalloc)."""
        self._check(self.lib.beat_b200_resolve_noalloc(self.handle, R, ctypes.c_void_p(d_b_ptr),
                                                       ctypes.c_void_p(d_x_ptr)))

    def stream_handle(self) -> int:
        """cudaStream_t of this context as an integer (for torch.cuda.ExternalStream)."""
        return int(self.lib.beat_b200_stream(self.handle) or 0)


def _ptrs(arrays):
    """ctypes array of the data pointers of `arrays` (None -> NULL)."""
    return (ctypes.c_void_p * len(arrays))(*[None if a is None else a.ctypes.data for a in arrays])


def _handles(ctxs):
    return (ctypes.c_void_p * len(ctxs))(*[c.handle.value for c in ctxs])


def sweep_batch(ctxs, k_signed, eta, q, opts=None, dirs=None):
    """Several meshes' frequency sweeps as one job list (beat_b200_sweep_batch):
    ``ctxs[m]`` is mesh m's context, ``k_signed[m]`` / ``eta[m]`` its
    frequencies' wavenumbers and couplings, ``q[m]`` its F x R x nfreq Neumann
    data, ``opts[m]`` (or None) its options.  The lanes take the jobs in
    decreasing order of cost.  Returns per mesh (p: N x R x nfreq, far field:
    M x R x nfreq or None, diagnostics)."""
    nm = len(ctxs)
    L = ctxs[0].lib
    ks = [np.ascontiguousarray(k, dtype=np.float64).ravel() for k in k_signed]
    es = [np.ascontiguousarray(e, dtype=np.float64).ravel() for e in eta]
    qs, ps, ffs, diags = [], [], [], []
    dd = None if dirs is None else np.ascontiguousarray(dirs, dtype=np.float64).reshape(-1, 3)
    M = 0 if dd is None else dd.shape[0]
    for m, c in enumerate(ctxs):
        nf = ks[m].size
        if es[m].size != nf:
            raise ValueError("k_signed and eta must have one entry per frequency")
        qm = np.asfortranarray(np.asarray(q[m], dtype=np.complex128).reshape(c.F, -1, nf))
        qs.append(qm)
        R = qm.shape[1]
        ps.append(np.zeros((c.V, R, nf), dtype=np.complex128, order="F"))
        ffs.append(np.zeros((M, R, nf), dtype=np.complex128, order="F") if M else None)
        diags.append((Diag * max(nf, 1))())
    nfreq = (ctypes.c_int32 * nm)(*[k.size for k in ks])
    Rs = (ctypes.c_int32 * nm)(*[qm.shape[1] for qm in qs])
    optarr = None
    if opts is not None:
        optarr = (Opts * nm)(*[o if o is not None else Context.opts() for o in opts])
    dg = (ctypes.c_void_p * nm)(*[ctypes.addressof(d) for d in diags])
    st = L.beat_b200_sweep_batch(nm, _handles(ctxs), nfreq, _ptrs(ks), _ptrs(es), Rs, _ptrs(qs), optarr, _ptrs(ps),
                                 M, _dp(dd) if dd is not None else None, _ptrs(ffs) if M else None, dg)
    for c in ctxs[1:]:
        c.generation += 1
    ctxs[0]._check(st)
    return [(ps[m], ffs[m], [diags[m][i].as_dict() for i in range(ks[m].size)]) for m in range(nm)]


def sweep_batch_device(ctxs, k_signed, eta, d_q, R, d_p, opts=None, dirs=None, d_ff=None):
    """beat_b200_sweep_batch_device: per mesh m, d_q[m], d_p[m] and d_ff[m] are
    device pointers (F x R, N x R, M x R complex128 slices, one per frequency).
    Returns each mesh's per-frequency diagnostics."""
    nm = len(ctxs)
    L = ctxs[0].lib
    ks = [np.ascontiguousarray(k, dtype=np.float64).ravel() for k in k_signed]
    es = [np.ascontiguousarray(e, dtype=np.float64).ravel() for e in eta]
    dd = None if dirs is None else np.ascontiguousarray(dirs, dtype=np.float64).reshape(-1, 3)
    M = 0 if dd is None else dd.shape[0]
    diags = [(Diag * max(k.size, 1))() for k in ks]
    nfreq = (ctypes.c_int32 * nm)(*[k.size for k in ks])
    Rs = (ctypes.c_int32 * nm)(*R)
    optarr = None
    if opts is not None:
        optarr = (Opts * nm)(*[o if o is not None else Context.opts() for o in opts])
    vpa = ctypes.c_void_p * nm
    dg = vpa(*[ctypes.addressof(d) for d in diags])
    st = L.beat_b200_sweep_batch_device(nm, _handles(ctxs), nfreq, _ptrs(ks), _ptrs(es), Rs, vpa(*d_q), optarr,
                                        vpa(*d_p), M, _dp(dd) if dd is not None else None,
                                        vpa(*d_ff) if M else None, dg)
    for c in ctxs[1:]:
        c.generation += 1
    ctxs[0]._check(st)
    return [[diags[m][i].as_dict() for i in range(ks[m].size)] for m in range(nm)]
