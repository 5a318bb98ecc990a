"""Host-side mirror of the reference's exterior direct-system interface.

Paths relative to ``src/beat_engine/julia_local/``:

* :func:`solve_exterior_direct_b200` mirrors ``solve_exterior_direct_cuda``
  (``BeatEngineCompiledDriver.jl:870-915``): Neumann values per excitation in,
  boundary pressures per excitation out, one factorisation for all of them,
  plus the assembly and solve seconds.
* :func:`evaluate_galerkin_field_b200` mirrors ``evaluate_galerkin_field_cuda``
  (``src/BeatEngineCudaField.jl:329-389``).
* :func:`exterior_neumann` mirrors ``exterior_neumann``
  (``BeatEngineCompiledDriver.jl:825-839``) for tag-driven excitations,
  including the rigid-translation motion factor ``n_f . axis``.
* ``BURTON_MILLER_ASSEMBLY = "b200_direct"`` is the new value of the
  ``burton_miller_assembly`` solver option that selects this path
  (the reference accepts ``direct_system`` / ``operator_matrices``,
  ``BeatEngineCompiledDriver.jl:1066-1069``).

Wavenumbers are passed unsigned, as the reference passes them; the phasor
convention is an argument instead of the reference's global.  Errors raise
:class:`~beat_engine_b200._lib.BeatB200Error` (the reference raises through
``error(...)`` into a ``failed`` worker event).
"""
from __future__ import annotations

import time
from typing import Sequence

import numpy as np

from . import _lib
from .mesh import BoundaryMesh
from .phasor import (NEGATIVE_TIME_PHASOR, burton_miller_coupling, neumann_scale, outgoing_wavenumber)

BURTON_MILLER_ASSEMBLY = "b200_direct"
PRECISIONS = {"float64": _lib.FP64, "mixed_fp32_ir": _lib.MIXED_FP32_IR}


class ExteriorB200Cache:
    """Per-mesh device context: the analogue of the reference's
    ``device_cache`` / ``device_singular_cache`` pair built once per request
    (``BeatEngineCompiledDriver.jl:1133-1176``) and reused over frequencies."""

    def __init__(self, mesh: BoundaryMesh, quadrature_order: int = 4, singular_order: int = 4, device: int = 0):
        self.mesh = mesh
        self.quadrature_order = quadrature_order
        self.singular_order = singular_order
        self.ctx = _lib.Context(device)
        self.ctx.set_mesh(mesh.vertices, mesh.faces, quadrature_order, singular_order)

    def close(self):
        self.ctx.close()


def exterior_assembly_selection(options: dict) -> dict:
    """The solver-option checks of ``solve_exterior_request``
    (``BeatEngineCompiledDriver.jl:1055-1076``) with ``b200_direct`` added to
    the allowed ``burton_miller_assembly`` values: ``precision`` float32 or
    float64 (default float32), ``bem_backend`` cpu / cuda / rocm / metal
    (default cpu), ``burton_miller_assembly`` direct_system / operator_matrices
    / b200_direct (default direct_system), all case-insensitive.  This path
    runs when the backend is cuda and the assembly b200_direct; b200_direct on
    another backend is refused.  Violations raise ``ValueError`` with the
    reference's messages (the assembly one lists the new value).  Returns the
    normalised choices, ``b200_assembly`` and, when it is set, the precision
    form of ``b200_precision``."""
    precision_name = str(options.get("precision", "float32")).lower()
    if precision_name not in ("float32", "float64"):
        raise ValueError("Exterior precision must be float32 or float64.")
    backend = str(options.get("bem_backend", "cpu")).lower()
    if backend not in ("cpu", "cuda", "rocm", "metal"):
        raise ValueError("Exterior BEM backend must be cpu, cuda, rocm, or metal.")
    requested = str(options.get("burton_miller_assembly", "direct_system")).lower()
    if requested not in ("direct_system", "operator_matrices", BURTON_MILLER_ASSEMBLY):
        raise ValueError("Exterior burton_miller_assembly must be direct_system, operator_matrices, or "
                         f"{BURTON_MILLER_ASSEMBLY}.")
    b200 = requested == BURTON_MILLER_ASSEMBLY
    if b200 and backend != "cuda":
        raise ValueError(f"Exterior burton_miller_assembly = {BURTON_MILLER_ASSEMBLY} needs bem_backend = cuda.")
    return {"precision": precision_name, "bem_backend": backend, "burton_miller_assembly": requested,
            "b200_assembly": b200, "b200_precision": solver_options_precision(options) if b200 else None}


def solver_options_precision(options: dict) -> int:
    """``b200_precision`` solver option -> precision form (default mixed)."""
    name = str(options.get("b200_precision", "mixed_fp32_ir")).lower()
    if name not in PRECISIONS:
        raise ValueError(f"b200_precision must be one of {sorted(PRECISIONS)}; got {name!r}")
    return PRECISIONS[name]


def solve_exterior_direct_b200(mesh: BoundaryMesh, neumann_values: Sequence[np.ndarray], wavenumber: float, *,
                               cache: ExteriorB200Cache | None = None, precision: str = "mixed_fp32_ir",
                               phasor_convention: str = NEGATIVE_TIME_PHASOR, ir_restart: int = 20,
                               ir_rtol: float = 1e-10, lu_split_terms: int = 3, quadrature_order: int = 4,
                               singular_order: int = 4):
    """Assemble the Burton-Miller system for every excitation, factor once,
    solve all columns.  Returns ``(pressures, assembly_s, solve_s, report)``
    with ``pressures`` a list of length-N complex vectors, like the reference."""
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
    own = cache is None
    if own:
        cache = ExteriorB200Cache(mesh, quadrature_order, singular_order)
    try:
        q = np.stack([np.asarray(v, dtype=np.complex128) for v in neumann_values], axis=1)
        k = outgoing_wavenumber(wavenumber, phasor_convention)
        eta = burton_miller_coupling(wavenumber, phasor_convention).imag
        opts = _lib.Context.opts(PRECISIONS[precision], ir_restart=ir_restart, ir_rtol=ir_rtol,
                                 lu_split_terms=lu_split_terms)
        t0 = time.perf_counter()
        p, diag = cache.ctx.solve(k, eta, q, opts)
        wall = time.perf_counter() - t0
        assembly_s = diag["assembly_ms"] / 1e3
        solve_s = max(wall - assembly_s, 0.0)
        report = dict(diag, burton_miller_assembly=BURTON_MILLER_ASSEMBLY, factorization_count=1,
                      linear_solver="b200_lu" if precision == "float64" else "b200_lu_gmres_ir",
                      b200_precision=precision)
        return [p[:, i].copy() for i in range(p.shape[1])], assembly_s, solve_s, report
    finally:
        if own:
            cache.close()


def evaluate_galerkin_field_b200(points, mesh: BoundaryMesh, pressure, q, wavenumber: float,
                                 cache: ExteriorB200Cache, phasor_convention: str = NEGATIVE_TIME_PHASOR):
    """Pressure at observation points (``M`` or ``M x R``)."""
    k = outgoing_wavenumber(wavenumber, phasor_convention)
    out = cache.ctx.field(k, points, pressure, q)
    return out[:, 0] if np.asarray(pressure).ndim == 1 else out


def evaluate_far_field_b200(directions, mesh: BoundaryMesh, pressure, q, wavenumber: float,
                            cache: ExteriorB200Cache, phasor_convention: str = NEGATIVE_TIME_PHASOR):
    """Far-field pattern ``lim r exp(-i k r) p(r d)`` (no reference counterpart)."""
    k = outgoing_wavenumber(wavenumber, phasor_convention)
    out = cache.ctx.farfield(k, directions, pressure, q)
    return out[:, 0] if np.asarray(pressure).ndim == 1 else out


def rigid_translation_axis(motion_axis, symmetry_mode: str = "off") -> np.ndarray:
    """The unit direction of a rigid-translation source, checked as the
    reference checks it (``prescribed_motion_axis``,
    ``BeatEngineCompiledDriver.jl:728-770``): three finite numbers, not all
    zero, scaled by the largest magnitude and then normalised (an axis gives a
    direction, not a speed), and lying in every active symmetry plane (x: no x
    component; xy: no x or y component) to 1e-8.  Violations raise
    ``ValueError`` with the reference's messages."""
    raw = list(motion_axis) if isinstance(motion_axis, (list, tuple, np.ndarray)) else None
    if raw is None or len(raw) != 3:
        raise ValueError("Rigid-translation source requires a three-component motion_axis.")
    if not all(isinstance(v, (int, float, np.integer, np.floating)) and not isinstance(v, (bool, np.bool_))
               and np.isfinite(v) for v in raw):
        raise ValueError("Rigid-translation source motion_axis must contain three finite numbers.")
    ax = np.asarray(raw, dtype=np.float64)
    scale = float(np.max(np.abs(ax)))
    if not scale > 0.0:
        raise ValueError("Rigid-translation source motion_axis must be finite and nonzero.")
    ax = ax / scale
    ax = ax / np.linalg.norm(ax)
    planes = {"x": (0,), "xy": (0, 1)}.get(str(symmetry_mode).lower(), ())
    if any(abs(ax[c]) > 1e-8 for c in planes):
        raise ValueError("Rigid-translation source motion_axis must lie in the physical symmetry planes.")
    return ax


def exterior_neumann(mesh: BoundaryMesh, tags, amplitudes, density: float, omega: float,
                     phasor_convention: str = NEGATIVE_TIME_PHASOR, motion_axis=None, symmetry_mode: str = "off"):
    """Per-face Neumann data ``q_f = neumann_scale(rho, omega) * amplitude``
    on faces carrying one of ``tags`` (times ``n_f . axis`` for a rigid
    translation, the axis checked and normalised by
    :func:`rigid_translation_axis`), zero elsewhere."""
    values = np.zeros(mesh.num_faces, dtype=np.complex128)
    scale = neumann_scale(density, omega, phasor_convention)
    factor = np.ones(mesh.num_faces)
    if motion_axis is not None:
        factor = mesh.normals @ rigid_translation_axis(motion_axis, symmetry_mode)
    for tag, amp in zip(tags, amplitudes):
        sel = mesh.physical_tags == tag
        values[sel] = scale * amp * factor[sel]
    return values


def bem_normal_velocity_neumann(velocity, density: float, omega: float,
                                phasor_convention: str = NEGATIVE_TIME_PHASOR):
    """``neumann_scale .* motion`` for explicit per-face velocities
    (the ``bem_normal_velocity`` branch of ``exterior_neumann``)."""
    return neumann_scale(density, omega, phasor_convention) * np.asarray(velocity, dtype=np.complex128)
