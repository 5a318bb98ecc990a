"""Phasor convention helpers (``src/BeatEnginePhasor.jl:1-24``).

The reference keeps the active convention in a global; the caller passes it
explicitly here.  ``s = +1`` for ``exp(-i omega t)`` (the reference default) and
``s = -1`` for ``exp(+i omega t)``.
"""
from __future__ import annotations

NEGATIVE_TIME_PHASOR = "exp(-i omega t)"
POSITIVE_TIME_PHASOR = "exp(+i omega t)"


def propagation_sign(convention: str = NEGATIVE_TIME_PHASOR) -> int:
    if convention == NEGATIVE_TIME_PHASOR:
        return 1
    if convention == POSITIVE_TIME_PHASOR:
        return -1
    raise ValueError(f"Unsupported phasor convention: {convention!r}")


def outgoing_wavenumber(k: float, convention: str = NEGATIVE_TIME_PHASOR) -> float:
    """``outgoing_wavenumber(k) = s*|k|``."""
    return propagation_sign(convention) * abs(k)


def neumann_scale(density: float, omega: float, convention: str = NEGATIVE_TIME_PHASOR) -> complex:
    """``neumann_scale(rho, omega) = i*s*rho*omega``: dp/dn per unit normal velocity."""
    return complex(0.0, propagation_sign(convention) * density * omega)


def time_derivative(omega: float, convention: str = NEGATIVE_TIME_PHASOR) -> complex:
    return complex(0.0, -propagation_sign(convention) * omega)


def burton_miller_coupling(k: float, convention: str = NEGATIVE_TIME_PHASOR) -> complex:
    """``eta = i*s/|k|`` (purely imaginary)."""
    return complex(0.0, propagation_sign(convention) / abs(k))
