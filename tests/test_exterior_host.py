"""Host-side mirror of the reference's exterior interface, on the CPU (no GPU).

Neumann data of tag-driven and explicit-velocity excitations
(``exterior_neumann``, BeatEngineCompiledDriver.jl:825-839), the
rigid-translation axis and its checks (``prescribed_motion_axis``,
BeatEngineCompiledDriver.jl:728-770; ``exterior_motion_factor``,
compiled_ground_contract.jl:47-50), the ``b200_precision`` solver option, and
the solver-option checks that select this path
(BeatEngineCompiledDriver.jl:1055-1076 with ``b200_direct`` added).
"""
import numpy as np
import pytest

from beat_engine_b200 import _lib
from beat_engine_b200 import exterior as E
from beat_engine_b200 import mesh as M
from beat_engine_b200.phasor import NEGATIVE_TIME_PHASOR, POSITIVE_TIME_PHASOR, neumann_scale


@pytest.fixture(scope="module")
def tagged_sphere():
    m = M.reference_sphere(0.1, 1)
    tags = np.where(np.asarray(m.normals)[:, 2] > 0.0, 7, 3)  # upper half tag 7, lower half tag 3
    return M.BoundaryMesh(np.asarray(m.vertices), np.asarray(m.faces), tags)


def test_precision_option():
    assert E.solver_options_precision({}) == _lib.MIXED_FP32_IR
    assert E.solver_options_precision({"b200_precision": "float64"}) == _lib.FP64
    assert E.solver_options_precision({"b200_precision": "MIXED_FP32_IR"}) == _lib.MIXED_FP32_IR
    with pytest.raises(ValueError):
        E.solver_options_precision({"b200_precision": "float16"})
    assert E.BURTON_MILLER_ASSEMBLY == "b200_direct"


@pytest.mark.parametrize("convention", [NEGATIVE_TIME_PHASOR, POSITIVE_TIME_PHASOR])
def test_tagged_neumann_values(tagged_sphere, convention):
    m = tagged_sphere
    rho, omega = 1.21, 2 * np.pi * 500.0
    q = E.exterior_neumann(m, [7], [0.5 - 0.25j], rho, omega, convention)
    sel = m.physical_tags == 7
    assert np.all(q[~sel] == 0.0)
    assert np.allclose(q[sel], neumann_scale(rho, omega, convention) * (0.5 - 0.25j), rtol=1e-15, atol=0.0)
    # two tags with their own amplitudes
    q2 = E.exterior_neumann(m, [7, 3], [1.0, 2.0], rho, omega, convention)
    assert np.allclose(q2[sel], neumann_scale(rho, omega, convention))
    assert np.allclose(q2[~sel], 2.0 * neumann_scale(rho, omega, convention))


def test_rigid_translation_factor(tagged_sphere):
    m = tagged_sphere
    rho, omega = 1.21, 2 * np.pi * 2000.0
    q = E.exterior_neumann(m, [7, 3], [1.0, 1.0], rho, omega, motion_axis=[0.0, 0.0, 1.0])
    assert np.allclose(q, neumann_scale(rho, omega) * np.asarray(m.normals)[:, 2], rtol=1e-14, atol=0.0)
    # an axis gives a direction, not a speed: any positive multiple gives the same data
    for axis in ([0.0, 0.0, 5.0], [0.0, 0.0, 1e-200], [0.0, 0.0, 1e200]):
        assert np.allclose(E.exterior_neumann(m, [7, 3], [1.0, 1.0], rho, omega, motion_axis=axis), q,
                           rtol=1e-14, atol=0.0)
    ax = E.rigid_translation_axis([0.0, 3.0, 4.0])
    assert np.allclose(ax, [0.0, 0.6, 0.8], rtol=0, atol=1e-16)


@pytest.mark.parametrize("axis,message", [
    ([0.0, 1.0], "three-component"),
    ("xyz", "three-component"),
    ([0.0, np.nan, 1.0], "three finite numbers"),
    ([0.0, np.inf, 1.0], "three finite numbers"),
    ([True, 0.0, 1.0], "three finite numbers"),
    ([0.0, 0.0, 0.0], "finite and nonzero"),
])
def test_rigid_translation_axis_rejects(axis, message):
    with pytest.raises(ValueError, match=message):
        E.rigid_translation_axis(axis)


def test_rigid_translation_axis_must_lie_in_symmetry_planes():
    assert np.allclose(E.rigid_translation_axis([0.0, 1.0, 1.0], "x"), [0.0, 2 ** -0.5, 2 ** -0.5])
    assert np.allclose(E.rigid_translation_axis([0.0, 0.0, 2.0], "xy"), [0.0, 0.0, 1.0])
    assert np.allclose(E.rigid_translation_axis([1.0, 0.0, 0.0], "ground"), [1.0, 0.0, 0.0])  # no plane check
    for axis, mode in (([1e-3, 0.0, 1.0], "x"), ([0.0, 1e-3, 1.0], "xy"), ([1e-3, 0.0, 1.0], "xy")):
        with pytest.raises(ValueError, match="symmetry planes"):
            E.rigid_translation_axis(axis, mode)
    # within 1e-8 of the plane is accepted
    E.rigid_translation_axis([1e-9, 0.0, 1.0], "x")


def test_explicit_velocity_neumann():
    rho, omega = 1.21, 2 * np.pi * 100.0
    v = np.array([1.0, -2.0 + 0.5j, 0.0])
    assert np.allclose(E.bem_normal_velocity_neumann(v, rho, omega), neumann_scale(rho, omega) * v)
    assert np.allclose(E.bem_normal_velocity_neumann(v, rho, omega, POSITIVE_TIME_PHASOR),
                       neumann_scale(rho, omega, POSITIVE_TIME_PHASOR) * v)


def test_assembly_selection():
    sel = E.exterior_assembly_selection({"bem_backend": "CUDA", "burton_miller_assembly": "B200_direct"})
    assert sel["b200_assembly"] and sel["b200_precision"] == _lib.MIXED_FP32_IR
    assert sel["precision"] == "float32" and sel["bem_backend"] == "cuda"
    sel = E.exterior_assembly_selection({"bem_backend": "cuda", "burton_miller_assembly": "b200_direct",
                                         "b200_precision": "float64", "precision": "float64"})
    assert sel["b200_assembly"] and sel["b200_precision"] == _lib.FP64
    # the reference's own values keep their paths
    for assembly in ("direct_system", "operator_matrices"):
        for backend in ("cpu", "cuda", "rocm", "metal"):
            sel = E.exterior_assembly_selection({"bem_backend": backend, "burton_miller_assembly": assembly})
            assert not sel["b200_assembly"] and sel["b200_precision"] is None
    assert E.exterior_assembly_selection({})["burton_miller_assembly"] == "direct_system"


@pytest.mark.parametrize("options,message", [
    ({"precision": "float16"}, "precision must be float32 or float64"),
    ({"bem_backend": "opencl"}, "backend must be cpu, cuda, rocm, or metal"),
    ({"burton_miller_assembly": "hmatrix"}, "must be direct_system, operator_matrices, or b200_direct"),
    ({"burton_miller_assembly": "b200_direct"}, "needs bem_backend = cuda"),
    ({"burton_miller_assembly": "b200_direct", "bem_backend": "metal"}, "needs bem_backend = cuda"),
    ({"burton_miller_assembly": "b200_direct", "bem_backend": "cuda", "b200_precision": "bf16"}, "b200_precision"),
])
def test_assembly_selection_rejects(options, message):
    with pytest.raises(ValueError, match=message):
        E.exterior_assembly_selection(options)


def test_symmetry_mode_names():
    assert _lib.symmetry_mode(" XY ") == 2 and _lib.symmetry_mode("Ground") == 3 and _lib.symmetry_mode("off") == 0
    assert _lib.symmetry_mode(1) == 1
    with pytest.raises(ValueError, match="Unsupported image mode: yz. Expected off, x, xy, or ground."):
        _lib.symmetry_mode("yz")
