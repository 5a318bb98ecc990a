"""The right-hand-side policy (beat_b200_rhs_use_operator, restating
exterior_use_rhs_operator, exterior_rhs_policy.jl:15-44) on the CPU: the
reference's own decision table (tests/exterior_rhs_policy_tests.jl:3-21)
with synthetic byte counts.  Pure host logic of the library; no device."""
import pytest

from beat_engine_b200 import _lib

GIB = 1024 ** 3
MATRIX, OPERATOR = 4 * GIB, 8 * GIB


def use(mode, n, matrix=MATRIX, operator=OPERATOR, available=32 * GIB):
    return _lib.use_rhs_operator(mode, n, matrix, operator, available)


def test_reference_decision_table():
    assert use("auto", 60)
    assert use("auto", 2)
    # one excitation has no repeated integration to save
    assert not use("auto", 1)
    assert not use("auto", 0)
    assert not use("matrix_free", 60)
    assert use("cached_operator", 1)
    assert use(" Cached_Operator ", 2)
    # 4 + 8 GiB + 512 MiB = 12.5 GiB
    assert use("auto", 60, available=13 * GIB)
    assert not use("auto", 60, available=12 * GIB)
    assert not use("cached_operator", 60, available=12 * GIB)
    assert not use("auto", 60, operator=0)
    with pytest.raises(ValueError):
        use("fast", 60)
    assert _lib.rhs_mode("MATRIX_FREE") == "matrix_free"


def test_margin_boundary_and_unknown_mode_code():
    lib = _lib.load()
    margin = 512 * 1024 ** 2
    assert lib.beat_b200_rhs_use_operator(_lib.RHS_AUTO, 2, MATRIX, OPERATOR, MATRIX + OPERATOR + margin) == 1
    assert lib.beat_b200_rhs_use_operator(_lib.RHS_AUTO, 2, MATRIX, OPERATOR, MATRIX + OPERATOR + margin - 1) == 0
    assert lib.beat_b200_rhs_use_operator(_lib.RHS_CACHED, 0, MATRIX, OPERATOR, 32 * GIB) == 0
    assert lib.beat_b200_rhs_use_operator(_lib.RHS_AUTO, 2, -1, OPERATOR, 32 * GIB) == 0
    assert lib.beat_b200_rhs_use_operator(7, 2, MATRIX, OPERATOR, 32 * GIB) == -1


def test_flags_for_modes():
    assert _lib.rhs_flags("auto") == 0
    assert _lib.rhs_flags("matrix_free") == _lib.FLAG_RHS_MATRIX_FREE
    assert _lib.rhs_flags("cached_operator") == _lib.FLAG_RHS_CACHED
