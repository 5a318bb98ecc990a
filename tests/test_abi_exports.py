"""CPU checks of the C ABI: the library loads, exports every symbol the header
declares, and its host-only entry points behave (no GPU work here)."""
import ctypes
import os
import re

import pytest

from beat_engine_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "beat_b200.h")


def declared_symbols():
    text = open(HEADER, encoding="utf-8").read()
    return sorted(set(re.findall(r"\b(beat_b200_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert sorted(_lib.EXPORTS) == declared_symbols()


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    for name in declared_symbols():
        assert hasattr(L, name), name


def test_abi_version_and_defaults():
    L = _lib.load()
    assert L.beat_b200_abi_version() == 2
    o = _lib.Opts()
    L.beat_b200_default_opts(ctypes.byref(o))
    assert o.precision == _lib.MIXED_FP32_IR and o.ir_restart == 20 and abs(o.ir_rtol - 1e-10) < 1e-20
    assert o.lu_split_terms == 3


def test_null_context_is_rejected():
    L = _lib.load()
    assert L.beat_b200_set_mesh(None, 3, None, 1, None, 4, 4) == _lib.INVALID_ARG
    assert L.beat_b200_last_error(None) == b"null context"
    assert L.beat_b200_device_bytes(None) == 0
    assert L.beat_b200_destroy(None) == _lib.OK


def test_create_without_gpu_reports_no_device():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    assert _lib.load().beat_b200_create(0, ctypes.byref(h)) == _lib.NO_DEVICE


def test_host_marshaling_layouts():
    """The ctypes layer hands the library column-major complex buffers of the
    documented shapes (checked against a stub, no GPU call)."""
    import numpy as np

    seen = []

    class Stub:
        def __getattr__(self, name):
            def f(*args):
                seen.append((name, args))
                return 0
            return f

    c = _lib.Context.__new__(_lib.Context)
    c.lib, c.handle, c.V, c.F = Stub(), ctypes.c_void_p(1), 5, 6
    p, _ = c.solve(1.0, 1.0, np.ones((6, 3), complex))
    assert p.shape == (5, 3) and p.flags["F_CONTIGUOUS"]
    A, b = c.assemble(1.0, 1.0, np.ones((6, 2), complex))
    assert A.shape == (5, 5) and b.shape == (5, 2)
    assert c.field(1.0, np.zeros((4, 3)), np.ones((5, 2), complex), np.ones((6, 2), complex)).shape == (4, 2)
    assert c.farfield(1.0, np.zeros((4, 3)), np.ones(5, complex), np.ones(6, complex)).shape == (4, 1)
    with pytest.raises(ValueError):
        c.solve(1.0, 1.0, np.ones((7, 1), complex))
    assert [s[0] for s in seen] == ["beat_b200_solve", "beat_b200_assemble", "beat_b200_field",
                                    "beat_b200_farfield"]
