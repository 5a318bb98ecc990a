"""The autotuner's selection and cache (beat_engine_b200.autotune), on the
host with a stand-in context whose costs are known: the fastest panel width
and lane count win, the result is stored under the device / size / precision
key, and a second call reads it without measuring.  The measurement on a
real context runs in the GPU test at the end."""
import time

import numpy as np
import pytest

from beat_engine_b200 import _lib, autotune


class FakeContext:
    V, F = 100, 196

    def __init__(self):
        self.calls = 0

    def solve(self, k, eta, q, opts):
        self.calls += 1
        if opts.lu_block == 256:  # a width the library refuses for this size
            raise _lib.BeatB200Error(_lib.INVALID_ARG, "panel outgrows shared memory")
        return None, {"lu_ms": {64: 3.0, 128: 2.0}[opts.lu_block]}

    def sweep(self, ks, etas, qs, opts):
        self.calls += 1
        assert len(ks) == len(etas) == qs.shape[2]
        time.sleep(0.002 * len(ks) / {2: 1.0, 4: 3.0, 6: 2.0, 8: 1.5}[opts.sweep_lanes])


def test_tune_picks_the_fastest_and_caches(tmp_path):
    ctx = FakeContext()
    q = np.ones((ctx.F, 3), complex)
    cache = str(tmp_path / "tune.json")
    e = autotune.tune(ctx, 20.0, 0.05, q, cache=cache, device=0)
    assert (e["lu_block"], e["sweep_lanes"], e["cached"]) == (128, 4, False)
    assert "N=100|F=196|R=3" in e["key"]
    n = ctx.calls
    e2 = autotune.tune(ctx, 20.0, 0.05, q, cache=cache, device=0)
    assert e2["cached"] and ctx.calls == n and e2["lu_block"] == 128
    o = autotune.opts_for(e2, _lib.FP64)
    assert (o.precision, o.lu_block, o.sweep_lanes) == (_lib.FP64, 128, 4)


@pytest.mark.gpu
def test_tune_on_a_context(tmp_path):
    from beat_engine_b200 import mesh as M
    m = M.reference_sphere(0.1, 3)
    rng = np.random.default_rng(1)
    q = rng.standard_normal((m.num_faces, 2)) + 1j * rng.standard_normal((m.num_faces, 2))
    with _lib.Context(0) as c:
        c.set_mesh(m.vertices, m.faces, 4, 4)
        e = autotune.tune(c, 30.0, 1 / 30.0, q, cache=str(tmp_path / "t.json"), lanes=(2, 4))
        assert e["lu_block"] in autotune.BLOCKS and e["sweep_lanes"] in (2, 4)
        p, d = c.solve(30.0, 1 / 30.0, q, autotune.opts_for(e))
        assert d["lu_block"] == e["lu_block"] and d["ir_converged"] == 1
