"""Autotuner of the solve's launch choices, per device and system size.

The choices a sweep exposes (``beat_b200_opts``):

* ``lu_block``: the LU's panel width (64, 128 or 256 columns).  Narrow panels
  shorten each panel's dependent chain but give the trailing updates less
  work per launch; the best width depends on N.
* ``sweep_lanes``: how many frequencies are in flight at once.  More lanes
  overlap one frequency's latency-bound phases (panels, substitutions) with
  other frequencies' SM-filling ones (element pairs, trailing updates), at
  the price of one workspace per lane.

``tune`` measures both on the caller's own context and mesh: every panel width
on one frequency solve (the diagnostics' CUDA-event ``lu_ms``), then every lane
count on a short sweep (wall time of the synchronous sweep call), and keeps the
fastest.  Results are cached in a JSON file keyed by the device name, N, F, R
and the precision form, so a later run with the same key (the same mesh size
on the same GPU model) reads them instead of measuring.  The element-pair
kernel's tile (32 faces, two CTAs per SM) is fixed by its shared-memory
accumulators and is not a tuning choice.
"""
from __future__ import annotations

import json
import os
import time

import numpy as np

from . import _lib

BLOCKS = (64, 128, 256)
LANES = (2, 4, 6, 8)


def default_cache() -> str:
    return os.environ.get("BEAT_B200_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "beat_b200", "autotune.json"))


def device_name(device: int = 0) -> str:
    try:
        import torch
        return torch.cuda.get_device_name(device)
    except Exception:  # torch absent or no device name: key on the ordinal
        return f"cuda:{device}"


def key_of(ctx, R: int, precision: int, device: int = 0) -> str:
    return f"{device_name(device)}|N={ctx.V}|F={ctx.F}|R={R}|precision={precision}"


def _load(path):
    try:
        with open(path, encoding="utf-8") as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _store(path, table):
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tmp = path + f".tmp{os.getpid()}"
    with open(tmp, "w", encoding="utf-8") as fh:
        json.dump(table, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def tune(ctx, k_signed, eta, q, precision: int = _lib.MIXED_FP32_IR, cache: str | None = None,
         blocks=BLOCKS, lanes=LANES, device: int = 0, refresh: bool = False) -> dict:
    """Best ``lu_block`` and ``sweep_lanes`` for this context's mesh with the
    Neumann data ``q`` (F x R) around wavenumber ``k_signed``: read from the
    cache, or measured and stored.  Returns ``{"lu_block", "sweep_lanes",
    "measured", "key", "cached"}``."""
    q = np.asfortranarray(np.asarray(q, dtype=np.complex128).reshape(ctx.F, -1))
    R = q.shape[1]
    path = cache or default_cache()
    key = key_of(ctx, R, precision, device)
    table = _load(path)
    if key in table and not refresh:
        return dict(table[key], key=key, cached=True)
    lu = {}
    for nb in blocks:
        opts = _lib.Context.opts(precision, lu_block=nb)
        try:
            ctx.solve(k_signed, eta, q, opts)  # warm: workspace, first-launch costs
        except _lib.BeatB200Error as e:
            if e.status != _lib.INVALID_ARG:  # a width this size cannot take (its panel outgrows shared memory)
                raise
            continue
        lu[nb] = min(ctx.solve(k_signed, eta, q, opts)[1]["lu_ms"] for _ in range(2))
    if not lu:
        raise ValueError(f"no panel width of {tuple(blocks)} fits this system")
    best_nb = min(lu, key=lu.get)
    fps = {}
    for L in lanes:
        n = 2 * L
        ks = np.asarray(k_signed, dtype=np.float64) * np.linspace(0.9, 1.1, n)
        qs = np.repeat(q[:, :, None], n, axis=2)
        opts = _lib.Context.opts(precision, lu_block=best_nb, sweep_lanes=L)
        etas = eta * float(k_signed) / ks  # the coupling scales as 1 / |k|
        ctx.sweep(ks[:L], etas[:L], qs[:, :, :L], opts)  # creates and sizes the lanes
        t0 = time.perf_counter()
        ctx.sweep(ks, etas, qs, opts)
        fps[L] = n / (time.perf_counter() - t0)
    best_l = max(fps, key=fps.get)
    entry = {"lu_block": int(best_nb), "sweep_lanes": int(best_l),
             "measured": {"lu_ms": {str(a): b for a, b in lu.items()},
                          "sweep_freq_solves_per_s": {str(a): b for a, b in fps.items()}}}
    table = _load(path)  # another process may have written meanwhile
    table[key] = entry
    _store(path, table)
    return dict(entry, key=key, cached=False)


def opts_for(entry: dict, precision: int = _lib.MIXED_FP32_IR, **kw) -> _lib.Opts:
    """Solve options with a tuned entry's panel width and lane count."""
    return _lib.Context.opts(precision, lu_block=entry["lu_block"], sweep_lanes=entry["sweep_lanes"], **kw)
