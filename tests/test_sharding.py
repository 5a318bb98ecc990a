"""Multi-GPU frequency sweeps (beat_engine_b200.sharding), host logic on the
CPU: the partition, and two gloo ranks (world size 2, spawned processes)
running run_sharded / sweep_sharded with stand-in work.  The in-order gather,
the paired-index check and the every-rank error path are what the GPU runs
rely on; no device is involved."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from beat_engine_b200 import sharding


def test_partition_round_robin_and_cost_balanced():
    assert sharding.partition(7, 2) == [[0, 2, 4, 6], [1, 3, 5]]
    assert sharding.partition(0, 3) == [[], [], []]
    shares = sharding.partition(6, 2, cost=[10, 1, 1, 1, 1, 6])
    loads = [sum([10, 1, 1, 1, 1, 6][i] for i in s) for s in shares]
    assert sorted(i for s in shares for i in s) == list(range(6))
    assert max(loads) - min(loads) <= 2  # LPT puts 10 alone against 6 + the ones
    with pytest.raises(ValueError):
        sharding.partition(3, 0)
    with pytest.raises(ValueError):
        sharding.partition(3, 2, cost=[1, 2])


def test_single_process_runs_everything_in_order():
    out = sharding.run_sharded(5, lambda idx: {i: i * 10 for i in reversed(idx)})
    assert out == [0, 10, 20, 30, 40]


class FakeContext:
    """ctx.sweep stand-in: p and the far field encode the wavenumber."""

    def __init__(self, N=3, M=2):
        self.N, self.M = N, M

    def sweep(self, ks, eta, q, opts=None, dirs=None):
        nf, R = ks.size, q.shape[1]
        p = np.empty((self.N, R, nf), complex)
        ff = np.empty((self.M, R, nf), complex)
        for j, k in enumerate(ks):
            p[:, :, j] = k + 1j * q[0, :, j]
            ff[:, :, j] = -k
        return p, ff, [{"k": float(k)} for k in ks]


def _worker(rank, world, port, outdir, scenario):
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        if scenario == "order":
            res = sharding.run_sharded(9, lambda idx: {i: (i, rank) for i in idx}, cost=[1] * 8 + [20])
            owners = [r for _, r in res]
            result = {"values": [v for v, _ in res], "owners": owners}
        elif scenario == "error":
            def work(idx):
                if rank == 1:
                    raise ValueError("out of device memory (simulated)")
                return {i: i for i in idx}
            try:
                sharding.run_sharded(4, work)
                result = {"raised": None}
            except sharding.ShardError as e:
                result = {"raised": str(e)}
        elif scenario == "duplicate":
            try:
                sharding.run_sharded(4, lambda idx: {0: rank, **{i: i for i in idx}})
                result = {"raised": None}
            except sharding.ShardError as e:
                result = {"raised": str(e)}
        elif scenario == "sweep":
            ks = np.array([3.0, 5.0, 7.0, 11.0, 13.0])
            q = np.zeros((4, 2, 5), complex)
            q[0, :, :] = np.arange(10).reshape(2, 5)
            p, ff, diags = sharding.sweep_sharded(FakeContext(), ks, 1 / ks, q, dirs=np.zeros((2, 3)))
            result = {"p": p.tolist(), "ff": ff.tolist(), "k": [d["k"] for d in diags]}
        np.save(os.path.join(outdir, f"rank{rank}.npy"), np.array([result], dtype=object), allow_pickle=True)
    finally:
        dist.destroy_process_group()


def _run(scenario):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(2, port, d, scenario), nprocs=2, join=True, start_method="spawn")
        return [np.load(os.path.join(d, f"rank{r}.npy"), allow_pickle=True)[0] for r in range(2)]


def test_two_ranks_gather_in_order():
    r0, r1 = _run("order")
    assert r0["values"] == list(range(9)) and r1["values"] == list(range(9))
    # cost 20 goes to rank 0 first, then the unit items fill rank 1 (load 8 < 20)
    assert r0["owners"] == r1["owners"] == [1] * 8 + [0]


def test_a_failing_rank_raises_on_every_rank():
    r0, r1 = _run("error")
    for r in (r0, r1):
        assert r["raised"] is not None and "rank 1" in r["raised"] and "simulated" in r["raised"]


def test_duplicated_index_raises_on_every_rank():
    r0, r1 = _run("duplicate")
    for r in (r0, r1):
        assert r["raised"] is not None and "two results for index 0" in r["raised"]


def test_sweep_sharded_reassembles_frequencies():
    r0, r1 = _run("sweep")
    ks = [3.0, 5.0, 7.0, 11.0, 13.0]
    for r in (r0, r1):
        p = np.array(r["p"])
        assert r["k"] == ks
        assert np.allclose(p[:, :, 2].real, 7.0) and np.allclose(p[0, :, 3].imag, [3, 8])
        assert np.allclose(np.array(r["ff"])[:, :, 4], -13.0)
