"""Sharding clips over ranks (one process per GPU), tested with gloo on CPU.

The imaging engine itself needs a GPU; these tests run the host logic of the
multi-GPU path — the shard plan, the ordered all-gather and the failure of a
rank — with a stand-in per-clip function, two processes, gloo, 127.0.0.1.
"""

from __future__ import annotations

import os
import socket
import tempfile

import numpy as np
import pytest

from lithobat_b200.distributed import clip_cost, gather_results, run_sharded, shard_plan


def test_shard_plan_covers_every_clip_once_and_balances_uneven_sizes():
    rng = np.random.default_rng(0)
    sizes = rng.choice([256, 512, 1024, 2048], size=256, p=[0.4, 0.3, 0.2, 0.1])
    costs = [clip_cost(int(n), 204) for n in sizes]
    for world in (1, 2, 4, 8):
        parts = shard_plan(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) <= 1.05 * (sum(costs) / world) + max(costs)
        assert all(p == sorted(p) for p in parts)
    assert shard_plan(costs, 4) == shard_plan(list(costs), 4)   # deterministic


def test_shard_plan_with_more_ranks_than_clips():
    parts = shard_plan([1.0, 2.0], 4)
    assert sorted(i for p in parts for i in p) == [0, 1]
    assert sum(1 for p in parts if not p) == 2


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir, fail_rank):
    from datetime import timedelta

    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=10))
    try:
        rng = np.random.default_rng(1)
        clips = [rng.random((n, n)) for n in (8, 16, 8, 32, 16, 8, 24)]
        costs = [clip_cost(c.shape[0]) for c in clips]

        def fn(batch):
            if rank == fail_rank:
                raise RuntimeError("injected failure on this rank")
            return [float(c.sum()) * 2.0 for c in batch]

        try:
            mine, res = run_sharded(clips, costs, fn, rank, world)
            full = gather_results(len(clips), mine, res)
            np.save(os.path.join(out_dir, f"rank{rank}.npy"), np.array(full))
        except Exception as e:  # noqa: BLE001 — reported to the parent through a file
            with open(os.path.join(out_dir, f"rank{rank}.err"), "w") as f:
                f.write(type(e).__name__ + ": " + str(e))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:  # noqa: BLE001
            pass


def _spawn(world, fail_rank):
    import torch.multiprocessing as mp
    out = tempfile.mkdtemp()
    mp.start_processes(_worker, args=(world, _free_port(), out, fail_rank), nprocs=world, join=True,
                       start_method="spawn")
    return out


def test_two_ranks_gather_results_in_input_order():
    out = _spawn(2, fail_rank=-1)
    rng = np.random.default_rng(1)
    clips = [rng.random((n, n)) for n in (8, 16, 8, 32, 16, 8, 24)]
    want = np.array([float(c.sum()) * 2.0 for c in clips])
    for r in range(2):
        got = np.load(os.path.join(out, f"rank{r}.npy"))
        np.testing.assert_array_equal(got, want)


def test_a_failing_rank_is_reported_on_every_rank():
    """Rank 1 raises before the exchange: it reports its own error, and rank 0's
    gather ends with an error (peer gone / timeout) instead of hanging."""
    out = _spawn(2, fail_rank=1)
    errs = {r: open(os.path.join(out, f"rank{r}.err")).read() for r in range(2)
            if os.path.exists(os.path.join(out, f"rank{r}.err"))}
    assert "injected failure" in errs.get(1, "")
    assert 0 in errs, "rank 0 must see the failure of rank 1"
    assert not os.path.exists(os.path.join(out, "rank0.npy"))
