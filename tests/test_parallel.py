"""Multi-process plumbing on CPU (gloo, world size 2): RHS-column shards, the
gather of the receiver traces and the all-reduce of adjoint gradients."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from temf3dt_b200.parallel import assemble_traces, gather_traces, reduce_gradients, shard_range


def test_shard_range_covers_the_columns_once():
    for n in (1, 7, 64, 65):
        for world in (1, 2, 3, 8):
            parts = [shard_range(n, world, r) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[i][1] == parts[i + 1][0] for i in range(world - 1))
            sizes = [hi - lo for lo, hi in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(4, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # 64 sources with one receiver each, sharded by columns
        lo, hi = shard_range(64, world, rank)
        rows = 5
        local = np.zeros((rows, hi - lo, 9))
        for j in range(hi - lo):
            local[:, j, :] = lo + j + 0.01 * np.arange(rows)[:, None]
        parts = gather_traces(local, world)
        full = assemble_traces(parts)
        # per-rank gradient contributions, summed over ranks
        g = reduce_gradients(np.full(10, float(rank + 1)), world)
        out.put((rank, full, g))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_gather_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, full, g in res:
        assert full.shape == (5, 64, 9)
        assert np.allclose(full[0, :, 0], np.arange(64))
        assert np.allclose(g, 3.0)


def _oracle_columns(cols):
    """The CPU oracle's run (src/FETD_FWD.f90:1229-1640 restated) of each RHS
    column of a small multi-source case: the loop, its first half, the loop
    reversed and its second half (the receiver traces, rows x 1 x 9 each)."""
    import dataclasses
    from oracle import fetd_oracle as O
    from tests.golden_cases import synth_oracle_model, tiny_synth
    om = synth_oracle_model(tiny_synth(time_maximum=6e-6))
    se, sd = om.src_edg, om.src_drc
    h = len(se) // 2
    variants = [(se, sd), (se[:h], sd[:h]), (se[::-1], -sd[::-1]), (se[h:], sd[h:])]
    return [O.run_fetd(dataclasses.replace(om, src_edg=variants[k][0], src_drc=variants[k][1])).fields
            for k in cols]


def _oracle_rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        lo, hi = shard_range(4, world, rank)
        local = np.concatenate(_oracle_columns(range(lo, hi)), axis=1)
        out.put((rank, assemble_traces(gather_traces(local, world))))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_oracle_column_shards_equal_one_rank():
    """Two gloo ranks each run the oracle on their shard of four RHS columns
    and gather the receiver traces; the result equals one rank running every
    column (the sharded multi-source path has no per-step exchange)."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    single = np.concatenate(_oracle_columns(range(4)), axis=1)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_oracle_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=600) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, full in res:
        assert full.shape == single.shape
        assert np.array_equal(full, single)
