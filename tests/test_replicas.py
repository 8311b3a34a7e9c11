"""Replica mode (more than one GPU) host logic, on CPU with the gloo backend.

Each of two ranks answers its own share of one query stream; the shares cover the stream
exactly once, the whole-job time is the maximum over ranks, and the answers gathered in rank
order are the single-process answers.  The per-query work here is the oracle's (CPU) engine
standing in for the device path, which these CPU tests cannot run.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import replicas


def test_shard_covers_everything_once():
    for n in (0, 1, 7, 16384, 16385):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                lo, hi = replicas.shard(n, r, world)
                assert 0 <= lo <= hi <= n
                seen.extend(range(lo, hi))
            assert seen == list(range(n))
    with pytest.raises(ValueError):
        replicas.shard(10, 2, 2)


def test_single_process_needs_no_group():
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.sum_over_ranks(7) == 7


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, result_dir):
    import datetime
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    for p in (os.path.join(root, "wukong-cube_b200"), os.path.join(root, "oracle")):
        sys.path.insert(0, p)
    import oracle
    import workloads
    import wukong_b200 as wk
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        tr, v = wk.synth_generate(5, seed=0)
        g = wk.GStore(tr)
        inst = {t: g.get_index(t, wk.IN) for t in range(v["t_org"], v["t_doc"] + 1)}
        qs = workloads.light_queries(v, inst, 101, seed=9)
        lo, hi = replicas.shard(len(qs), rank, world)
        o = oracle.OracleStore(tr)
        rows, st = o.run_many([q.flat() for q in qs[lo:hi]], [q.nvars for q in qs[lo:hi]], 1)
        np.save(os.path.join(result_dir, "rows_%d.npy" % rank), rows)
        total = replicas.sum_over_ranks(hi - lo)
        slowest = replicas.max_over_ranks(10.0 + rank)
        np.save(os.path.join(result_dir, "agg_%d.npy" % rank), np.array([total, slowest]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_answer_the_stream(tmp_path, graph20):
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    import oracle
    import workloads
    import wukong_b200 as wk
    tr, v = wk.synth_generate(5, seed=0)
    g = wk.GStore(tr)
    inst = {t: g.get_index(t, wk.IN) for t in range(v["t_org"], v["t_doc"] + 1)}
    qs = workloads.light_queries(v, inst, 101, seed=9)
    o = oracle.OracleStore(tr)
    want, _ = o.run_many([q.flat() for q in qs], [q.nvars for q in qs], 1)
    got = np.concatenate([np.load(tmp_path / ("rows_%d.npy" % r)) for r in range(world)])
    assert np.array_equal(got, want)
    for r in range(world):
        total, slowest = np.load(tmp_path / ("agg_%d.npy" % r))
        assert total == len(qs)
        assert slowest == 10.0 + world - 1
