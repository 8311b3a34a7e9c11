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


def _elastic_rank(rank, world, port, result_dir, n_batches, per_batch):
    """Rank 1 leaves between batches (announced) after its first batch; rank 2 takes a batch and
    stops before answering it, without a word (its heartbeat goes stale).  Rank 0 stays."""
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
    store = dist.distributed_c10d._get_default_store()
    tr, v = wk.synth_generate(5, seed=0, generator_only=True)
    o = oracle.OracleStore(tr)
    inst = {t: o.get_index(t, wk.IN) for t in range(v["t_org"], v["t_doc"] + 1)}
    qs = workloads.light_queries(v, inst, n_batches * per_batch, seed=9)
    wq = replicas.WorkQueue(store, rank, world, n_batches, stale_s=1.0)
    dist.barrier()   # every rank is in before any leaves
    answered = 0
    while True:
        i = wq.claim()
        if i is None:
            break
        if rank == 2 and answered == 1:
            os._exit(0)   # took batch i and stopped: no answer, no goodbye
        part = qs[i * per_batch:(i + 1) * per_batch]
        rows, st = o.run_many([q.flat() for q in part], [q.nvars for q in part], 1)
        assert (st == 0).all()
        np.save(os.path.join(result_dir, "batch_%d.npy" % i), rows)
        np.save(os.path.join(result_dir, "by_%d_%d.npy" % (i, rank)), np.array([rank]))
        wq.done(i)
        answered += 1
        if rank == 1 and answered == 1:
            wq.leave()   # between batches
            break
        if rank == 0 and answered == 1:
            import time
            time.sleep(0.5)   # let the others take their batches before rank 0 runs on
    np.save(os.path.join(result_dir, "answered_%d.npy" % rank), np.array([answered]))
    if rank == 0:
        import time
        time.sleep(0.2)
    os._exit(0)   # a survivor leaves without a collective the departed ranks would never join


def test_replicas_keep_answering_when_ranks_leave(tmp_path, graph20):
    world, n_batches, per_batch = 3, 9, 20
    mp.spawn(_elastic_rank, args=(world, _free_port(), str(tmp_path), n_batches, per_batch),
             nprocs=world, join=True)
    import oracle
    import workloads
    import wukong_b200 as wk
    tr, v = wk.synth_generate(5, seed=0)
    o = oracle.OracleStore(tr)
    inst = {t: o.get_index(t, wk.IN) for t in range(v["t_org"], v["t_doc"] + 1)}
    qs = workloads.light_queries(v, inst, n_batches * per_batch, seed=9)
    want, _ = o.run_many([q.flat() for q in qs], [q.nvars for q in qs], 1)
    got = np.concatenate([np.load(tmp_path / ("batch_%d.npy" % i)) for i in range(n_batches)])
    assert np.array_equal(got, want)   # every batch answered, once, whoever answered it
    for i in range(n_batches):
        assert len(list(tmp_path.glob("by_%d_*.npy" % i))) == 1
    assert int(np.load(tmp_path / "answered_1.npy")[0]) == 1     # left after one batch
    assert not (tmp_path / "answered_2.npy").exists()             # stopped mid-stream
    assert len(list(tmp_path.glob("by_*_2.npy"))) == 1           # its one answered batch counts
