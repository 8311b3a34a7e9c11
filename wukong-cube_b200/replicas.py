"""Replica mode on more than one GPU.

Queries are independent and the whole store fits one GPU, so N GPUs run N replicas: one
process per GPU, each holding the full store and answering its own contiguous share of the
query stream.  There is no collective on the data path; the only collective is the reduction of
each rank's device time to the maximum over ranks (whole-job time), and a gather of per-rank
counts where a caller wants them.  (The reference's multi-server mode partitions vertices and
ships rows between servers per step, sparql.hpp:741-808; on one node that exchange buys
nothing while every GPU can hold the whole graph.)
"""
import time

import torch
import torch.distributed as dist


def shard(n_items, rank, world):
    """Contiguous [lo, hi) share of n_items for `rank`; shares differ by at most one item."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d of %d" % (rank, world))
    base, extra = divmod(n_items, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def max_over_ranks(value, device="cpu"):
    """The maximum of a per-rank float over all ranks (the rank's own value without a group)."""
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, device="cpu"):
    """The sum of a per-rank integer over all ranks."""
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return int(value)
    t = torch.tensor([int(value)], dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return int(t.item())


class WorkQueue:
    """A query stream cut into batches, answered by replicas that may leave between batches.

    The batches are handed out through the process group's key-value store (the c10d store
    every rank already holds), not through a collective, so a rank that leaves costs the others
    nothing but its unfinished work:

    - `claim()` takes the next batch from a shared counter (store.add), so every batch goes to
      exactly one rank while all ranks stay;
    - `done(i)` records batch i as answered; `beat()` is the rank's heartbeat, written after
      every batch; `leave()` announces that the rank stops (between batches);
    - once the counter runs past the last batch, `claim()` looks for batches that were claimed
      but never recorded done by a rank that has left (announced, or silent for longer than
      `stale_s`) and re-claims each one for exactly one surviving rank (a second store.add on a
      per-batch key).

    A rank keeps answering until `claim()` returns None: every batch has then been answered by
    some rank, or is held by a rank that is still alive.  Results are keyed by batch, so which
    rank answered a batch does not change the stream's answers.  The store lives with rank 0
    (the rendezvous host), so rank 0 is the one rank that must stay.
    """

    def __init__(self, store, rank, world, n_batches, stale_s=5.0, prefix="wq"):
        self.store, self.rank, self.world = store, rank, world
        self.n, self.stale_s, self.p = n_batches, stale_s, prefix
        self._unowned_since = {}   # batch -> when this rank first saw it counted but unowned
        self.beat()

    def _k(self, *parts):
        return "/".join((self.p,) + tuple(str(x) for x in parts))

    def _has(self, key):
        return self.store.check([key])

    def beat(self):
        self.store.set(self._k("hb", self.rank), repr(time.time()))

    def leave(self):
        self.store.set(self._k("left", self.rank), "1")

    def done(self, i):
        self.store.set(self._k("done", i), str(self.rank))
        self.beat()

    def gone(self, r):
        """Has rank r left: announced, or no heartbeat for longer than stale_s?"""
        if r == self.rank:
            return False
        if self._has(self._k("left", r)):
            return True
        if not self._has(self._k("hb", r)):
            return False
        return time.time() - float(self.store.get(self._k("hb", r)).decode()) > self.stale_s

    def claim(self):
        """The next batch this rank answers, or None when nothing is left for it."""
        i = self.store.add(self._k("next"), 1) - 1
        if i < self.n:
            self.store.set(self._k("owner", i), str(self.rank))
            return i
        while True:
            waiting = False
            for j in range(self.n):
                if self._has(self._k("done", j)):
                    continue
                if not self._has(self._k("owner", j)):
                    # counted out a moment ago and its taker is about to record itself; a taker
                    # that left in between leaves it unowned for good, and after stale_s it is
                    # retaken like a departed rank's batch
                    t0 = self._unowned_since.setdefault(j, time.time())
                    if time.time() - t0 <= self.stale_s:
                        waiting = True
                        continue
                    owner = -1
                else:
                    owner = int(self.store.get(self._k("owner", j)).decode())
                if owner == self.rank:
                    continue
                if owner >= 0 and not self.gone(owner):
                    waiting = True
                    continue
                # a departed rank held batch j: the first survivor to ask takes it over
                if self.store.add(self._k("retake", j, owner), 1) == 1:
                    self.store.set(self._k("owner", j), str(self.rank))
                    return j
            if not waiting:
                return None
            self.beat()
            time.sleep(0.05)
