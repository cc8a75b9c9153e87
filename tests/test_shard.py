"""Sharded contraction across ranks (one process per GPU in production), on
CPU with world-size-2 gloo process groups: the library plans each rank's slab
of C (host-only), the oracle computes the slab from the matching slices of A
or B, and the library's gather hands every slab to every rank; the result is
the whole contraction on both ranks. The planner's slabs are disjoint and
cover C for every rank count."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CASES = [
    # (idx_A, idx_B, idx_C, lens): the cut label in A and C, in B and C, none
    ("abk", "kc", "acb", {"a": 7, "b": 5, "k": 3, "c": 4}),
    ("ka", "kbc", "cab", {"a": 3, "b": 4, "k": 6, "c": 9}),
    ("k", "k", "", {"k": 11}),
]


def _data(case, seed=0):
    iA, iB, iC, L = CASES[case]
    rng = np.random.default_rng(seed + case)
    A = rng.uniform(-1, 1, [L[c] for c in iA])
    B = rng.uniform(-1, 1, [L[c] for c in iB])
    C = rng.uniform(-1, 1, [L[c] for c in iC])
    return iA, iB, iC, A, B, C


def _slice(X, idx, label, b, e):
    sl = tuple(slice(b, e) if c == label else slice(None) for c in idx)
    return X[sl]


def _worker(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import oracle
    import tblis_b200 as tb
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out = []
        for case in range(len(CASES)):
            iA, iB, iC, A, B, C = _data(case)
            want = C.copy()
            oracle.orc_mult(0.5, A, iA, B, iB, -1.5, want, iC)
            label, b, e = tb.shard_plan(A, iA, B, iB, C, iC, world, rank)
            mine = C.copy()
            if label:
                # this rank's slab from the matching slices
                cs = np.ascontiguousarray(_slice(mine, iC, label, b, e))
                oracle.orc_mult(0.5, np.ascontiguousarray(_slice(A, iA, label, b, e)), iA,
                                np.ascontiguousarray(_slice(B, iB, label, b, e)), iB, -1.5, cs, iC)
                _slice(mine, iC, label, b, e)[...] = cs
            elif e > b:
                oracle.orc_mult(0.5, A, iA, B, iB, -1.5, mine, iC)
            Ct = torch.from_numpy(mine)
            tb.gather_shards(A, iA, B, iB, Ct, iC, rank, world)
            out.append(float(np.max(np.abs(Ct.numpy() - want))))
        dist.barrier()
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def test_two_ranks_assemble_the_whole_contraction():
    import torch.multiprocessing as mp
    port = 29700 + (os.getpid() % 1000)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, errs in res:
        assert all(e <= 1e-13 for e in errs), (rank, errs)


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("nranks", [1, 2, 3, 8, 13])
def test_slabs_are_disjoint_and_cover(case, nranks):
    sys.path.insert(0, ROOT)
    import tblis_b200 as tb
    iA, iB, iC, A, B, C = _data(case)
    plans = [tb.shard_plan(A, iA, B, iB, C, iC, nranks, r) for r in range(nranks)]
    labels = {p[0] for p in plans}
    assert len(labels) == 1                       # every rank cuts the same label
    label = labels.pop()
    if not label:
        assert [p[2] - p[1] for p in plans] == [1] + [0] * (nranks - 1)
        return
    n = C.shape[iC.index(label)]
    cover = np.zeros(n, int)
    for _, b, e in plans:
        cover[b:e] += 1
    assert np.all(cover == 1)
    # the longest label that is in C and exactly one of A and B
    cands = [c for c in iC if (c in iA) != (c in iB)]
    assert n == max(C.shape[iC.index(c)] for c in cands)
