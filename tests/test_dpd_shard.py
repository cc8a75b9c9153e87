"""A DPD contraction split across ranks (tblis_b200_dpd_shard_plan /
tblis_b200_dpd_mult_shard / dpd_gather_shards), on CPU: the plan is host-only,
so world-size-2 gloo ranks plan, the reference computes the contraction, each
rank keeps only its blocks, and the library's gather hands every rank the
whole C. The units (row bands of the irrep GEMMs) cover every stored block
of C exactly once and balance the FLOPs."""
import os
import sys

import numpy as np
import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
needs_ref = pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built")

VIR = [6, 2, 4, 3, 5, 1, 4, 3]
OCC = [2, 1, 2, 1, 2, 1, 1, 1]
CASES = [
    # (labels, lengths per label, irreps of A, B, C)
    (("abef", "efij", "abij"), {"a": VIR, "b": VIR, "e": VIR, "f": VIR, "i": OCC, "j": OCC}, (0, 0, 0)),
    (("aeim", "mbej", "aibj"), {"a": VIR, "b": VIR, "e": VIR, "i": OCC, "j": OCC, "m": OCC}, (1, 1, 0)),
    (("abz", "bcz", "acz"), {"a": VIR, "b": OCC, "c": VIR, "z": [1, 2, 1, 1, 2, 1, 1, 1]}, (0, 0, 0)),
]


def _reference(irr, T, data, labels, alpha, beta):
    """The reference's DPD contraction through its FULL path (dense round
    trip), which agrees with its default path without batch labels and, with
    them, with its BLOCKED path and the mathematics (tests/test_gpu_dpd_abc.py)."""
    (A, B, C), (a, b, c), (iA, iB, iC) = T, data, labels
    want = c.copy()
    batch = any(x in iB and x in iC for x in iA)
    old = oracle.ref_dpd_impl(2 if batch else 0)
    try:
        oracle.ref_dpd_mult(8, alpha, irr[0], A.lens, a, iA, irr[1], B.lens, b, iB, beta, irr[2], C.lens, want, iC)
    finally:
        oracle.ref_dpd_impl(old)
    return want


def _tensors(case, seed=0):
    sys.path.insert(0, ROOT)
    import tblis_b200 as tb
    (iA, iB, iC), L, irr = CASES[case]
    T = [tb.DpdTensor(r, 8, [L[c] for c in ix]) for r, ix in zip(irr, (iA, iB, iC))]
    rng = np.random.default_rng(seed + case)
    data = [rng.uniform(-1, 1, t.size()) for t in T]
    return (iA, iB, iC), irr, T, data


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("nranks", [1, 2, 3, 8, 13])
def test_units_cover_once_and_balance(case, nranks):
    import tblis_b200 as tb
    (iA, iB, iC), irr, (A, B, C), _ = _tensors(case)
    owner, flops = tb.dpd_shard_plan(A, iA, B, iB, C, iC, nranks)
    # every stored block of C (non-empty or not) appears once, with a valid rank
    n, nd = 8, len(iC)
    stored = 0
    for t in np.ndindex(*([n] * nd)):
        x = 0
        for v in t:
            x ^= v
        stored += x == irr[2]
    assert len(owner) == stored
    assert all(0 <= r < nranks for r in owner.values())
    # every rank derives the same split; the largest share is close to the mean
    assert tb.dpd_shard_plan(A, iA, B, iB, C, iC, nranks) == (owner, flops)
    if nranks <= 3:
        assert max(flops) <= 1.2 * sum(flops) / nranks


def _worker(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import tblis_b200 as tb
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out = []
        for case in range(len(CASES)):
            (iA, iB, iC), irr, (A, B, C), (a, b, c) = _tensors(case)
            want = _reference(irr, (A, B, C), (a, b, c), (iA, iB, iC), 0.5, -1.5)
            # this rank's share: its blocks from the reference, the rest as before
            owner, _ = tb.dpd_shard_plan(A, iA, B, iB, C, iC, world)
            mine = c.copy()
            for t, r in owner.items():
                if r != rank:
                    continue
                off, Ls, S = C.block(t)
                if np.prod(Ls) == 0:
                    continue
                idx = off + (np.asarray(S)[:, None] * np.indices(Ls).reshape(len(Ls), -1)).sum(0)
                mine[idx] = want[idx]
            C.data = torch.from_numpy(mine)
            tb.dpd_gather_shards(A, iA, B, iB, C, iC, rank, world)
            out.append(float(np.max(np.abs(C.data.numpy() - want))))
        dist.barrier()
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


@needs_ref
def test_two_ranks_assemble_the_whole_contraction():
    import torch.multiprocessing as mp
    port = 29300 + (os.getpid() % 1000)
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
        assert all(e == 0.0 for e in errs), (rank, errs)
