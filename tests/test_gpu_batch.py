"""GPU parity of batched contractions (tblis_b200_tensor_mult_batch: many
small contractions of mixed shapes in one grouped launch) against the
oracle."""
import numpy as np
import pytest

import oracle
from tests.helpers import random_contraction, make_operand, normwise_rel, to_device, view_of

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _batch(cuda, seeds, max_len=9):
    import torch
    import tblis_b200 as tb
    items, refs, outs = [], [], []
    for s in seeds:
        rng = np.random.default_rng(s)
        idx_A, idx_B, idx_C, lens = random_contraction(rng, max_len=max_len)
        A = make_operand(idx_A, lens, rng)
        B = make_operand(idx_B, lens, rng)
        C = make_operand(idx_C, lens, rng)
        alpha, beta = float(rng.choice([1.0, -0.5])), float(rng.choice([0.0, 1.0, 0.25]))
        ref = C[1].copy()
        oracle.orc_mult(alpha, A[1], idx_A, B[1], idx_B, beta, ref, idx_C)
        _, dA = to_device(*A, torch, cuda)
        _, dB = to_device(*B, torch, cuda)
        dCb, dC = to_device(*C, torch, cuda)
        items.append((alpha, dA, idx_A, dB, idx_B, beta, dC, idx_C))
        refs.append(ref)
        outs.append((dCb, C))
    rep = tb.mult_batch(items)
    torch.cuda.synchronize()
    worst = 0.0
    for ref, (dCb, C) in zip(refs, outs):
        got = view_of(dCb.cpu().numpy(), C[1].shape, C[2])
        worst = max(worst, normwise_rel(got, ref))
    return worst, rep


def test_batch_of_mixed_contractions(cuda):
    worst, rep = _batch(cuda, range(5000, 5060))
    assert worst <= TOL
    assert rep["kernels"] >= 1 and rep["m"] >= 1


def test_batch_replay_with_new_data(cuda):
    # same shapes twice (different seeds draw the same shapes only by chance, so
    # reuse the seeds): the second call hits the cached plan and graph
    w1, _ = _batch(cuda, range(6000, 6020))
    w2, rep = _batch(cuda, range(6000, 6020))
    assert w1 <= TOL and w2 <= TOL


def test_batch_of_ladder_like_4index(cuda):
    """4-index ladder-like members (2 labels per group), extents 4..12."""
    import torch
    import tblis_b200 as tb
    rng = np.random.default_rng(77)
    items, refs, outs = [], [], []
    for _ in range(40):
        l = {c: int(rng.integers(4, 13)) for c in "abefij"}
        pa, pb, pc = (list(rng.permutation(4)) for _ in range(3))
        ia = "".join(np.array(list("abef"))[pa])
        ib = "".join(np.array(list("efij"))[pb])
        ic = "".join(np.array(list("abij"))[pc])
        A = rng.uniform(-1, 1, [l[c] for c in ia])
        B = rng.uniform(-1, 1, [l[c] for c in ib])
        C = rng.uniform(-1, 1, [l[c] for c in ic])
        ref = C.copy()
        oracle.orc_mult(1.0, A, ia, B, ib, 1.0, ref, ic)
        dC = torch.from_numpy(C).to(cuda)
        items.append((1.0, torch.from_numpy(A).to(cuda), ia, torch.from_numpy(B).to(cuda), ib, 1.0, dC, ic))
        refs.append(ref)
        outs.append(dC)
    tb.mult_batch(items)
    torch.cuda.synchronize()
    for ref, dC in zip(refs, outs):
        assert normwise_rel(dC.cpu().numpy(), ref) <= TOL


def test_batch_of_1500_4index_members(cuda):
    """1,500 4-index members (extents 8..20, every operand in a random index
    order), tens of thousands of tiles in one grouped launch. Every member
    against numpy's FP64 einsum, a seeded sample against the oracle; run
    twice (the second run replays the plan's graph), beta 1 so that the
    second result holds both runs."""
    import torch
    import tblis_b200 as tb
    rng = np.random.default_rng(2024)
    items, hosts = [], []
    for _ in range(1500):
        l = {c: int(rng.integers(8, 21)) for c in "abefij"}
        ia = "".join(rng.permutation(list("abef")))
        ib = "".join(rng.permutation(list("efij")))
        ic = "".join(rng.permutation(list("abij")))
        A = rng.uniform(-1, 1, [l[c] for c in ia])
        B = rng.uniform(-1, 1, [l[c] for c in ib])
        C = rng.uniform(-1, 1, [l[c] for c in ic])
        items.append((0.5, torch.from_numpy(A).to(cuda), ia, torch.from_numpy(B).to(cuda), ib, 1.0,
                      torch.from_numpy(C).to(cuda), ic))
        hosts.append((A, B, C))
    prepared = tb.PreparedBatch(items)
    prepared.run()
    prepared.run()
    torch.cuda.synchronize()
    sample = set(np.random.default_rng(5).choice(len(items), 25, replace=False).tolist())
    worst = 0.0
    for j, ((_, _, ia, _, ib, _, dC, ic), (A, B, C)) in enumerate(zip(items, hosts)):
        ref = C + 2*0.5*np.einsum("%s,%s->%s" % (ia, ib, ic), A, B, optimize=True)
        got = dC.cpu().numpy()
        worst = max(worst, normwise_rel(got, ref))
        if j in sample:
            want = C.copy()
            oracle.orc_mult(0.5, A, ia, B, ib, 1.0, want, ic)
            oracle.orc_mult(0.5, A, ia, B, ib, 1.0, want, ic)
            assert normwise_rel(got, want) <= TOL
    assert worst <= TOL
