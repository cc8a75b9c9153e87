"""GPU tests of the continuous-batching server: results against the oracle,
each result bit-identical alone and in a mix, HBM-budget admission, batches
overlapping on the device, and a failing request not disturbing others."""
import time

import numpy as np
import pytest

import oracle
from tests.helpers import random_contraction, make_operand, normwise_rel, to_device, view_of

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _requests(torch, cuda, seeds, max_len=10):
    out = []
    for s in seeds:
        rng = np.random.default_rng(s)
        idx_A, idx_B, idx_C, lens = random_contraction(rng, max_len=max_len)
        A = make_operand(idx_A, lens, rng)
        B = make_operand(idx_B, lens, rng)
        C = make_operand(idx_C, lens, rng)
        alpha, beta = float(rng.choice([1.0, 0.5])), float(rng.choice([0.0, 1.0]))
        ref = C[1].copy()
        oracle.orc_mult(alpha, A[1], idx_A, B[1], idx_B, beta, ref, idx_C)
        _, dA = to_device(*A, torch, cuda)
        _, dB = to_device(*B, torch, cuda)
        dCb, dC = to_device(*C, torch, cuda)
        out.append(dict(args=(alpha, dA, idx_A, dB, idx_B, beta, dC, idx_C), ref=ref, Cb=dCb, C=C))
    return out


def test_results_match_oracle(cuda):
    import torch
    import tblis_b200 as tb
    srv = tb.Server(hbm_budget_bytes=8 << 30, slots=4)
    reqs = _requests(torch, cuda, range(8000, 8060))
    ids = [srv.submit(*r["args"]) for r in reqs]
    lats = [srv.wait(i) for i in ids]
    torch.cuda.synchronize()
    for r in reqs:
        got = view_of(r["Cb"].cpu().numpy(), r["C"][1].shape, r["C"][2])
        assert normwise_rel(got, r["ref"]) <= TOL
    st = srv.stats()
    assert st["completed"] == 60 and st["failed"] == 0 and min(lats) >= 0
    srv.close()


def test_same_result_alone_and_in_the_mix(cuda):
    import torch
    import tblis_b200 as tb
    g = torch.Generator(device=cuda)
    g.manual_seed(1)
    A = torch.empty((48, 40, 36), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g)
    B = torch.empty((36, 52, 40), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g)
    C0 = torch.empty((52, 48), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g)
    srv = tb.Server(slots=4)
    alone = C0.clone()
    srv.wait(srv.submit(1.0, A, "abc", B, "cdb", 0.5, alone, "da"))
    others = _requests(torch, cuda, range(9000, 9040))
    mixed = C0.clone()
    ids = [srv.submit(*r["args"]) for r in others[:20]]
    mid = srv.submit(1.0, A, "abc", B, "cdb", 0.5, mixed, "da")
    ids += [srv.submit(*r["args"]) for r in others[20:]]
    srv.wait(mid)
    for i in ids:
        srv.wait(i)
    torch.cuda.synchronize()
    assert torch.equal(alone, mixed)
    srv.close()


def test_budget_admission(cuda):
    import torch
    import tblis_b200 as tb
    # each request holds 3 x 8 MB; a 40 MB budget admits one at a time
    srv = tb.Server(hbm_budget_bytes=40 << 20, slots=4)
    n = 1024
    mats = [(torch.rand((n, n), dtype=torch.float64, device=cuda), torch.rand((n, n), dtype=torch.float64, device=cuda),
             torch.zeros((n, n), dtype=torch.float64, device=cuda)) for _ in range(6)]
    ids = [srv.submit(1.0, a, "ik", b, "kj", 0.0, c, "ij") for a, b, c in mats]
    for i in ids:
        srv.wait(i)
    torch.cuda.synchronize()
    for a, b, c in mats:
        assert torch.allclose(c, a @ b, rtol=1e-12, atol=1e-12)
    st = srv.stats()
    assert st["batches"] == 6 and st["mean_batch"] == 1.0
    big = torch.zeros((2048, 2048), dtype=torch.float64, device=cuda)
    with pytest.raises(tb.TblisError) as e:
        srv.submit(1.0, big, "ik", big, "kj", 0.0, big, "ij")
    assert e.value.code == 7
    srv.close()


def test_batches_overlap_on_device(cuda):
    """Requests arriving while a long batch runs are admitted into another
    slot instead of waiting for it (continuous batching)."""
    import torch
    import tblis_b200 as tb
    srv = tb.Server(slots=4)
    # the small requests (and their references) are built before the long
    # one is submitted, so that they arrive while it still runs
    small = _requests(torch, cuda, range(9500, 9508), max_len=6)
    n = 8192
    a = torch.rand((n, n), dtype=torch.float64, device=cuda)
    b = torch.rand((n, n), dtype=torch.float64, device=cuda)
    c = torch.zeros((n, n), dtype=torch.float64, device=cuda)
    torch.cuda.synchronize()
    big = srv.submit(1.0, a, "ik", b, "kj", 0.0, c, "ij")      # ~40 ms on the GPU
    time.sleep(0.003)
    ids = [srv.submit(*r["args"]) for r in small]
    lat_small = [srv.wait(i) for i in ids]
    lat_big = srv.wait(big)
    torch.cuda.synchronize()
    st = srv.stats()
    assert st["max_concurrent_batches"] >= 2
    for r in small:
        got = view_of(r["Cb"].cpu().numpy(), r["C"][1].shape, r["C"][2])
        assert normwise_rel(got, r["ref"]) <= TOL
    srv.close()


def test_failed_request_is_isolated(cuda):
    import torch
    import tblis_b200 as tb
    srv = tb.Server(slots=2)
    good = _requests(torch, cuda, range(9700, 9705))
    A = torch.ones((3, 4), dtype=torch.float64, device=cuda)
    B = torch.ones((5, 2), dtype=torch.float64, device=cuda)   # k lengths differ: 4 vs 5
    C = torch.ones((3, 2), dtype=torch.float64, device=cuda)
    ids = [srv.submit(*r["args"]) for r in good[:2]]
    bad = srv.submit(1.0, A, "ik", B, "kj", 0.0, C, "ij")
    ids += [srv.submit(*r["args"]) for r in good[2:]]
    with pytest.raises(tb.TblisError):
        srv.wait(bad)
    for i in ids:
        srv.wait(i)
    torch.cuda.synchronize()
    for r in good:
        got = view_of(r["Cb"].cpu().numpy(), r["C"][1].shape, r["C"][2])
        assert normwise_rel(got, r["ref"]) <= TOL
    srv.close()


def test_tolerant_requests_use_int8_slices(cuda):
    """Large requests whose tolerance allows it run as Ozaki INT8 slices: the
    result meets each request's tolerance, is the same alone and in a mix,
    and a zero tolerance keeps the plain FP64 path."""
    import torch
    import tblis_b200 as tb
    g = torch.Generator(device=cuda)
    g.manual_seed(7)
    m, n, k = 1024, 768, 4096
    a = torch.empty((m, k), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g)
    b = torch.empty((k, n), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g)
    exact = a @ b
    srv = tb.Server(slots=3)
    outs = {}
    for tol in (1e-10, 1e-13, 0.0):
        c = torch.zeros((m, n), dtype=torch.float64, device=cuda)
        srv.wait(srv.submit(1.0, a, "ik", b, "kj", 0.0, c, "ij", tolerance=tol))
        outs[tol] = c
    torch.cuda.synchronize()
    assert srv.stats()["ozaki"] == 2
    for tol in (1e-10, 1e-13):
        err = (torch.linalg.norm(outs[tol] - exact)/torch.linalg.norm(exact)).item()
        assert err <= tol
    assert (torch.linalg.norm(outs[0.0] - exact)/torch.linalg.norm(exact)).item() <= 1e-14
    # the same request among small ones
    small = _requests(torch, cuda, range(9800, 9830), max_len=8)
    c = torch.zeros((m, n), dtype=torch.float64, device=cuda)
    ids = [srv.submit(*r["args"]) for r in small[:15]]
    mid = srv.submit(1.0, a, "ik", b, "kj", 0.0, c, "ij", tolerance=1e-13)
    ids += [srv.submit(*r["args"]) for r in small[15:]]
    for i in ids + [mid]:
        srv.wait(i)
    torch.cuda.synchronize()
    assert torch.equal(c, outs[1e-13])
    for r in small:
        got = view_of(r["Cb"].cpu().numpy(), r["C"][1].shape, r["C"][2])
        assert normwise_rel(got, r["ref"]) <= TOL
    assert srv.stats()["ozaki"] == 3
    srv.close()


def test_repeated_shapes_across_batches(cuda):
    """Requests that share a shape (lengths, strides, labels) reuse the
    server's cached view and device scatter vectors: four shapes, each
    submitted in three waves with fresh operands and scalars, every result
    against torch."""
    import torch
    import tblis_b200 as tb
    g = torch.Generator(device=cuda)
    g.manual_seed(12)
    shapes = [((9, 7, 5), "ac", "cb", "ab"), ((33, 17, 40), "ca", "bc", "ba"),
              ((64, 80, 96), "ac", "cb", "ab"), ((5, 130, 3), "ac", "bc", "ba")]
    srv = tb.Server(hbm_budget_bytes=8 << 30, slots=4)
    try:
        for wave in range(3):
            work = []
            for (m, n, k), ia, ib, ic in shapes * 4:
                dims = {"a": m, "b": n, "c": k}
                mk = lambda lab: torch.empty([dims[x] for x in lab], dtype=torch.float64,
                                             device=cuda).uniform_(-1, 1, generator=g)
                A, B, C = mk(ia), mk(ib), mk(ic)
                alpha, beta = 0.5 + wave, (0.0, 1.0, -0.5)[wave]
                want = alpha * torch.einsum("%s,%s->%s" % (ia, ib, ic), A, B) + (beta * C if beta else 0.0)
                rid = srv.submit(alpha, A, ia, B, ib, beta, C, ic, 1e-14)
                work.append((rid, C, want))
            for rid, C, want in work:
                srv.wait(rid)
                err = (torch.linalg.vector_norm(C - want) / torch.linalg.vector_norm(want)).item()
                assert err <= 1e-14, (wave, err)
    finally:
        srv.close()
