"""GPU parity: tblis_tensor_mult (FP64 DMMA block-scatter path) against the
oracle on the same seeded inputs. Tolerance: plain FP64 at most 1e-13
normwise relative error (the north-star bound for the plain path)."""
import numpy as np
import pytest

import oracle
from tests.helpers import (random_contraction, make_operand, normwise_rel, to_device, view_of,
                           random_tensor, strided_empty)

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _run_gpu(torch, dev, alpha, A, idx_A, B, idx_B, beta, C, idx_C, method=0):
    import tblis_b200 as tb
    (Ab, Av, As), (Bb, Bv, Bs), (Cb, Cv, Cs) = A, B, C
    _, dA = to_device(Ab, Av, As, torch, dev)
    _, dB = to_device(Bb, Bv, Bs, torch, dev)
    dCb, dC = to_device(Cb, Cv, Cs, torch, dev)
    if method:
        rep = tb.mult_ex(alpha, dA, idx_A, dB, idx_B, beta, dC, idx_C, method=method)
    else:
        tb.mult(alpha, dA, idx_A, dB, idx_B, beta, dC, idx_C)
        rep = None
    torch.cuda.synchronize()
    out = dCb.cpu().numpy()
    return view_of(out, Cv.shape, Cs), rep


@pytest.mark.parametrize("seed", range(40))
def test_random_contractions_match_oracle(cuda, seed):
    import torch
    rng = np.random.default_rng(1000 + seed)
    idx_A, idx_B, idx_C, lens = random_contraction(rng)
    A = make_operand(idx_A, lens, rng)
    B = make_operand(idx_B, lens, rng)
    C = make_operand(idx_C, lens, rng)
    alpha, beta = float(rng.choice([1.0, 0.5, -2.0])), float(rng.choice([0.0, 1.0, 0.75]))
    ref = C[1].copy()
    oracle.orc_mult(alpha, A[1], idx_A, B[1], idx_B, beta, ref, idx_C)
    got, _ = _run_gpu(torch, cuda, alpha, A, idx_A, B, idx_B, beta, C, idx_C)
    assert normwise_rel(got, ref) <= TOL, (idx_A, idx_B, idx_C, lens)


@pytest.mark.parametrize("seed", range(8))
def test_larger_contractions_match_reference(cuda, seed):
    """Bigger extents (multi-tile, split-K, batch dims), against the reference
    library itself when it was built, else the oracle."""
    import torch
    rng = np.random.default_rng(77 + seed)
    idx_A, idx_B, idx_C, lens = random_contraction(rng, max_len=23, max_labels=(2, 2, 2, 1))
    A = make_operand(idx_A, lens, rng)
    B = make_operand(idx_B, lens, rng)
    C = make_operand(idx_C, lens, rng)
    ref = C[1].copy()
    if oracle.have_ref():
        oracle.ref_mult(1.0, A[1], idx_A, B[1], idx_B, 1.0, ref, idx_C, threads=4)
    else:
        oracle.orc_mult(1.0, A[1], idx_A, B[1], idx_B, 1.0, ref, idx_C)
    got, _ = _run_gpu(torch, cuda, 1.0, A, idx_A, B, idx_B, 1.0, C, idx_C)
    assert normwise_rel(got, ref) <= TOL


def test_dense_24_column_major(cuda):
    """C[abij] = A[abef]*B[efij], every extent 24, column-major (the plain
    dense workload at full size)."""
    import torch
    rng = np.random.default_rng(1)
    shp = [24, 24, 24, 24]
    A = random_tensor(shp, rng)
    B = random_tensor(shp, rng)
    C = random_tensor(shp, rng)
    ref = C[1].copy()
    oracle.orc_mult(1.0, A[1], "abef", B[1], "efij", 0.0, ref, "abij")
    got, rep = _run_gpu(torch, cuda, 1.0, A, "abef", B, "efij", 0.0, C, "abij", method=1)
    assert normwise_rel(got, ref) <= TOL
    assert rep["m"] == 576 and rep["n"] == 576 and rep["k"] == 576 and rep["kernels"] >= 1


def test_ring_small_exact(cuda):
    """C[aibj] += A[aeim]*B[mbej] in its permuted layouts at o=8, v=24."""
    import torch
    rng = np.random.default_rng(2)
    o, v = 8, 24
    A = random_tensor([v, v, o, o], rng)
    B = random_tensor([o, v, v, o], rng)
    C = random_tensor([v, o, v, o], rng)
    ref = C[1].copy()
    oracle.orc_mult(1.0, A[1], "aeim", B[1], "mbej", 1.0, ref, "aibj")
    got, _ = _run_gpu(torch, cuda, 1.0, A, "aeim", B, "mbej", 1.0, C, "aibj")
    assert normwise_rel(got, ref) <= TOL


def _sampled_check(torch, cuda, idx_A, idx_B, idx_C, shpA, shpB, shpC, beta, seed, nsample=400):
    """Full-size contraction on the GPU; a seeded sample of C entries checked
    against the oracle (relative to the sampled entries' norm)."""
    import tblis_b200 as tb
    g = torch.Generator(device=cuda)
    g.manual_seed(seed)
    # column-major storage in the given label order
    def colmajor(shape):
        t = torch.empty(list(reversed(shape)), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g)
        return t.permute(*reversed(range(len(shape))))
    A = colmajor(shpA)
    B = colmajor(shpB)
    C = colmajor(shpC)
    C0 = C.clone()
    tb.mult(1.0, A, idx_A, B, idx_B, beta, C, idx_C)
    torch.cuda.synchronize()
    rng = np.random.default_rng(seed)
    samp = np.stack([rng.integers(0, s, nsample) for s in shpC], axis=1)
    got = C[tuple(torch.from_numpy(samp[:, d]).to(cuda) for d in range(len(shpC)))].cpu().numpy()
    An = A.cpu().numpy()
    Bn = B.cpu().numpy()
    C0n = C0.cpu().numpy()
    want = oracle.orc_mult_sample(1.0, An, idx_A, Bn, idx_B, beta, C0n, idx_C, samp)
    return normwise_rel(got, want)


def test_ring_full_size_sampled(cuda):
    """C[aibj] += A[aeim]*B[mbej], o=64, v=256 (2.15 GB per operand)."""
    import torch
    o, v = 64, 256
    err = _sampled_check(torch, cuda, "aeim", "mbej", "aibj", [v, v, o, o], [o, v, v, o], [v, o, v, o],
                         1.0, seed=5)
    assert err <= TOL


def test_ladder_full_size_sampled(cuda):
    """C[abij] = A[abef]*B[efij], o=48, v=160."""
    import torch
    o, v = 48, 160
    err = _sampled_check(torch, cuda, "abef", "efij", "abij", [v, v, v, v], [v, v, o, o], [v, v, o, o],
                         0.0, seed=6)
    assert err <= TOL


def test_host_pointers_are_staged(cuda):
    """numpy (host) operands go through the same GPU path via staging."""
    import tblis_b200 as tb
    rng = np.random.default_rng(3)
    _, A, _ = random_tensor([7, 9, 5], rng, [2, 0, 1], pad=1)
    _, B, _ = random_tensor([5, 11, 9], rng, [1, 2, 0])
    Cb, C, _ = random_tensor([11, 7], rng, [1, 0], pad=2)
    ref = C.copy()
    oracle.orc_mult(0.5, A, "abc", B, "cdb", 0.25, ref, "da")
    before = tb.kernel_count()
    tb.mult(0.5, A, "abc", B, "cdb", 0.25, C, "da")
    assert tb.kernel_count() > before
    assert normwise_rel(C, ref) <= TOL


def test_beta_zero_never_reads_c(cuda):
    import torch
    import tblis_b200 as tb
    rng = np.random.default_rng(4)
    A = torch.from_numpy(rng.uniform(-1, 1, (33, 17))).to(cuda)
    B = torch.from_numpy(rng.uniform(-1, 1, (17, 45))).to(cuda)
    C = torch.full((33, 45), float("nan"), dtype=torch.float64, device=cuda)
    tb.mult(1.0, A, "ik", B, "kj", 0.0, C, "ij")
    torch.cuda.synchronize()
    assert torch.isfinite(C).all()
    ref = A.cpu().numpy() @ B.cpu().numpy()
    assert normwise_rel(C.cpu().numpy(), ref) <= TOL


def test_alpha_zero_and_empty_k(cuda):
    import torch
    import tblis_b200 as tb
    rng = np.random.default_rng(5)
    A = torch.from_numpy(rng.uniform(-1, 1, (6, 4))).to(cuda)
    B = torch.from_numpy(rng.uniform(-1, 1, (4, 5))).to(cuda)
    C0 = torch.from_numpy(rng.uniform(-1, 1, (6, 5))).to(cuda)
    C = C0.clone()
    tb.mult(0.0, A, "ik", B, "kj", 2.0, C, "ij")
    torch.cuda.synchronize()
    assert torch.allclose(C, 2.0 * C0, rtol=0, atol=0)
    # zero-length contracted index => C = beta*C
    Ae = torch.empty((6, 0), dtype=torch.float64, device=cuda)
    Be = torch.empty((0, 5), dtype=torch.float64, device=cuda)
    C = C0.clone()
    tb.mult(1.0, Ae, "ik", Be, "kj", 0.5, C, "ij")
    torch.cuda.synchronize()
    assert torch.allclose(C, 0.5 * C0, rtol=0, atol=0)
    # zero-length output index => nothing happens
    Ce = torch.empty((0, 5), dtype=torch.float64, device=cuda)
    tb.mult(1.0, A[:0], "ik", B, "kj", 0.5, Ce, "ij")


def test_side_effects_on_c_scalar(cuda):
    """C's scalar is reset to 1 and conj to 0 after the call
    (src/iface/3t/mult.cxx:162-163)."""
    import torch
    import tblis_b200 as tb
    A = torch.ones((3, 4), dtype=torch.float64, device=cuda)
    B = torch.ones((4, 2), dtype=torch.float64, device=cuda)
    C = torch.ones((3, 2), dtype=torch.float64, device=cuda)
    a, b, c = tb._View(A, 1.0), tb._View(B), tb._View(C, 3.0)
    tb.lib.tblis_tensor_mult(None, None, a.ref, b"ik", b.ref, b"kj", c.ref, b"ij")
    tb._check()
    assert c.t.scalar.data[0] == 1.0 and c.t.conj == 0
    torch.cuda.synchronize()
    assert torch.all(C == 7.0)


def test_bad_labels_raise(cuda):
    import torch
    import tblis_b200 as tb
    A = torch.ones((3, 4), dtype=torch.float64, device=cuda)
    B = torch.ones((4, 2), dtype=torch.float64, device=cuda)
    C = torch.ones((3, 2), dtype=torch.float64, device=cuda)
    with pytest.raises(tb.TblisError):
        tb.mult(1.0, A, "ik", B, "kj", 0.0, C, "iz")
    B5 = torch.ones((5, 2), dtype=torch.float64, device=cuda)
    with pytest.raises(tb.TblisError):
        tb.mult(1.0, A, "ik", B5, "kj", 0.0, C, "ij")  # mismatched k lengths


@pytest.mark.parametrize("method,tol", [(1, 1e-13), (2, 1e-12)])
def test_large_host_operand_pipelined(cuda, method, tol):
    """A host-resident A of 800 MB is copied in slabs overlapped with the
    contraction of the slabs already on the device, and C's slabs go back as
    they finish; the result matches the device-resident call (FP64) or meets
    the tolerance (Ozaki). Two layouts: slabs of one contiguous block each
    (a outermost) and slabs of 10^4 pitched rows (e, f outermost)."""
    import torch
    import tblis_b200 as tb
    v, o = 100, 8
    g = torch.Generator(device=cuda)
    g.manual_seed(3)
    dA = torch.empty((v, v, v, v), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g)
    dB = torch.empty((v, v, o, o), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g)
    dC = torch.zeros((v, v, o, o), dtype=torch.float64, device=cuda)
    tb.mult_ex(1.0, dA, "abef", dB, "efij", 0.0, dC, "abij", method=1)
    torch.cuda.synchronize()
    want = dC.cpu()
    hA = dA.cpu().pin_memory()
    hB = dB.cpu()
    # the same tensor stored with its rows (a, b) fastest: row chunks overlap
    for A, lab in ((hA, "abef"), (hA.permute(2, 3, 0, 1).contiguous(), "efab")):
        C = torch.full((v, v, o, o), 7.0, dtype=torch.float64)
        rep = tb.mult_ex(1.0, A, lab, hB, "efij", 0.0, C, "abij", method=method, tolerance=tol)
        err = (torch.linalg.norm(C - want) / torch.linalg.norm(want)).item()
        assert err <= tol, (lab, err, rep)
    del dA, dB, dC
    torch.cuda.empty_cache()


@pytest.mark.parametrize("method, tol", [(1, 1e-14), (2, 1e-12)])
def test_large_host_operand_k_slices(cuda, method, tol):
    """A host-resident A (1000 x 100000, 800 MB, a fastest) whose C label
    would give slab rows of 4000 bytes: it is copied in slices of the
    contracted label instead, each slice accumulating into C."""
    import torch
    import tblis_b200 as tb
    m, k, n = 1000, 100000, 24
    g = torch.Generator(device=cuda)
    g.manual_seed(8)
    dA = torch.empty((k, m), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g).t()
    dB = torch.empty((k, n), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g)
    dC = torch.empty((n, m), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g).t()
    want = dC.clone()
    tb.mult_ex(1.0, dA, "ak", dB, "kb", 0.5, want, "ab", method=1)
    torch.cuda.synchronize()
    want = want.cpu()
    hA = dA.t().cpu().pin_memory().t()
    C = dC.t().cpu().t()
    rep = tb.mult_ex(1.0, hA, "ak", dB.cpu(), "kb", 0.5, C, "ab", method=method, tolerance=tol)
    err = (torch.linalg.norm(C - want) / torch.linalg.norm(want)).item()
    assert err <= tol, (err, rep)
