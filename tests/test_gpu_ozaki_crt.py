"""GPU parity of Ozaki scheme II (method 6, and method 2 when it picks it):
FP64 contractions from one INT8 GEMM per pairwise-coprime modulus and the
Chinese remainder theorem. The residues, the modular GEMMs and the
reconstruction are exact, so the only error is the rounding of the scaled
operands to integers: the normwise error against the FP64 oracle must stay
within the tolerance (moduli count chosen per call) or within four times the
a-priori estimate the call reports."""
import numpy as np
import pytest

import oracle
from tests.helpers import random_contraction, make_operand, normwise_rel, to_device, view_of

pytestmark = pytest.mark.gpu


def _spread(rng, shape, lo=-20, hi=20):
    return rng.uniform(-1, 1, shape) * np.ldexp(1.0, rng.integers(lo, hi + 1, shape))


def _run(torch, dev, method, alpha, A, idx_A, B, idx_B, beta, C, idx_C, slices=0, tol=1e-12):
    import tblis_b200 as tb
    dA = torch.from_numpy(np.ascontiguousarray(A)).to(dev)
    dB = torch.from_numpy(np.ascontiguousarray(B)).to(dev)
    dC = torch.from_numpy(np.ascontiguousarray(C)).to(dev)
    rep = tb.mult_ex(alpha, dA, idx_A, dB, idx_B, beta, dC, idx_C, method=method, slices=slices, tolerance=tol)
    tb.synchronize()     # raises if a kernel gave up a bounded wait
    return dC.cpu().numpy(), rep


@pytest.mark.parametrize("nm", [3, 6, 9, 12, 13, 16])
def test_error_within_estimate_for_each_moduli_count(cuda, nm):
    import torch
    rng = np.random.default_rng(nm)
    A = _spread(rng, (300, 1000), -8, 8)
    B = _spread(rng, (1000, 290), -8, 8)
    C = rng.uniform(-1, 1, (300, 290))
    ref = C.copy()
    oracle.orc_mult(1.0, A, "ik", B, "kj", 0.5, ref, "ij")
    got, rep = _run(torch, cuda, 6, 1.0, A, "ik", B, "kj", 0.5, C, "ij", slices=nm)
    err = normwise_rel(got, ref)
    assert rep["method"] == 6 and rep["slices"] == nm
    assert err <= 4 * rep["est_error"] + 1e-15, (nm, err, rep["est_error"])


def test_ladder_shape_meets_1e12(cuda):
    """The ladder's input distribution at a reduced size (o=8, v=24); the
    moduli count chosen for 1e-12 must deliver it."""
    import torch
    rng = np.random.default_rng(42)
    o, v = 8, 24
    A = _spread(rng, (v, v, v, v))
    B = _spread(rng, (v, v, o, o))
    C = np.zeros((v, v, o, o))
    ref = C.copy()
    oracle.orc_mult(1.0, A, "abef", B, "efij", 0.0, ref, "abij")
    got, rep = _run(torch, cuda, 6, 1.0, A, "abef", B, "efij", 0.0, C, "abij", tol=1e-12)
    assert normwise_rel(got, ref) <= 1e-12, rep
    assert rep["method"] == 6 and 2 <= rep["slices"] <= 16 and rep["est_error"] <= 1e-12 / 4


@pytest.mark.parametrize("seed", range(12))
def test_random_strided_contractions(cuda, seed):
    """Permuted, padded, batched operands through the scatter vectors."""
    import torch
    import tblis_b200 as tb
    rng = np.random.default_rng(7000 + seed)
    idx_A, idx_B, idx_C, lens = random_contraction(rng, max_len=9)
    A = make_operand(idx_A, lens, rng)
    B = make_operand(idx_B, lens, rng)
    C = make_operand(idx_C, lens, rng)
    ref = C[1].copy()
    oracle.orc_mult(0.5, A[1], idx_A, B[1], idx_B, 0.25, ref, idx_C)
    _, dA = to_device(*A, torch, cuda)
    _, dB = to_device(*B, torch, cuda)
    dCb, dC = to_device(*C, torch, cuda)
    rep = tb.mult_ex(0.5, dA, idx_A, dB, idx_B, 0.25, dC, idx_C, method=6, tolerance=1e-12)
    tb.synchronize()
    got = view_of(dCb.cpu().numpy(), C[1].shape, C[2])
    assert normwise_rel(got, ref) <= 1e-12, (idx_A, idx_B, idx_C, lens, rep)


@pytest.mark.parametrize("beta", [0.0, 0.75])
def test_long_k_runs_in_exact_chunks(cuda, beta):
    """K above 131072 (4096 k steps of 32) would overflow the INT32 sums of
    one run: it runs as two launches whose residues the combination sums
    modulo each modulus; beta applies once (a NaN in C with beta = 0 must not
    reach the result)."""
    import torch
    rng = np.random.default_rng(9)
    K = 140000
    A = rng.uniform(-1, 1, (130, K))
    B = rng.uniform(-1, 1, (K, 20))
    C = rng.uniform(-1, 1, (130, 20))
    ref = C.copy()
    oracle.orc_mult(1.0, A, "ik", B, "kj", beta, ref, "ij")
    if beta == 0.0:
        C[3, 5] = np.nan
    got, rep = _run(torch, cuda, 6, 1.0, A, "ik", B, "kj", beta, C, "ij", slices=14)
    assert np.all(np.isfinite(got))
    assert normwise_rel(got, ref) <= 1e-12


def test_zero_rows_columns_and_integers(cuda):
    """Zero rows of A and zero columns of B (shift 0, all residues 0), and
    small-integer operands, which scale to integers without rounding: the
    moduli hold the product exactly and only the FP64 evaluation of the
    reconstructed integer rounds (a few ulps), and the zero rows and columns
    of C come out exactly zero."""
    import torch
    rng = np.random.default_rng(3)
    A = rng.integers(-1000, 1001, (200, 300)).astype(np.float64)
    B = rng.integers(-1000, 1001, (300, 270)).astype(np.float64)
    A[7, :] = 0.0
    B[:, 100] = 0.0
    C = np.zeros((200, 270))
    ref = C.copy()
    oracle.orc_mult(1.0, A, "ik", B, "kj", 0.0, ref, "ij")
    got, rep = _run(torch, cuda, 6, 1.0, A, "ik", B, "kj", 0.0, C, "ij", slices=13)
    assert normwise_rel(got, ref) <= 1e-15
    assert not got[7].any() and not got[:, 100].any()


def test_auto_choice_follows_work(cuda):
    """Method 2 picks whichever scheme its time model (INT8 GEMMs plus plane
    writing plus, for moduli, the combination) puts first: on a large
    GEMM-dominated contraction at 1e-12 that is 13 moduli against 21 slice
    pairs; at 1e-3 two slices (3 pairs) against five moduli."""
    import torch
    import tblis_b200 as tb
    g = torch.Generator(device=cuda)
    g.manual_seed(11)
    A = torch.empty((8192, 4096), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g).t()
    A = torch.ldexp(A, torch.randint(-20, 21, A.shape, device=cuda, generator=g, dtype=torch.int32))
    B = torch.empty((4096, 8192), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g).t()
    ref = torch.zeros((4096, 4096), dtype=torch.float64, device=cuda)
    tb.mult_ex(1.0, A, "ik", B, "kj", 0.0, ref, "ij", method=1)
    nref = torch.linalg.vector_norm(ref).item()
    for tol, method in ((1e-12, 6), (1e-3, 2)):
        C = torch.zeros_like(ref)
        rep = tb.mult_ex(1.0, A, "ik", B, "kj", 0.0, C, "ij", method=2, tolerance=tol)
        tb.synchronize()
        err = torch.linalg.vector_norm(C - ref).item() / nref
        assert rep["method"] == method and err <= tol, (tol, rep, err)
    assert rep["slices"] <= 3


def test_medium_size_matches_fp64_path(cuda):
    """m = 9216, n = 2304, k = 6144 with exponent spread in A (72 x 9 output
    tiles per modulus): the moduli result at 1e-12 matches the FP64 path."""
    import torch
    import tblis_b200 as tb
    g = torch.Generator(device=cuda)
    g.manual_seed(21)
    A = torch.empty((6144, 9216), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g).t()
    B = torch.empty((2304, 6144), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g).t()
    exps = torch.randint(-20, 21, A.shape, device=cuda, generator=g, dtype=torch.int32)
    A = torch.ldexp(A, exps)
    C = torch.empty((2304, 9216), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g).t()
    ref = C.clone()
    tb.mult_ex(1.0, A, "ik", B, "kj", 0.5, ref, "ij", method=1)
    rep = tb.mult_ex(1.0, A, "ik", B, "kj", 0.5, C, "ij", method=6, tolerance=1e-12)
    tb.synchronize()
    err = (torch.linalg.vector_norm(C - ref) / torch.linalg.vector_norm(ref)).item()
    assert rep["method"] == 6 and err <= 1e-12, (err, rep)
