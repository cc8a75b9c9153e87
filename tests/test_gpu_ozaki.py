"""GPU parity of the Ozaki INT8 split-precision contraction (method 2):
normwise error against the FP64 oracle must stay within the requested
tolerance (slice count chosen per call) or, with an explicit slice count,
within the a-priori estimate the call reports."""
import numpy as np
import pytest

import oracle
from tests.helpers import (random_contraction, make_operand, normwise_rel, to_device, view_of,
                           random_tensor)

pytestmark = pytest.mark.gpu


def _spread(rng, shape, lo=-20, hi=20):
    return rng.uniform(-1, 1, shape) * np.ldexp(1.0, rng.integers(lo, hi + 1, shape))


def _gpu_ozaki(torch, dev, alpha, A, idx_A, B, idx_B, beta, C, idx_C, slices=0, tol=1e-12):
    import tblis_b200 as tb
    dA = torch.from_numpy(np.ascontiguousarray(A)).to(dev)
    dB = torch.from_numpy(np.ascontiguousarray(B)).to(dev)
    dC = torch.from_numpy(np.ascontiguousarray(C)).to(dev)
    rep = tb.mult_ex(alpha, dA, idx_A, dB, idx_B, beta, dC, idx_C, method=2, slices=slices, tolerance=tol)
    tb.synchronize()     # raises if a kernel gave up a bounded wait
    return dC.cpu().numpy(), rep


@pytest.mark.parametrize("slices", [3, 5, 7])
def test_matrix_error_tracks_slices(cuda, slices):
    import torch
    rng = np.random.default_rng(slices)
    A = rng.uniform(-1, 1, (300, 257))
    B = rng.uniform(-1, 1, (257, 190))
    C = rng.uniform(-1, 1, (300, 190))
    ref = C.copy()
    oracle.orc_mult(1.0, A, "ik", B, "kj", 0.5, ref, "ij")
    got, rep = _gpu_ozaki(torch, cuda, 1.0, A, "ik", B, "kj", 0.5, C, "ij", slices=slices)
    err = normwise_rel(got, ref)
    assert rep["slices"] == slices and rep["method"] == 2
    # 7 bits per slice: the error shrinks geometrically with the slice count
    assert err <= 50 * 2.0 ** (-7 * slices), (slices, err)


def test_tolerance_1e12_with_exponent_spread(cuda):
    """The ladder's input distribution (uniform(-1,1)*2^k, k in [-20,20]) at a
    reduced size; the chosen slice count must deliver <= 1e-12."""
    import torch
    rng = np.random.default_rng(42)
    o, v = 8, 24
    A = _spread(rng, (v, v, v, v))
    B = _spread(rng, (v, v, o, o))
    C = np.zeros((v, v, o, o))
    ref = C.copy()
    oracle.orc_mult(1.0, A, "abef", B, "efij", 0.0, ref, "abij")
    got, rep = _gpu_ozaki(torch, cuda, 1.0, A, "abef", B, "efij", 0.0, C, "abij", tol=1e-12)
    err = normwise_rel(got, ref)
    assert err <= 1e-12, (err, rep)
    assert rep["est_error"] <= 1e-12 / 4 and 1 <= rep["slices"] <= 8


@pytest.mark.parametrize("tol", [1e-6, 1e-10, 1e-13])
def test_slice_count_follows_tolerance(cuda, tol):
    import torch
    rng = np.random.default_rng(7)
    A = rng.uniform(-1, 1, (130, 200))
    B = rng.uniform(-1, 1, (200, 70))
    C = np.zeros((130, 70))
    ref = C.copy()
    oracle.orc_mult(2.0, A, "ik", B, "kj", 0.0, ref, "ij")
    got, rep = _gpu_ozaki(torch, cuda, 2.0, A, "ik", B, "kj", 0.0, C, "ij", tol=tol)
    assert normwise_rel(got, ref) <= tol
    assert rep["slices"] <= 8


@pytest.mark.parametrize("seed", range(12))
def test_random_strided_contractions(cuda, seed):
    """Permuted, padded, batched operands through the same scatter vectors
    as the FP64 path."""
    import torch
    import tblis_b200 as tb
    rng = np.random.default_rng(3000 + seed)
    idx_A, idx_B, idx_C, lens = random_contraction(rng, max_len=9)
    A = make_operand(idx_A, lens, rng)
    B = make_operand(idx_B, lens, rng)
    C = make_operand(idx_C, lens, rng)
    ref = C[1].copy()
    oracle.orc_mult(0.5, A[1], idx_A, B[1], idx_B, 0.25, ref, idx_C)
    _, dA = to_device(*A, torch, cuda)
    _, dB = to_device(*B, torch, cuda)
    dCb, dC = to_device(*C, torch, cuda)
    rep = tb.mult_ex(0.5, dA, idx_A, dB, idx_B, 0.25, dC, idx_C, method=2, tolerance=1e-12)
    torch.cuda.synchronize()
    got = view_of(dCb.cpu().numpy(), C[1].shape, C[2])
    assert normwise_rel(got, ref) <= 1e-12, (idx_A, idx_B, idx_C, lens, rep)


def test_long_k_is_split_exactly(cuda):
    """K beyond the INT32-exact range of one launch (8 slices: 65536) runs as
    several launches accumulating into C."""
    import torch
    rng = np.random.default_rng(9)
    A = rng.uniform(-1, 1, (96, 70000))
    B = rng.uniform(-1, 1, (70000, 40))
    C = rng.uniform(-1, 1, (96, 40))
    ref = C.copy()
    oracle.orc_mult(1.0, A, "ik", B, "kj", 1.0, ref, "ij")
    got, rep = _gpu_ozaki(torch, cuda, 1.0, A, "ik", B, "kj", 1.0, C, "ij", slices=8)
    assert normwise_rel(got, ref) <= 1e-13
    assert rep["kernels"] >= 2 + 2 + 2


def test_config_selects_ozaki(cuda):
    import torch
    import tblis_b200 as tb
    rng = np.random.default_rng(5)
    A = torch.from_numpy(rng.uniform(-1, 1, (64, 96))).to(cuda)
    B = torch.from_numpy(rng.uniform(-1, 1, (96, 80))).to(cuda)
    C = torch.zeros((64, 80), dtype=torch.float64, device=cuda)
    cfg = tb.get_config("b200_ozaki_i8")
    assert cfg
    tb.mult(1.0, A, "ik", B, "kj", 0.0, C, "ij", cfg=cfg)
    torch.cuda.synchronize()
    ref = A.cpu().numpy() @ B.cpu().numpy()
    assert normwise_rel(C.cpu().numpy(), ref) <= 1e-12
