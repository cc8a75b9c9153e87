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
    # about 8 bits per slice: the error shrinks geometrically with the slice count
    assert err <= 50 * 2.0 ** (-8 * slices + 1), (slices, err)


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
    assert rep["est_error"] <= 1e-12 / 4
    # slices (method 2) or moduli (reported as method 6), whichever is less work
    assert (rep["method"] == 2 and 1 <= rep["slices"] <= 8) or (rep["method"] == 6 and 2 <= rep["slices"] <= 16)


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
    assert rep["slices"] <= (8 if rep["method"] == 2 else 16)


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


@pytest.mark.parametrize("beta", [0.0, 0.75])
def test_long_k_is_split_exactly(cuda, beta):
    """K beyond the INT32-exact range of one run of k steps (8 slices: 16640)
    is cut into five runs inside one launch, each flushed into C before the
    accumulators restart; beta applies once (a NaN in C with beta = 0 must not
    reach the result)."""
    import torch
    rng = np.random.default_rng(9)
    A = rng.uniform(-1, 1, (96, 70000))
    B = rng.uniform(-1, 1, (70000, 40))
    C = rng.uniform(-1, 1, (96, 40))
    ref = C.copy()
    oracle.orc_mult(1.0, A, "ik", B, "kj", beta, ref, "ij")
    if beta == 0.0:
        C[3, 5] = np.nan
    got, rep = _gpu_ozaki(torch, cuda, 1.0, A, "ik", B, "kj", beta, C, "ij", slices=8)
    assert np.all(np.isfinite(got))
    assert normwise_rel(got, ref) <= 1e-13


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


def _gpu_method(torch, dev, method, alpha, A, idx_A, B, idx_B, beta, C, idx_C, slices=0, tol=1e-12):
    import tblis_b200 as tb
    dA = torch.from_numpy(np.ascontiguousarray(A)).to(dev)
    dB = torch.from_numpy(np.ascontiguousarray(B)).to(dev)
    dC = torch.from_numpy(np.ascontiguousarray(C)).to(dev)
    rep = tb.mult_ex(alpha, dA, idx_A, dB, idx_B, beta, dC, idx_C, method=method, slices=slices, tolerance=tol)
    tb.synchronize()
    return dC.cpu().numpy(), rep


@pytest.mark.parametrize("tol", [1e-8, 1e-12])
def test_bf16_slices_meet_tolerance(cuda, tol):
    """Ozaki with BF16 digit planes (exact FP32 accumulation over K chunks of
    the launch) on the ladder's exponent-spread inputs; K = 1600 spans
    several exactness chunks."""
    import torch
    rng = np.random.default_rng(11)
    A = _spread(rng, (96, 40, 40))
    B = _spread(rng, (40, 40, 72))
    C = rng.uniform(-1, 1, (96, 72))
    ref = C.copy()
    oracle.orc_mult(1.5, A, "aef", B, "efb", 0.5, ref, "ab")
    got, rep = _gpu_method(torch, cuda, 3, 1.5, A, "aef", B, "efb", 0.5, C, "ab", tol=tol)
    assert rep["method"] == 3 and 1 <= rep["slices"] <= 8
    assert normwise_rel(got, ref) <= tol


def test_bf16_and_int8_slices_meet_their_estimates(cuda):
    """INT8 planes carry base-254 digits (about 8 bits a slice), BF16 planes
    base-128 digits (7 bits): with the same slice count both stay within the
    a-priori error each call reports, INT8 the tighter one."""
    import torch
    rng = np.random.default_rng(12)
    A = rng.uniform(-1, 1, (200, 300))
    B = rng.uniform(-1, 1, (300, 130))
    C = np.zeros((200, 130))
    ref = A @ B
    i8, ri = _gpu_method(torch, cuda, 2, 1.0, A, "ik", B, "kj", 0.0, C, "ij", slices=4)
    bf, rb = _gpu_method(torch, cuda, 3, 1.0, A, "ik", B, "kj", 0.0, C, "ij", slices=4)
    e_i8, e_bf = normwise_rel(i8, ref), normwise_rel(bf, ref)
    assert e_i8 <= 4 * ri["est_error"] and e_bf <= 4 * rb["est_error"]
    assert ri["est_error"] < rb["est_error"] and e_i8 < e_bf


@pytest.mark.parametrize("method,bound", [(4, 2e-3), (5, 1.5e-2)])
def test_single_pass_low_precision(cuda, method, bound):
    """One TF32 (method 4) or BF16 (method 5) pass with FP32 accumulation:
    error of the order of the input rounding, reported as such."""
    import torch
    rng = np.random.default_rng(13)
    A = _spread(rng, (64, 30, 30), -6, 6)
    B = _spread(rng, (30, 30, 80), -6, 6)
    C = np.zeros((64, 80))
    ref = C.copy()
    oracle.orc_mult(1.0, A, "aef", B, "efb", 0.0, ref, "ab")
    got, rep = _gpu_method(torch, cuda, method, 1.0, A, "aef", B, "efb", 0.0, C, "ab")
    err = normwise_rel(got, ref)
    assert rep["method"] == method and rep["slices"] == 1
    assert err <= bound, err
    assert err >= 1e-9      # a genuine low-precision pass, not an FP64 one


def test_named_configs_select_methods(cuda):
    import ctypes
    import torch
    import tblis_b200 as tb
    for name, method in [("b200_fp64", 1), ("b200_ozaki_i8", 2), ("b200_ozaki_bf16", 3),
                         ("b200_tf32", 4), ("b200_bf16", 5), ("b200_ozaki_crt", 6)]:
        cfg = tb.lib.tblis_get_config(name.encode())
        assert cfg
        a = torch.rand((40, 50), dtype=torch.float64, device=cuda)
        b = torch.rand((50, 30), dtype=torch.float64, device=cuda)
        c = torch.zeros((40, 30), dtype=torch.float64, device=cuda)
        rep = tb.mult_ex(1.0, a, "ik", b, "kj", 0.0, c, "ij", cfg=ctypes.c_void_p(cfg))
        # the INT8 Ozaki config runs slices (2) or moduli (6)
        assert rep["method"] == method or (method == 2 and rep["method"] == 6)
        err = (torch.linalg.norm(c - a @ b) / torch.linalg.norm(a @ b)).item()
        assert err <= (1e-12 if method in (1, 2, 3, 6) else 2e-2)


def test_medium_exponent_spread_matches_fp64(cuda):
    """A medium-size contraction (m = 9216, n = 2304, k = 6144: 72 x 36 output
    tiles, 340 MB of A planes, one exactness run) with exponent spread in A:
    the Ozaki result at tolerance 1e-12 matches the FP64 path."""
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
    rep = tb.mult_ex(1.0, A, "ik", B, "kj", 0.5, C, "ij", method=2, tolerance=1e-12)
    torch.cuda.synchronize()
    err = (torch.linalg.vector_norm(C - ref) / torch.linalg.vector_norm(ref)).item()
    assert rep["slices"] >= 1 and err <= 1e-12
