"""GPU parity of dcomplex contractions (four real products per complex
product on the FP64 path) against the reference's own complex contraction:
random label splits and permuted strides, real and complex alpha and beta,
and conjugation flags, which the reference applies in its REFERENCE
implementation (mult_ref, src/internal/3t/dense/mult.cxx:653-720)."""
import ctypes

import numpy as np
import pytest

import oracle
from tests.helpers import random_contraction

pytestmark = pytest.mark.gpu


def _cplx(rng, shape, perm):
    """A complex128 array with its dimensions stored in the order `perm`."""
    dims = [shape[p] for p in perm]
    base = np.asarray(rng.uniform(-1, 1, dims) + 1j * rng.uniform(-1, 1, dims), dtype=np.complex128)
    return base.transpose(np.argsort(perm)) if base.ndim else base


def _dev_view(torch, x, dev):
    """x on `dev` with the same memory order of its dimensions."""
    if x.ndim == 0:
        return torch.from_numpy(np.array(x)).to(dev)
    order = np.argsort([-s for s in x.strides], kind="stable")
    flat = torch.from_numpy(np.ascontiguousarray(x.transpose(order))).to(dev)
    return flat.permute(*np.argsort(order).tolist())


def _gpu_mult(torch, dev, alpha, A, idx_A, B, idx_B, beta, C, idx_C, conj_A=False, conj_B=False):
    import tblis_b200 as tb
    dA, dB, dC = _dev_view(torch, A, dev), _dev_view(torch, B, dev), _dev_view(torch, C, dev)
    a, b, c = tb._View(dA, alpha), tb._View(dB), tb._View(dC, beta)
    a.t.conj, b.t.conj = int(conj_A), int(conj_B)
    tb.lib.tblis_tensor_mult(None, None, a.ref, tb._labels(idx_A), b.ref, tb._labels(idx_B), c.ref,
                             tb._labels(idx_C))
    tb._check()
    torch.cuda.synchronize()
    return dC.cpu().numpy()


def _rel(x, y):
    return np.linalg.norm(x - y) / max(1e-300, np.linalg.norm(y))


@pytest.mark.parametrize("seed", range(10))
def test_random_complex_contractions(cuda, seed):
    import torch
    rng = np.random.default_rng(500 + seed)
    idx_A, idx_B, idx_C, lens = random_contraction(rng, max_len=9)
    A = _cplx(rng, [lens[c] for c in idx_A], rng.permutation(len(idx_A)))
    B = _cplx(rng, [lens[c] for c in idx_B], rng.permutation(len(idx_B)))
    C = _cplx(rng, [lens[c] for c in idx_C], rng.permutation(len(idx_C)))
    alpha = [1.0, 0.5 - 0.25j, 2j][seed % 3]
    beta = [0.0, 1.0, 0.3 + 0.7j, -0.5][seed % 4]
    want = C.copy()
    oracle.ref_mult(alpha, A, idx_A, B, idx_B, beta, want, idx_C)
    got = _gpu_mult(torch, cuda, alpha, A, idx_A, B, idx_B, beta, C, idx_C)
    assert _rel(got, want) <= 1e-13


@pytest.mark.parametrize("conj_A,conj_B", [(True, False), (False, True), (True, True)])
def test_conjugation_flags(cuda, conj_A, conj_B):
    import torch
    rng = np.random.default_rng(7)
    A = _cplx(rng, [6, 7, 5], [2, 0, 1])
    B = _cplx(rng, [5, 8, 7], [0, 1, 2])
    C = _cplx(rng, [8, 6], [1, 0])
    want = C.copy()
    old = oracle.ref_dense_impl(2)
    try:
        oracle.ref_mult(0.5 + 1j, A, "abc", B, "cdb", 0.25, want, "da", conj_A=conj_A, conj_B=conj_B)
    finally:
        oracle.ref_dense_impl(old)
    # the same by numpy
    a = np.conj(A) if conj_A else A
    b = np.conj(B) if conj_B else B
    np_want = (0.5 + 1j) * np.einsum("abc,cdb->da", a, b) + 0.25 * C
    assert _rel(want, np_want) <= 1e-13
    got = _gpu_mult(torch, cuda, 0.5 + 1j, A, "abc", B, "cdb", 0.25, C, "da", conj_A, conj_B)
    assert _rel(got, want) <= 1e-13


def test_complex_beta_zero_never_reads_c(cuda):
    import torch
    rng = np.random.default_rng(8)
    A = _cplx(rng, [9, 4], [0, 1])
    B = _cplx(rng, [4, 11], [1, 0])
    C = np.full((9, 11), np.nan + 1j * np.nan)
    got = _gpu_mult(torch, cuda, 1.0 - 1j, A, "ik", B, "kj", 0.0, C, "ij")
    assert np.all(np.isfinite(got))
    assert _rel(got, (1.0 - 1j) * (A @ B)) <= 1e-13


@pytest.mark.parametrize("method", [2, 6])
def test_complex_contraction_on_the_ozaki_paths(cuda, method):
    """A dcomplex contraction on an Ozaki method (2: INT8 slices or moduli,
    whichever the models pick; 6: moduli): each real product of the 4M split
    runs on that INT8 path, with slices or moduli chosen for the tolerance,
    and the complex result stays within it against the reference's own
    complex contraction."""
    import torch
    import tblis_b200 as tb
    rng = np.random.default_rng(77)
    lens = {"a": 40, "b": 36, "e": 48, "f": 30, "i": 20, "j": 24}
    A = _cplx(rng, [lens[c] for c in "abef"], [2, 0, 3, 1])
    B = _cplx(rng, [lens[c] for c in "efij"], [1, 3, 0, 2])
    C = _cplx(rng, [lens[c] for c in "abij"], [0, 1, 2, 3])
    alpha, beta = 0.5 - 0.25j, 0.3 + 0.7j
    want = C.copy()
    oracle.ref_mult(alpha, A, "abef", B, "efij", beta, want, "abij")
    dA, dB, dC = _dev_view(torch, A, cuda), _dev_view(torch, B, cuda), _dev_view(torch, C, cuda)
    rep = tb.mult_ex(alpha, dA, "abef", dB, "efij", beta, dC, "abij", method=method, tolerance=1e-12)
    torch.cuda.synchronize()
    assert rep["slices"] > 0                      # the real products ran on the INT8 path
    err = _rel(dC.cpu().numpy(), want)
    assert err <= 1e-12, err
