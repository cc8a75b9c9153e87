"""GPU parity of the float, scomplex and dcomplex paths against the reference
run on the same data: level-1 add (permute / trace / replicate), dot, reduce,
scale, set and shift with conj flags and complex scalars
(src/iface/1t/*.cxx, src/kernels/1v/*.hpp), and float / scomplex contractions
(src/iface/3t/mult.cxx over src/util/basic_types.h:97-98 types)."""
import numpy as np
import pytest

import oracle
from tests.helpers import strided_empty, view_of

pytestmark = pytest.mark.gpu

DTYPES = [np.float32, np.complex64, np.complex128]
# normwise relative tolerance per type: the GPU and the reference sum in
# different orders (float rounding), or compute in FP64 (float mult)
TOL = {np.float32: 2e-6, np.complex64: 2e-6, np.complex128: 1e-14}


def typed_tensor(shape, rng, dtype, order=None, pad=0):
    base, view, strides = strided_empty(shape, order, pad, rng, dtype=dtype)
    vals = rng.uniform(-1.0, 1.0, base.size)
    if np.dtype(dtype).kind == "c":
        vals = vals + 1j * rng.uniform(-1.0, 1.0, base.size)
    base[:] = vals.astype(dtype)
    return base, view, strides


def device(torch, cuda, t):
    base, view, strides = t
    db = torch.from_numpy(base.copy()).to(cuda)
    return db, torch.as_strided(db, tuple(view.shape), tuple(strides))


def rel(got, want):
    d = np.linalg.norm((np.asarray(got) - np.asarray(want)).ravel())
    n = np.linalg.norm(np.asarray(want).ravel())
    return d / n if n > 0 else d


def scalar(dtype, v):
    return complex(v) if np.dtype(dtype).kind == "c" else complex(v).real


ADD_CASES = [
    ("abcd", "cadb", (5, 6, 7, 3), (7, 5, 3, 6)),          # permutation
    ("abcd", "abcd", (33, 6, 7, 3), (33, 6, 7, 3)),        # same order (vector path)
    ("abcd", "db", (5, 6, 7, 3), (3, 6)),                  # trace
    ("ab", "cbad", (5, 6), (4, 6, 5, 3)),                  # replicate
    ("ab", "ba", (130, 70), (70, 130)),                    # 2-D transpose, partial tiles
]


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("case", range(len(ADD_CASES)))
@pytest.mark.parametrize("conj", [(False, False), (True, False), (True, True)])
@pytest.mark.parametrize("ab", [(1.0, 0.0), (0.5 - 0.25j, -1.5 + 1j), (0.0, 2.0 - 1j)])
def test_add(cuda, dtype, case, conj, ab):
    import torch
    import tblis_b200 as tb
    idx_A, idx_B, lA, lB = ADD_CASES[case]
    alpha, beta = scalar(dtype, ab[0]), scalar(dtype, ab[1])
    rng = np.random.default_rng(100 + case)
    A = typed_tensor(list(lA), rng, dtype, list(rng.permutation(len(lA))))
    B = typed_tensor(list(lB), rng, dtype, list(rng.permutation(len(lB))), pad=1)
    want = B[0].copy()
    oracle.ref_add(alpha, A[1], idx_A, beta, view_of(want, B[1].shape, B[2]), idx_B,
                   conj_A=conj[0], conj_B=conj[1])
    _, dA = device(torch, cuda, A)
    dBb, dB = device(torch, cuda, B)
    tb.add(alpha, dA, idx_A, beta, dB, idx_B, conj_A=conj[0], conj_B=conj[1])
    torch.cuda.synchronize()
    got = dBb.cpu().numpy()
    # the padding between elements is untouched; the elements match
    assert rel(got, want) <= TOL[dtype] * 4


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("conj", [(False, False), (True, False), (False, True), (True, True)])
def test_dot(cuda, dtype, conj):
    import torch
    import tblis_b200 as tb
    rng = np.random.default_rng(11)
    A = typed_tensor([29, 31, 7], rng, dtype, [2, 0, 1], pad=1)
    B = typed_tensor([31, 29, 7], rng, dtype, [0, 1, 2])
    want = oracle.ref_dot(A[1], "abc", B[1], "bac", conj_A=conj[0], conj_B=conj[1])
    _, dA = device(torch, cuda, A)
    _, dB = device(torch, cuda, B)
    got = tb.dot(dA, "abc", dB, "bac", conj_A=conj[0], conj_B=conj[1])
    scale = np.sqrt(np.sum(np.abs(A[1]) ** 2) * np.sum(np.abs(B[1]) ** 2))
    assert abs(got - want) <= TOL[dtype] * 10 * scale
    # host operands
    got2 = tb.dot(A[1], "abc", B[1], "bac", conj_A=conj[0], conj_B=conj[1])
    assert abs(got2 - want) <= TOL[dtype] * 10 * scale


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("op", range(7))
@pytest.mark.parametrize("alpha", [1.0, -0.5 + 0.75j])
@pytest.mark.parametrize("conj", [False, True])
def test_reduce(cuda, dtype, op, alpha, conj):
    """Complex values order by their real parts (MAX / MIN) and by modulus
    (the ABS ops); a scalar with a negative real part swaps MAX and MIN."""
    import torch
    import tblis_b200 as tb
    rng = np.random.default_rng(40 + op)
    A = typed_tensor([37, 5, 11], rng, dtype, [1, 2, 0], pad=1)
    a = scalar(dtype, alpha)
    want, wi = oracle.ref_reduce(op, A[1], "abc", a, conj)
    _, dA = device(torch, cuda, A)
    view = tb._View(dA, a, conj)
    import ctypes
    r = tb.tblis_scalar()
    r.type = view.t.type
    idx = ctypes.c_ssize_t(-1)
    tb.lib.tblis_tensor_reduce(None, None, op, view.ref, b"abc", ctypes.byref(r), ctypes.byref(idx))
    tb._check()
    got = tb._scalar_value(r, view.t.type)
    mag = max(1.0, abs(want))
    assert abs(got - want) <= TOL[dtype] * 40 * mag, (got, want)
    if op in (2, 3, 4, 5):
        assert idx.value == wi


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("kind", [0, 1, 2])
@pytest.mark.parametrize("conj", [False, True])
def test_set_scale_shift(cuda, dtype, kind, conj):
    import torch
    import tblis_b200 as tb
    rng = np.random.default_rng(70 + kind)
    A = typed_tensor([9, 13, 4], rng, dtype, [2, 0, 1], pad=1)
    alpha, value = scalar(dtype, 1.25 - 0.5j), scalar(dtype, -0.75 + 2j)
    want = A[0].copy()
    oracle.ref_unary(kind, view_of(want, A[1].shape, A[2]), "abc", alpha, value, conj)
    dAb, dA = device(torch, cuda, A)
    if kind == 0:
        tb.set(value, dA, "abc")
    elif kind == 1:
        tb.scale(alpha, dA, "abc", conj=conj)
    else:
        tb.shift(value, alpha, dA, "abc", conj=conj)
    torch.cuda.synchronize()
    assert rel(dAb.cpu().numpy(), want) <= TOL[dtype]


MULT_CASES = [
    ("abef", "efij", "abij", {"a": 7, "b": 5, "e": 6, "f": 4, "i": 3, "j": 8}),
    ("aeim", "mbej", "aibj", {"a": 6, "e": 5, "i": 4, "m": 7, "b": 3, "j": 5}),
    ("ak", "kb", "ab", {"a": 130, "k": 96, "b": 70}),
]


@pytest.mark.parametrize("dtype", [np.float32, np.complex64])
@pytest.mark.parametrize("case", range(len(MULT_CASES)))
@pytest.mark.parametrize("beta", [0.0, 0.5 + 0.25j])
@pytest.mark.parametrize("host", [False, True])
def test_mult_float_and_scomplex(cuda, dtype, case, beta, host):
    """float / scomplex contractions are computed in FP64 / dcomplex and
    rounded back: they agree with the reference's float arithmetic to float
    rounding."""
    import torch
    import tblis_b200 as tb
    iA, iB, iC, lens = MULT_CASES[case]
    rng = np.random.default_rng(200 + case)
    A = typed_tensor([lens[c] for c in iA], rng, dtype, list(rng.permutation(len(iA))), pad=1)
    B = typed_tensor([lens[c] for c in iB], rng, dtype, list(rng.permutation(len(iB))))
    C = typed_tensor([lens[c] for c in iC], rng, dtype, list(rng.permutation(len(iC))), pad=1)
    alpha, beta = scalar(dtype, 0.75 + 0.5j), scalar(dtype, beta)
    want = C[0].copy()
    oracle.ref_mult(alpha, A[1], iA, B[1], iB, beta, view_of(want, C[1].shape, C[2]), iC)
    if host:
        got = C[0].copy()
        tb.mult(alpha, A[1], iA, B[1], iB, beta, view_of(got, C[1].shape, C[2]), iC)
    else:
        _, dA = device(torch, cuda, A)
        _, dB = device(torch, cuda, B)
        dCb, dC = device(torch, cuda, C)
        tb.mult(alpha, dA, iA, dB, iB, beta, dC, iC)
        torch.cuda.synchronize()
        got = dCb.cpu().numpy()
    assert rel(got, want) <= 1e-5
    # the padding of C (never part of the tensor) is unchanged
    mask = np.ones(C[0].size, bool)
    mask[np.unique(view_of(np.arange(C[0].size), C[1].shape, C[2]).ravel())] = False
    assert np.array_equal(got[mask], C[0][mask])


@pytest.mark.parametrize("conj", [(True, False), (False, True), (True, True)])
def test_mult_scomplex_conj(cuda, conj):
    import torch
    import tblis_b200 as tb
    rng = np.random.default_rng(9)
    A = typed_tensor([12, 9, 7], rng, np.complex64, [0, 1, 2])
    B = typed_tensor([9, 7, 10], rng, np.complex64, [2, 0, 1])
    C = typed_tensor([12, 10], rng, np.complex64, [1, 0])
    want = np.asarray(C[1]).copy()
    ca = np.conj(A[1]) if conj[0] else A[1]
    cb = np.conj(B[1]) if conj[1] else B[1]
    want = (1.0 - 0.5j) * np.einsum("aef,efb->ab", ca.astype(np.complex128), cb.astype(np.complex128)) \
        + (0.25 + 1j) * want
    _, dA = device(torch, cuda, A)
    _, dB = device(torch, cuda, B)
    dCb, dC = device(torch, cuda, C)
    tb.mult(1.0 - 0.5j, dA, "aef", dB, "efb", 0.25 + 1j, dC, "ab", conj_A=conj[0], conj_B=conj[1])
    torch.cuda.synchronize()
    got = dC.cpu().numpy()
    assert rel(got, want) <= 1e-6


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_host_output_with_gaps_keeps_the_gaps(cuda, dtype):
    """A host C whose storage has gaps (a strided view into a larger array)
    with beta = 0: the staged copy comes back whole, so the gaps must come
    back unchanged."""
    import tblis_b200 as tb
    rng = np.random.default_rng(5)
    A = typed_tensor([40, 30], rng, dtype, [0, 1])
    B = typed_tensor([30, 20], rng, dtype, [1, 0])
    big = rng.uniform(-1, 1, (80, 41)).astype(dtype)
    C = big[::2, 1::2]                       # every other row and column
    keep = big.copy()
    tb.mult(1.0, A[1], "ak", B[1], "kb", 0.0, C, "ab")
    want = A[1].astype(np.float64) @ B[1].astype(np.float64)
    assert rel(C, want) <= (1e-6 if dtype == np.float32 else 1e-14)
    mask = np.ones(big.shape, bool)
    mask[::2, 1::2] = False
    assert np.array_equal(big[mask], keep[mask])
    # the same through add with beta = 0
    big2 = keep.copy()
    D = big2[::2, 1::2]
    tb.add(2.0, A[1][:, :20], "ab", 0.0, D, "ab")
    assert rel(D, 2.0 * A[1][:, :20]) <= 1e-6
    assert np.array_equal(big2[mask], keep[mask])
