"""GPU parity of the level-1 kernels (add/transpose/trace/replicate, dot,
reduce, scale, set, shift) against the oracle on the same seeded inputs."""
import numpy as np
import pytest

import oracle
from tests.helpers import normwise_rel, random_tensor, to_device, view_of

pytestmark = pytest.mark.gpu


def _dev(torch, cuda, t):
    base, view, strides = t
    db, dv = to_device(base, view, strides, torch, cuda)
    return db, dv


ADD_CASES = [
    ("abcd", "cadb", (5, 6, 7, 3), (7, 5, 3, 6)),          # permutation
    ("abcd", "abcd", (33, 6, 7, 3), (33, 6, 7, 3)),        # same order (vector path)
    ("abcd", "db", (5, 6, 7, 3), (3, 6)),                  # trace
    ("ab", "cbad", (5, 6), (4, 6, 5, 3)),                  # replicate
    ("", "abc", (), (3, 4, 5)),                            # scalar broadcast
    ("abc", "", (3, 4, 5), ()),                            # full trace to a scalar
    ("ab", "ba", (130, 70), (70, 130)),                    # 2-D transpose, partial tiles
]


@pytest.mark.parametrize("case", range(len(ADD_CASES)))
@pytest.mark.parametrize("ab", [(1.0, 0.0), (0.5, -1.5), (0.0, 2.0), (0.0, 0.0)])
def test_add_matches_oracle(cuda, case, ab):
    import torch
    import tblis_b200 as tb
    idx_A, idx_B, lA, lB = ADD_CASES[case]
    alpha, beta = ab
    rng = np.random.default_rng(case)
    A = random_tensor(list(lA), rng, list(rng.permutation(len(lA))))
    B = random_tensor(list(lB), rng, list(rng.permutation(len(lB))), pad=1)
    ref = B[1].copy()
    oracle.orc_add(alpha, A[1], idx_A, beta, ref, idx_B)
    _, dA = _dev(torch, cuda, A)
    dBb, dB = _dev(torch, cuda, B)
    tb.add(alpha, dA, idx_A, beta, dB, idx_B)
    torch.cuda.synchronize()
    got = view_of(dBb.cpu().numpy(), B[1].shape, B[2])
    assert normwise_rel(got, ref) <= 1e-14


def test_transpose_full_size(cuda):
    """D[ijab] = C[abij] at v=256, o=64 (2.15 GB each way), bit-exact."""
    import torch
    import tblis_b200 as tb
    v, o = 256, 64
    g = torch.Generator(device=cuda)
    g.manual_seed(9)
    C = torch.empty((o, o, v, v), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g).permute(3, 2, 1, 0)
    D = torch.zeros((v, v, o, o), dtype=torch.float64, device=cuda).permute(3, 2, 1, 0)
    tb.add(1.0, C, "abij", 0.0, D, "ijab")
    torch.cuda.synchronize()
    assert torch.equal(D, C.permute(2, 3, 0, 1))


def test_dot_matches_oracle(cuda):
    import torch
    import tblis_b200 as tb
    rng = np.random.default_rng(11)
    A = random_tensor([29, 31, 7], rng, [2, 0, 1], pad=1)
    B = random_tensor([31, 29, 7], rng, [0, 1, 2])
    want = oracle.orc_dot(A[1], "abc", B[1], "bac")
    _, dA = _dev(torch, cuda, A)
    _, dB = _dev(torch, cuda, B)
    got = tb.dot(dA, "abc", dB, "bac")
    assert abs(got - want) <= 1e-13 * max(1.0, abs(want))
    # host operands
    got2 = tb.dot(A[1], "abc", B[1], "bac")
    assert abs(got2 - want) <= 1e-13 * max(1.0, abs(want))


@pytest.mark.parametrize("op", range(7))
@pytest.mark.parametrize("alpha", [1.0, -0.5])
def test_reduce_matches_oracle(cuda, op, alpha):
    import torch
    import tblis_b200 as tb
    rng = np.random.default_rng(12)
    A = random_tensor([41, 13, 9], rng, [1, 2, 0], pad=1)
    want_v, want_i = oracle.orc_reduce(op, A[1], "abc", alpha)
    _, dA = _dev(torch, cuda, A)
    dv = tb._View(dA, alpha)
    import ctypes
    r = tb.tblis_scalar()
    r.type = 1
    idx = ctypes.c_ssize_t(-7)
    tb.lib.tblis_tensor_reduce(None, None, op, dv.ref, b"abc", ctypes.byref(r), ctypes.byref(idx))
    tb._check()
    assert abs(r.data[0] - want_v) <= 1e-13 * max(1.0, abs(want_v))
    if op in (2, 3, 4, 5):
        assert idx.value == want_i


def test_reduce_ties_pick_first_in_iteration_order(cuda):
    import torch
    import tblis_b200 as tb
    A = torch.zeros((1000, 3), dtype=torch.float64, device=cuda)
    A[10, 1] = 5.0
    A[500, 2] = 5.0
    v, i = tb.reduce(tb.REDUCE_MAX, A, "ab")
    Ah = A.cpu().numpy()
    wv, wi = oracle.orc_reduce(2, Ah, "ab")
    assert v == wv == 5.0 and i == wi


@pytest.mark.parametrize("kind", ["set", "scale", "shift"])
def test_unary_matches_oracle(cuda, kind):
    import torch
    import tblis_b200 as tb
    rng = np.random.default_rng(13)
    A = random_tensor([17, 5, 23], rng, [2, 1, 0], pad=2)
    ref = A[1].copy()
    dAb, dA = _dev(torch, cuda, A)
    if kind == "set":
        oracle.orc_unary("set", ref, alpha=0.25)
        tb.set(0.25, dA, "abc")
    elif kind == "scale":
        oracle.orc_unary("scale", ref, alpha=-3.0)
        tb.scale(-3.0, dA, "abc")
    else:
        oracle.orc_unary("shift", ref, alpha=0.5, shift=2.0)
        tb.shift(2.0, 0.5, dA, "abc")
    torch.cuda.synchronize()
    got = view_of(dAb.cpu().numpy(), A[1].shape, A[2])
    assert normwise_rel(got, ref) <= 1e-15
    # padding between elements is untouched
    base_after = dAb.cpu().numpy()
    mask = np.ones(base_after.size, dtype=bool)
    idx = np.lib.stride_tricks.as_strided(np.arange(base_after.size), shape=A[1].shape,
                                          strides=[s * 8 for s in A[2]])
    mask[idx.ravel()] = False
    assert np.array_equal(base_after[mask], A[0][mask])


@pytest.mark.parametrize("dtype", ["float32", "float64", "complex64", "complex128"])
@pytest.mark.parametrize("shape", [(130, 70, 4), (64, 96, 6), (66, 34, 3), (65, 64, 2), (64, 65, 2)])
@pytest.mark.parametrize("beta", [0.0, 0.5])
def test_transpose_pairs_and_singles(cuda, dtype, shape, beta):
    """B[cba] = alpha*A[abc] + beta*B[cba] through the shared-memory transpose.
    Even unit extents with even strides take the paired form (two elements per
    access, 16 bytes for 8-byte types); an odd extent on either side, a
    16-byte element type or an offset base take single elements. Both agree
    with torch to rounding (a misplaced element would be an O(1) error)."""
    import torch
    import tblis_b200 as tb
    g = torch.Generator(device=cuda)
    g.manual_seed(sum(shape))
    dt = getattr(torch, dtype)
    real = torch.float32 if dtype in ("float32", "complex64") else torch.float64

    def rnd(*s):
        x = torch.empty(s, dtype=real, device=cuda).uniform_(-1, 1, generator=g)
        if dt.is_complex:
            x = torch.complex(x, torch.empty(s, dtype=real, device=cuda).uniform_(-1, 1, generator=g))
        return x
    a, b, c = shape
    A = rnd(c, b, a).permute(2, 1, 0)              # a fastest
    Bbuf = rnd(a * b * c + 1)                      # one extra element: offset (unaligned) view too
    for off in (0, 1):
        B = Bbuf[off:off + a * b * c].view(a, b, c)   # c fastest: B[cba] column-major
        before = B.clone()
        alpha = 0.75
        tb.add(alpha, A, "abc", beta, B, "abc")
        want = alpha * A + beta * before if beta != 0 else alpha * A
        torch.cuda.synchronize()
        tol = 1e-6 if real == torch.float32 else 1e-15
        err = (torch.linalg.vector_norm(B - want) / torch.linalg.vector_norm(want)).item()
        assert err <= tol, (dtype, shape, beta, off, err)
