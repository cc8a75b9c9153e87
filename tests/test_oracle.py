"""CPU tests: the oracle restatement pinned against the reference itself
(compiled from its own sources into oracle/_ref), and the product planner's
index work pinned bit for bit against both."""
import re
import os

import numpy as np
import pytest

import oracle
from tests.helpers import random_contraction, make_operand, normwise_rel, random_tensor

needs_ref = pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built")


@needs_ref
@pytest.mark.parametrize("seed", range(40))
def test_oracle_mult_matches_reference(seed):
    rng = np.random.default_rng(1000 + seed)
    idx_A, idx_B, idx_C, lens = random_contraction(rng)
    _, A, _ = make_operand(idx_A, lens, rng)
    _, B, _ = make_operand(idx_B, lens, rng)
    _, C0, _ = make_operand(idx_C, lens, rng)
    alpha, beta = rng.choice([1.0, 0.5, -2.0]), rng.choice([0.0, 1.0, 0.75])
    C1 = C0.copy()
    C2 = C0.copy()
    oracle.orc_mult(alpha, A, idx_A, B, idx_B, beta, C1, idx_C)
    oracle.ref_mult(alpha, A, idx_A, B, idx_B, beta, C2, idx_C, threads=2)
    assert normwise_rel(C1, C2) <= 1e-13


@needs_ref
@pytest.mark.parametrize("case", ["perm", "trace", "replicate", "scalar"])
def test_oracle_add_matches_reference(case):
    rng = np.random.default_rng(7)
    if case == "perm":
        idx_A, idx_B, lensA, lensB = "abcd", "cadb", (5, 6, 7, 3), (7, 5, 3, 6)
    elif case == "trace":
        idx_A, idx_B, lensA, lensB = "abcd", "db", (5, 6, 7, 3), (3, 6)
    elif case == "replicate":
        idx_A, idx_B, lensA, lensB = "ab", "cbad", (5, 6), (4, 6, 5, 3)
    else:
        idx_A, idx_B, lensA, lensB = "", "abc", (), (3, 4, 5)
    _, A, _ = random_tensor(list(lensA), rng, list(rng.permutation(len(lensA))))
    _, B0, _ = random_tensor(list(lensB), rng, list(rng.permutation(len(lensB))), pad=1)
    for alpha, beta in [(1.0, 0.0), (0.5, -1.5), (0.0, 2.0)]:
        B1, B2 = B0.copy(), B0.copy()
        oracle.orc_add(alpha, A, idx_A, beta, B1, idx_B)
        oracle.ref_add(alpha, A, idx_A, beta, B2, idx_B, threads=2)
        assert normwise_rel(B1, B2) <= 1e-14


@needs_ref
def test_oracle_dot_and_reduce_match_reference():
    rng = np.random.default_rng(11)
    _, A, _ = random_tensor([9, 8, 7], rng, [2, 0, 1], pad=1)
    _, B, _ = random_tensor([8, 9, 7], rng, [0, 1, 2])
    d1 = oracle.orc_dot(A, "abc", B, "bac")
    d2 = oracle.ref_dot(A, "abc", B, "bac")
    assert abs(d1 - d2) <= 1e-13 * max(1.0, abs(d2))
    for op in range(7):
        for alpha in (1.0, -0.5):
            v1, i1 = oracle.orc_reduce(op, A, "abc", alpha)
            v2, i2 = oracle.ref_reduce(op, A, "abc", alpha)
            assert abs(v1 - v2) <= 1e-13 * max(1.0, abs(v2)), (op, alpha)
            if op in (2, 3, 4, 5):
                assert i1 == i2, (op, alpha)


def _random_scatter_case(rng):
    nd = int(rng.integers(1, 5))
    lens = [int(rng.integers(1, 9)) for _ in range(nd)]
    strides = []
    s = 1
    for l in lens:
        strides.append(s)
        s *= l + int(rng.integers(0, 2))
    perm = rng.permutation(nd)
    strides = [strides[p] for p in perm]
    tot = int(np.prod(lens))
    BS = int(rng.choice([1, 2, 3, 4, 6, 8, 16]))
    pack_3d = bool(nd >= 2 and rng.random() < 0.5)
    off = int(rng.integers(0, tot))
    size = int(rng.integers(1, tot - off + 1))
    if pack_3d:
        off, size = 0, tot
    return lens, strides, BS, off, size, pack_3d


@needs_ref
@pytest.mark.parametrize("seed", range(60))
def test_block_scatter_oracle_bit_exact(seed):
    rng = np.random.default_rng(seed)
    lens, strides, BS, off, size, p3 = _random_scatter_case(rng)
    s1, b1 = oracle.orc_fill_block_scatter(lens, strides, BS, off, size, p3)
    s2, b2 = oracle.ref_fill_block_scatter(lens, strides, BS, off, size, p3)
    assert np.array_equal(s1, s2)
    assert np.array_equal(b1[::BS], b2[::BS])


@needs_ref
@pytest.mark.parametrize("seed", range(60))
def test_block_scatter_product_bit_exact(seed):
    import ctypes
    import tblis_b200 as tb
    rng = np.random.default_rng(seed)
    lens, strides, BS, off, size, p3 = _random_scatter_case(rng)
    n = len(lens)
    L = (ctypes.c_ssize_t * n)(*lens)
    S = (ctypes.c_ssize_t * n)(*strides)
    scat = (ctypes.c_ssize_t * size)()
    bs = (ctypes.c_ssize_t * size)()
    tb.lib.tblis_b200_fill_block_scatter(n, L, S, BS, off, size, scat, bs, int(p3))
    s2, b2 = oracle.ref_fill_block_scatter(lens, strides, BS, off, size, p3)
    assert np.array_equal(np.array(scat[:], dtype=np.int64), s2)
    assert np.array_equal(np.array(bs[:], dtype=np.int64)[::BS], b2[::BS])


@pytest.mark.parametrize("seed", range(40))
def test_product_groups_match_oracle(seed):
    import ctypes
    import tblis_b200 as tb
    rng = np.random.default_rng(500 + seed)
    idx_A, idx_B, idx_C, lens = random_contraction(rng)
    _, A, _ = make_operand(idx_A, lens, rng)
    _, B, _ = make_operand(idx_B, lens, rng)
    _, C, _ = make_operand(idx_C, lens, rng)
    g = oracle.orc_mult_groups(A, idx_A, B, idx_B, C, idx_C)
    va, vb, vc = tb._View(A), tb._View(B), tb._View(C)
    bufs = [ctypes.create_string_buffer(64) for _ in range(4)]
    mnkl = (ctypes.c_int64 * 4)()
    rc = tb.lib.tblis_b200_mult_groups(va.ref, idx_A.encode(), vb.ref, idx_B.encode(), vc.ref,
                                       idx_C.encode(), *bufs, mnkl)
    assert rc == 0
    prod = lambda x: int(np.prod(x)) if len(x) else 1
    for grp, buf, ext in zip(("AB", "AC", "BC", "ABC"), bufs, (mnkl[2], mnkl[0], mnkl[1], mnkl[3])):
        labels = buf.value.decode("latin1")
        assert sorted(labels) == sorted(g[grp]), grp
        assert ext == prod(g["len_" + grp]), grp


def test_library_exports_every_declared_symbol():
    import tblis_b200 as tb
    hdr = open(os.path.join(os.path.dirname(__file__), "..", "include", "tblis_b200.h")).read()
    names = set(re.findall(r"\b(tblis_\w+)\s*\(", hdr))
    assert len(names) >= 25
    for n in sorted(names):
        assert hasattr(tb.lib, n), n


def test_no_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    import tblis_b200 as tb
    rng = np.random.default_rng(0)
    A = rng.uniform(-1, 1, (4, 5))
    B = rng.uniform(-1, 1, (5, 3))
    C = np.zeros((4, 3))
    with pytest.raises(tb.TblisError) as e:
        tb.mult(1.0, A, "ab", B, "bc", 0.0, C, "ac")
    assert e.value.code == 4
    assert np.all(C == 0)
