"""GPU parity of the indexed-DPD contraction (tblis_b200_indexed_dpd_mult,
the entry of tblis::mult over indexed_dpd_varray_view) against the
reference's own indexed-DPD contraction on the same storage: label mixes with
indexed labels in the output, contracted over, or slicing a dense dimension,
entry factors including zero, and every kind of beta."""
import copy

import numpy as np
import pytest

import oracle
from tests.idx_dpd_helpers import cases

pytestmark = pytest.mark.gpu


def _gpu(torch, dev, nirrep, alpha, A, iA, B, iB, beta, C, iC):
    import tblis_b200 as tb

    def wrap(T):
        data = torch.from_numpy(T["data"]).to(dev)
        t = tb.IndexedDpdTensor(T["irrep"], nirrep, T["lens"], T["idx_irreps"], T["indices"], data, T["factors"])
        assert t.dense_size() * t.nidx == len(T["data"])
        return t, data
    a, _ = wrap(A)
    b, _ = wrap(B)
    c, dc = wrap(C)
    rep = tb.indexed_dpd_mult(alpha, a, iA, b, iB, beta, c, iC)
    torch.cuda.synchronize()
    return dc.cpu().numpy(), rep


@pytest.mark.parametrize("name,build", cases())
@pytest.mark.parametrize("beta", [0.0, 1.0, 0.5])
def test_matches_reference(cuda, name, build, beta):
    import torch
    rng = np.random.default_rng(sum(map(ord, name)) + 7)
    n, A, iA, B, iB, C, iC = build(rng)
    want = copy.deepcopy(C)
    oracle.ref_indexed_dpd_mult(n, 0.7, A, iA, B, iB, beta, want, iC, impl=0)
    got, rep = _gpu(torch, cuda, n, 0.7, A, iA, B, iB, beta, C, iC)
    scale = max(1.0, np.linalg.norm(want["data"]))
    assert np.linalg.norm(got - want["data"]) <= 1e-13 * scale, name


def test_zero_factor_and_host_storage(cuda):
    """A zero C factor clears its entry; host (numpy) storage is staged."""
    import tblis_b200 as tb
    rng = np.random.default_rng(5)
    n, A, iA, B, iB, C, iC = dict(cases())["ladder_indexed_j"](rng)
    C["factors"] = [0.0, 1.0, 2.0]
    want = copy.deepcopy(C)
    oracle.ref_indexed_dpd_mult(n, 1.0, A, iA, B, iB, 0.25, want, iC, impl=0)
    mk = lambda T: tb.IndexedDpdTensor(T["irrep"], n, T["lens"], T["idx_irreps"], T["indices"], T["data"],
                                       T["factors"])
    c = mk(C)
    tb.indexed_dpd_mult(1.0, mk(A), iA, mk(B), iB, 0.25, c, iC)
    assert np.linalg.norm(C["data"] - want["data"]) <= 1e-13 * max(1.0, np.linalg.norm(want["data"]))


def test_mismatched_indexed_irreps_only_scale(cuda):
    """Labels indexed with different irreps in two tensors contribute
    nothing: C is only scaled (src/internal/3t/indexed_dpd/mult.cxx:1226-1280)."""
    import torch
    from tests.idx_dpd_helpers import make
    rng = np.random.default_rng(9)
    n, A, iA, B, iB, _, iC = dict(cases())["ladder_indexed_j"](rng)
    v, o = [3, 2], [2, 3]
    # j indexed with irrep 1 in B but irrep 0 in C
    C = make(rng, n, 0, [v, v, o, o], [0], [[0], [1]], factors=[1.0, 3.0])
    want = copy.deepcopy(C)
    oracle.ref_indexed_dpd_mult(n, 1.0, A, iA, B, iB, 0.5, want, iC, impl=0)
    got, rep = _gpu(torch, cuda, n, 1.0, A, iA, B, iB, 0.5, C, iC)
    assert np.linalg.norm(got - want["data"]) <= 1e-14 * max(1.0, np.linalg.norm(want["data"]))
    assert rep["m"] == 0


@pytest.mark.parametrize("dtype", ["float64", "complex128"])
def test_triples_share_launches(cuda, dtype):
    """C[abij] (j indexed, 3 entries) = A[abem] (m indexed, 3 entries) *
    B[eimj] (m and j indexed, 9 entries): 9 consistent triples, 3 on each
    entry of C, run in 3 grouped launches (the k-th triple of every entry of
    C in the k-th launch) with the reference's result. dcomplex: the 4 real
    products of each triple into each part of C (complex alpha) make 12
    launches for the 72 real terms."""
    import torch
    from tests.idx_dpd_helpers import make, restated_mult
    rng = np.random.default_rng(21)
    n = 2
    v, o = [3, 2], [2, 3]
    A = make(rng, n, 1, [v, v, v, o], [1], [[0], [1], [2]], factors=[1.0, -0.5, 2.0])
    B = make(rng, n, 1, [v, o, o, o], [1, 1], [[m, j] for m in range(3) for j in range(3)])
    C = make(rng, n, 0, [v, v, o, o], [1], [[0], [1], [2]], factors=[1.0, 0.25, -1.0])
    if dtype == "float64":
        alpha = 0.75
        want = copy.deepcopy(C)
        oracle.ref_indexed_dpd_mult(n, alpha, A, "abem", B, "eimj", 0.5, want, "abij", impl=0)
        want = want["data"]
    else:
        alpha = 0.75 - 0.25j
        for T in (A, B, C):
            T["data"] = T["data"] + 1j * rng.uniform(-1, 1, T["data"].shape)
        want = restated_mult(n, alpha, A, "abem", B, "eimj", 0.5, C, "abij")
    got, rep = _gpu(torch, cuda, n, alpha, A, "abem", B, "eimj", 0.5, C, "abij")
    assert np.linalg.norm(got - want) <= 1e-13 * max(1.0, np.linalg.norm(want))
    assert rep["m"] == (3 if dtype == "float64" else 12)


def test_cxx_overload_matches_reference(cuda):
    """tblis::mult over indexed_dpd_varray_view through its mangled C++ name
    (libtblis_b200_cxx.so), on owning MArray tensors as a TBLIS program has."""
    import ctypes
    import os
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "cxx", "_bin",
                        "libdpd_driver.so")
    assert os.path.exists(path), "C++ test driver not built (make -C tests/cxx MARRAY=...)"
    drv = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
    sz = ctypes.c_ssize_t
    for name, build in cases():
        rng = np.random.default_rng(sum(map(ord, name)) + 11)
        n, A, iA, B, iB, C, iC = build(rng)
        want = copy.deepcopy(C)
        oracle.ref_indexed_dpd_mult(n, 1.25, A, iA, B, iB, 0.5, want, iC, impl=0)

        def args(T, lab):
            nidim = len(T["idx_irreps"])
            idx = [x for t in T["indices"] for x in t]
            nidx = max(1, len(T["indices"])) if nidim else 1
            return [ctypes.c_uint(T["irrep"]), ctypes.c_uint(len(T["lens"])),
                    (sz * (len(T["lens"]) * n))(*[x for r in T["lens"] for x in r]), ctypes.c_uint(nidim),
                    (ctypes.c_uint * max(1, nidim))(*T["idx_irreps"]), ctypes.c_long(nidx),
                    (sz * max(1, len(idx)))(*idx), ctypes.c_void_p(T["data"].ctypes.data),
                    (ctypes.c_double * nidx)(*T["factors"]), lab.encode()]
        rc = drv.driver_indexed_dpd_mult(ctypes.c_uint(n), ctypes.c_double(1.25), *args(A, iA), *args(B, iB),
                                         ctypes.c_double(0.5), *args(C, iC))
        assert rc == 0, name
        assert np.linalg.norm(C["data"] - want["data"]) <= 1e-13 * max(1.0, np.linalg.norm(want["data"])), name


# ---- level-1 ------------------------------------------------------------------------

def _wrap(tb, torch, dev, n, T):
    data = torch.from_numpy(T["data"]).to(dev)
    return tb.IndexedDpdTensor(T["irrep"], n, T["lens"], T["idx_irreps"], T["indices"], data, T["factors"]), data


def _l1_cases():
    from tests.idx_dpd_helpers import make

    def transpose(rng):
        # B[jba] (j indexed in both) = A[abj]
        n = 2
        a, b, j = [2, 3], [3, 1], [2, 2]
        A = make(rng, n, 1, [a, b, j], [1], [[0], [1]], factors=[1.0, -0.5])
        B = make(rng, n, 1, [b, a, j], [1], [[1], [0]], factors=[2.0, 0.0])
        return n, A, "abj", B, "baj"

    def sliced(rng):
        # j indexed in A, dense in B: each A entry adds into one slice of B
        n = 2
        a, j = [2, 3], [2, 2]
        A = make(rng, n, 1, [a, j], [1], [[0], [1]], factors=[1.5, 1.0])
        B = make(rng, n, 1, [a, j], [], [])
        return n, A, "aj", B, "aj"

    def trace(rng):
        # B[a] = sum_c A[ac], c indexed in A
        n = 2
        a, c = [3, 2], [2, 1]
        A = make(rng, n, 0, [a, c], [0], [[0], [1]], factors=[1.0, 2.0])
        B = make(rng, n, 0, [a], [], [])
        return n, A, "ac", B, "a"
    return [("transpose", transpose), ("sliced", sliced), ("trace", trace)]


@pytest.mark.parametrize("name,build", _l1_cases())
@pytest.mark.parametrize("beta", [0.0, 1.0, -0.5])
def test_level1_add(cuda, name, build, beta):
    import torch
    import tblis_b200 as tb
    rng = np.random.default_rng(sum(map(ord, name)))
    n, A, iA, B, iB = build(rng)
    want = copy.deepcopy(B)
    oracle.ref_indexed_dpd_add(n, 0.75, A, iA, beta, want, iB)
    a, _ = _wrap(tb, torch, cuda, n, A)
    b, db = _wrap(tb, torch, cuda, n, B)
    tb.indexed_dpd_add(0.75, a, iA, beta, b, iB)
    got = db.cpu().numpy()
    assert np.linalg.norm(got - want["data"]) <= 1e-14 * max(1.0, np.linalg.norm(want["data"])), name


@pytest.mark.parametrize("name,build", _l1_cases()[:2])
def test_level1_dot(cuda, name, build):
    import torch
    import tblis_b200 as tb
    rng = np.random.default_rng(3 + sum(map(ord, name)))
    n, A, iA, B, iB = build(rng)
    want = oracle.ref_indexed_dpd_dot(n, A, iA, B, iB)
    a, _ = _wrap(tb, torch, cuda, n, A)
    b, _ = _wrap(tb, torch, cuda, n, B)
    got = tb.indexed_dpd_dot(a, iA, b, iB)
    assert abs(got - want) <= 1e-13 * max(1.0, abs(want))


@pytest.mark.parametrize("op", range(7))
def test_level1_reduce(cuda, op):
    import torch
    import tblis_b200 as tb
    from tests.idx_dpd_helpers import make
    rng = np.random.default_rng(40 + op)
    n = 4
    A = make(rng, n, 3, [[2, 1, 3, 2], [1, 2, 2, 1], [2, 2, 1, 3]], [3], [[0], [2]], factors=[-0.5, 1.5])
    want, wi = oracle.ref_indexed_dpd_reduce(op, n, A, "abc")
    a, _ = _wrap(tb, torch, cuda, n, A)
    got, gi = tb.indexed_dpd_reduce(op, a, "abc")
    assert abs(got - want) <= 1e-13 * max(1.0, abs(want)), op
    if op not in (0, 1, 6):
        assert gi == wi


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_level1_unary(cuda, kind):
    import torch
    import tblis_b200 as tb
    from tests.idx_dpd_helpers import make
    rng = np.random.default_rng(50 + kind)
    n = 2
    A = make(rng, n, 1, [[2, 3], [3, 1], [2, 2]], [1], [[0], [1]], factors=[0.0, 1.5])
    want = copy.deepcopy(A)
    oracle.ref_indexed_dpd_unary(kind, 0.3, -2.0, n, want, "abc")
    a, da = _wrap(tb, torch, cuda, n, A)
    if kind == 0:
        tb.indexed_dpd_scale(0.3, a, "abc")
    elif kind == 1:
        tb.indexed_dpd_set(0.3, a, "abc")
    else:
        tb.indexed_dpd_shift(0.3, -2.0, a, "abc")
    got = da.cpu().numpy()
    assert np.linalg.norm(got - want["data"]) <= 1e-14 * max(1.0, np.linalg.norm(want["data"]))
