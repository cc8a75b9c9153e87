"""GPU parity of the DPD and indexed-DPD paths for float, scomplex and
dcomplex storage. DPD contraction and level-1 are compared against the
reference's own tblis::mult / add / dot / reduce / scale / set / shift over
dpd_varray_view of the same element type (src/iface/3t/mult.cxx:170-298,
src/iface/1t/*.cxx). Indexed DPD is compared against the FULL-form
restatement that the double path is pinned with, carried out in complex
arithmetic with complex factors."""
import numpy as np
import pytest

import oracle
from tests import idx_dpd_helpers as H

pytestmark = pytest.mark.gpu

DTYPES = [np.float32, np.complex64, np.complex128]
TOL = {np.float32: 3e-6, np.complex64: 3e-6, np.complex128: 1e-13}
REDUCE = {"SUM": 0, "SUM_ABS": 1, "MAX": 2, "MAX_ABS": 3, "MIN": 4, "MIN_ABS": 5, "NORM_2": 6}


def values(rng, n, dtype):
    v = rng.uniform(-1, 1, n)
    if np.dtype(dtype).kind == "c":
        v = v + 1j * rng.uniform(-1, 1, n)
    return v.astype(dtype)


def scalar(dtype, v):
    return complex(v) if np.dtype(dtype).kind == "c" else complex(v).real


def dpd(tb, rng, irrep, nirrep, lens, dtype, device=None):
    import torch
    T = tb.DpdTensor(irrep, nirrep, lens)
    data = values(rng, max(1, T.size()), dtype)
    T = tb.DpdTensor(irrep, nirrep, lens, data=torch.from_numpy(data).to(device) if device is not None else data)
    return T


def host(T):
    return T.data.cpu().numpy() if hasattr(T.data, "cpu") else T.data


def rel(got, want):
    d = np.linalg.norm((np.asarray(got) - np.asarray(want)).ravel())
    n = np.linalg.norm(np.asarray(want).ravel())
    return d / n if n > 0 else d


def ladder(rng, nirrep=4):
    occ = [int(x) for x in rng.integers(1, 5, nirrep)]
    vir = [int(x) for x in rng.integers(2, 8, nirrep)]
    return [vir, vir, vir, vir], [vir, vir, occ, occ], [vir, vir, occ, occ]


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("beta", [0.0, 0.5 - 0.75j])
@pytest.mark.parametrize("on_device", [True, False])
def test_dpd_mult(cuda, dtype, beta, on_device):
    import tblis_b200 as tb
    rng = np.random.default_rng(3)
    n = 4
    lA, lB, lC = ladder(rng, n)
    dev = cuda if on_device else None
    A = dpd(tb, rng, 0, n, lA, dtype, dev)
    B = dpd(tb, rng, 0, n, lB, dtype, dev)
    C = dpd(tb, rng, 0, n, lC, dtype, dev)
    alpha, beta = scalar(dtype, 0.75 + 0.25j), scalar(dtype, beta)
    want = host(C).copy()
    oracle.ref_dpd_mult_typed(n, alpha, 0, lA, host(A).copy(), "abef", 0, lB, host(B).copy(), "efij",
                              beta, 0, lC, want, "abij")
    tb.dpd_mult(alpha, A, "abef", B, "efij", beta, C, "abij")
    assert rel(host(C), want) <= TOL[dtype] * 3


@pytest.mark.parametrize("dtype", DTYPES)
def test_dpd_mult_ring_nonzero_irreps(cuda, dtype):
    """Ring-type labels interleave in the layout tree; non-zero irreps."""
    import tblis_b200 as tb
    rng = np.random.default_rng(300)
    n = 2
    o, v = [3, 2], [4, 5]
    lA, lB, lC = [v, v, o, o], [o, v, v, o], [v, o, v, o]
    A = dpd(tb, rng, 1, n, lA, dtype, cuda)
    B = dpd(tb, rng, 1, n, lB, dtype, cuda)
    C = dpd(tb, rng, 0, n, lC, dtype, cuda)
    alpha, beta = scalar(dtype, 1.0 - 0.5j), scalar(dtype, 1.0)
    want = host(C).copy()
    oracle.ref_dpd_mult_typed(n, alpha, 1, lA, host(A).copy(), "aeim", 1, lB, host(B).copy(), "mbej",
                              beta, 0, lC, want, "aibj")
    tb.dpd_mult(alpha, A, "aeim", B, "mbej", beta, C, "aibj")
    assert rel(host(C), want) <= TOL[dtype] * 3


ADD = {
    "transpose": ("abc", "cab"),
    "trace": ("abc", "ba"),
    "replicate": ("ab", "bca"),
}


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("case", list(ADD))
def test_dpd_add(cuda, dtype, case):
    import tblis_b200 as tb
    rng = np.random.default_rng(list(ADD).index(case))
    n = 4
    lens = {c: [int(x) for x in rng.integers(1, 5, n)] for c in "abc"}
    iA, iB = ADD[case]
    lA, lB = [lens[c] for c in iA], [lens[c] for c in iB]
    irrA, irrB = 1, (3 if case == "trace" else 1)
    A = dpd(tb, rng, irrA, n, lA, dtype, cuda)
    B = dpd(tb, rng, irrB, n, lB, dtype, cuda)
    alpha, beta = scalar(dtype, 0.75 - 1j), scalar(dtype, -1.25 + 0.5j)
    want = host(B).copy()
    oracle.ref_dpd_level1_typed("add", n, irrA, lA, host(A).copy(), iA, irrB, lB, want, iB, alpha, beta)
    tb.dpd_add(alpha, A, iA, beta, B, iB)
    assert rel(host(B), want) <= TOL[dtype] * 3


@pytest.mark.parametrize("dtype", DTYPES)
def test_dpd_dot_reduce(cuda, dtype):
    import tblis_b200 as tb
    rng = np.random.default_rng(11)
    n = 8
    lens = [[int(x) for x in rng.integers(1, 4, n)] for _ in range(3)]
    A = dpd(tb, rng, 5, n, lens, dtype, cuda)
    B = dpd(tb, rng, 5, n, [lens[1], lens[0], lens[2]], dtype, cuda)
    want = oracle.ref_dpd_level1_typed("dot", n, 5, lens, host(A).copy(), "abc", 5, [lens[1], lens[0], lens[2]],
                                       host(B).copy(), "bac")
    got = tb.dpd_dot(A, "abc", B, "bac")
    scale = np.linalg.norm(host(A)) * np.linalg.norm(host(B))
    assert abs(got - want) <= TOL[dtype] * 10 * scale
    for name, op in REDUCE.items():
        wv, wi = oracle.ref_dpd_level1_typed(("reduce", op), n, 5, lens, host(A).copy(), "abc")
        gv, gi = tb.dpd_reduce(op, A, "abc")
        assert abs(gv - wv) <= TOL[dtype] * 40 * max(1.0, abs(wv)), name
        if op in (2, 3, 4, 5):
            assert gi == wi, name


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("kind", ["scale", "set", "shift"])
def test_dpd_unary(cuda, dtype, kind):
    import tblis_b200 as tb
    rng = np.random.default_rng(21)
    n = 4
    lens = [[int(x) for x in rng.integers(1, 5, n)] for _ in range(3)]
    A = dpd(tb, rng, 2, n, lens, dtype, cuda)
    alpha, beta = scalar(dtype, 0.5 + 2j), scalar(dtype, -1.5 + 0.25j)
    want = host(A).copy()
    oracle.ref_dpd_level1_typed(kind, n, 2, lens, want, "abc", alpha=alpha, beta=beta)
    if kind == "scale":
        tb.dpd_scale(alpha, A, "abc")
    elif kind == "set":
        tb.dpd_set(alpha, A, "abc")
    else:
        tb.dpd_shift(alpha, beta, A, "abc")
    assert rel(host(A), want) <= TOL[dtype]


def _typed(T, rng, dtype):
    T = dict(T)
    T["data"] = values(rng, T["data"].size, dtype)
    if np.dtype(dtype).kind == "c":
        T["factors"] = [complex(f) * complex(1.0, 0.5 * (i % 3 - 1)) for i, f in enumerate(T["factors"])]
    return T


def _idx(tb, T, dtype, device):
    import torch
    data = torch.from_numpy(np.ascontiguousarray(T["data"])).to(device)
    return tb.IndexedDpdTensor(T["irrep"], N_IRREP[0], T["lens"], T["idx_irreps"], T["indices"], data=data,
                               factors=T["factors"])


N_IRREP = [0]


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("case", [c[0] for c in H.cases()])
def test_indexed_dpd_mult(cuda, dtype, case):
    import tblis_b200 as tb
    build = dict(H.cases())[case]
    rng = np.random.default_rng(7)
    n, A, iA, B, iB, C, iC = build(rng)
    A, B, C = _typed(A, rng, dtype), _typed(B, rng, dtype), _typed(C, rng, dtype)
    alpha, beta = scalar(dtype, 0.5 - 0.25j), scalar(dtype, 0.75 + 0.5j)
    want = H.restated_mult(n, alpha, A, iA, B, iB, beta, C, iC)
    N_IRREP[0] = n
    dA, dB, dC = _idx(tb, A, dtype, cuda), _idx(tb, B, dtype, cuda), _idx(tb, C, dtype, cuda)
    tb.indexed_dpd_mult(alpha, dA, iA, dB, iB, beta, dC, iC)
    got = dC.data.cpu().numpy()
    assert rel(got, want) <= TOL[dtype] * 3, case


@pytest.mark.parametrize("dtype", DTYPES)
def test_indexed_dpd_level1(cuda, dtype):
    """Indexed level-1 on complex / float entries: dot and scale through the
    entries' factors, checked on the FULL form."""
    import tblis_b200 as tb
    rng = np.random.default_rng(31)
    n, A, iA, B, iB, C, iC = dict(H.cases())["ladder_indexed_j"](rng)
    Bt = _typed(B, rng, dtype)
    N_IRREP[0] = n
    dB = _idx(tb, Bt, dtype, cuda)
    F = H.full(Bt, n)
    got = tb.indexed_dpd_dot(dB, iB, dB, iB)
    want = np.sum(F * F)
    assert abs(got - want) <= TOL[dtype] * 10 * max(1.0, np.sum(np.abs(F) ** 2))
    s = scalar(dtype, 1.5 - 0.5j)
    tb.indexed_dpd_scale(s, dB, iB)
    size, _ = H.dense_geometry(Bt, n)
    want = Bt["data"].astype(np.complex128 if np.dtype(dtype).kind == "c" else np.float64).copy()
    for e in range(len(Bt["indices"])):
        f = Bt["factors"][e]
        want[e * size:(e + 1) * size] *= (f * s) if f != 0 else 0.0
    assert rel(dB.data.cpu().numpy(), want) <= TOL[dtype]
