"""DPD and indexed-DPD contractions with batch labels (labels in A, B and C).

The reference routes these through src/internal/3t/dpd/mult.cxx:1082-1115 and
its FULL and BLOCKED alternates (:28-74, :670-847). Its FULL path (dense
round trip) and BLOCKED path (block by block) agree with each other and with
a numpy restatement of C = alpha*A*B + beta*C element-wise along the batch
labels (the CPU test below pins that); its default block path gives other
numbers on these inputs, so the GPU results are compared with FULL and
BLOCKED. Tolerance: plain FP64, 1e-13 normwise relative."""
import copy

import numpy as np
import pytest

import oracle
from tests.idx_dpd_helpers import make, restated_mult
from tests.test_gpu_dpd_cxx import call, driver, load, store, tuples  # noqa: F401 (driver is a fixture)

needs_ref = pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built")

# (A labels, B labels, C labels): one or two batch labels z, y with
# contracted, A-and-C and B-and-C labels present or absent
CASES = [
    ("abz", "bcz", "acz"),
    ("azb", "zbc", "caz"),
    ("abz", "bz", "az"),
    ("az", "bz", "abz"),
    ("bz", "bz", "z"),
    ("abzy", "bcyz", "aczy"),
    ("zab", "bcz", "zac"),
]
IRREPS = [(0, 0, 0), (1, 0, 1), (1, 1, 0), (1, 1, 1)]


def _lens(rng, labels, nirrep):
    return {c: [int(x) for x in rng.integers(0 if c not in "zy" else 1, 4, nirrep)] for c in labels}


def _tensors(seed, case, irreps, nirrep):
    rng = np.random.default_rng(seed)
    iA, iB, iC = case
    L = _lens(rng, set(iA + iB + iC), nirrep)
    A = make(rng, nirrep, irreps[0], [L[c] for c in iA], [], [])
    B = make(rng, nirrep, irreps[1], [L[c] for c in iB], [], [])
    C = make(rng, nirrep, irreps[2], [L[c] for c in iC], [], [])
    return A, B, C


def _reference(nirrep, alpha, A, iA, B, iB, beta, C, iC, impl):
    out = C["data"].copy()
    old = oracle.ref_dpd_impl(impl)
    try:
        oracle.ref_dpd_mult(nirrep, alpha, A["irrep"], A["lens"], A["data"], iA, B["irrep"], B["lens"], B["data"],
                            iB, beta, C["irrep"], C["lens"], out, iC)
    finally:
        oracle.ref_dpd_impl(old)
    return out


def _rel(got, want):
    n = np.linalg.norm(want)
    return np.linalg.norm(got - want) / (n if n else 1.0)


@needs_ref
@pytest.mark.parametrize("case", CASES)
def test_reference_full_and_blocked_agree_with_restatement(case):
    for nirrep in (2, 4):
        for k, irreps in enumerate(IRREPS):
            A, B, C = _tensors(31 + k, case, irreps, nirrep)
            full = _reference(nirrep, 0.5, A, case[0], B, case[1], 2.0, C, case[2], impl=2)
            blocked = _reference(nirrep, 0.5, A, case[0], B, case[1], 2.0, C, case[2], impl=1)
            mine = restated_mult(nirrep, 0.5, A, case[0], B, case[1], 2.0, C, case[2])
            assert _rel(blocked, full) <= 1e-14
            assert _rel(mine, full) <= 1e-14


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("nirrep", [2, 4])
@pytest.mark.parametrize("beta", [0.0, 0.75])
def test_dpd_batch_labels_match_reference(cuda, case, nirrep, beta):
    import torch
    import tblis_b200 as tb
    for k, irreps in enumerate(IRREPS):
        A, B, C = _tensors(100 * nirrep + 7 * k + len(case[0]), case, irreps, nirrep)
        want = _reference(nirrep, 0.5, A, case[0], B, case[1], beta, C, case[2], impl=2)
        tens = []
        for T in (A, B, C):
            t = tb.DpdTensor(T["irrep"], nirrep, T["lens"])
            t.data = torch.from_numpy(T["data"].copy()).to(cuda)
            tens.append(t)
        if beta == 0.0 and len(C["data"]):
            tens[2].data[0] = float("nan")       # beta == 0 never reads C
        tb.dpd_mult(0.5, tens[0], case[0], tens[1], case[1], beta, tens[2], case[2])
        torch.cuda.synchronize()
        got = tens[2].data.cpu().numpy()
        assert np.isfinite(got).all()
        assert _rel(got, want) <= 1e-13, (case, nirrep, irreps)


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("layout", range(6))
def test_dpd_batch_labels_every_storage_layout(driver, layout):
    """The C++ overload (TBLIS's tblis::mult over dpd_varray_view) on every
    MArray storage layout, against the reference's FULL path on the default
    layout."""
    nirrep = 4
    rng = np.random.default_rng(50 + layout)
    iA, iB, iC = "azbe", "ezcb", "zcab"
    L = _lens(rng, "abcez", nirrep)
    lA, lB, lC = [L[c] for c in iA], [L[c] for c in iB], [L[c] for c in iC]
    blocks = [{t: rng.uniform(-1, 1, [l[d][t[d]] for d in range(len(l))]) for t in tuples(0, nirrep, len(l))}
              for l in (lA, lB, lC)]
    dense = [store(0, nirrep, l, 5, b) for l, b in zip((lA, lB, lC), blocks)]
    A = {"irrep": 0, "lens": lA, "data": dense[0]}
    B = {"irrep": 0, "lens": lB, "data": dense[1]}
    C = {"irrep": 0, "lens": lC, "data": dense[2]}
    want = load(0, nirrep, lC, 5, _reference(nirrep, 0.75, A, iA, B, iB, 0.5, C, iC, impl=2))
    args = [dict(irrep=0, lens=l, layout=layout, perm=None, data=store(0, nirrep, l, layout, b), idx=ix)
            for l, b, ix in zip((lA, lB, lC), blocks, (iA, iB, iC))]
    assert call(driver, nirrep, 0.75, args[0], args[1], 0.5, args[2]) == 0
    got = load(0, nirrep, lC, layout, args[2]["data"])
    num = sum(np.sum((got[t] - want[t]) ** 2) for t in want)
    den = sum(np.sum(want[t] ** 2) for t in want)
    assert np.sqrt(num / den) <= 1e-13


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("beta", [0.0, 0.5])
def test_indexed_dpd_batch_label(cuda, beta):
    """Indexed DPD: z dense in all three tensors (a batch label of every
    entry triple), j indexed in B and C; against the reference's FULL path
    and the numpy restatement."""
    import torch
    import tblis_b200 as tb
    rng = np.random.default_rng(77)
    n = 2
    v, o, z = [3, 2], [2, 3], [2, 1]
    A = make(rng, n, 0, [v, z, v], [], [])
    B = make(rng, n, 1, [v, z, v, o], [1], [[0], [2]], factors=[0.5, -1.5])
    C = make(rng, n, 1, [v, z, v, o], [1], [[0], [1], [2]], factors=[1.0, 2.0, -0.25])
    iA, iB, iC = "aze", "ezbj", "azbj"
    want = copy.deepcopy(C)
    oracle.ref_indexed_dpd_mult(n, 0.7, A, iA, B, iB, beta, want, iC, impl=2)
    assert _rel(restated_mult(n, 0.7, A, iA, B, iB, beta, C, iC), want["data"]) <= 1e-14

    def wrap(T):
        data = torch.from_numpy(T["data"].copy()).to(cuda)
        return tb.IndexedDpdTensor(T["irrep"], n, T["lens"], T["idx_irreps"], T["indices"], data, T["factors"]), data
    a, _ = wrap(A)
    b, _ = wrap(B)
    c, dc = wrap(C)
    tb.indexed_dpd_mult(0.7, a, iA, b, iB, beta, c, iC)
    torch.cuda.synchronize()
    assert _rel(dc.cpu().numpy(), want["data"]) <= 1e-13
