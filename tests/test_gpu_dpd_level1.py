"""GPU parity of the DPD level-1 operations (tblis::add / dot / reduce /
scale / set / shift over dpd_varray_view) against the reference's own, on
the same default-layout storage: transposes, traces over A-only labels,
replication over B-only labels, an irrep mismatch that only scales, every
reduction (value and offset) and the unary updates."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

REDUCE = {"SUM": 0, "SUM_ABS": 1, "MAX": 2, "MAX_ABS": 3, "MIN": 4, "MIN_ABS": 5, "NORM_2": 6}


def _lens(rng, nirrep, lo=1, hi=5):
    return [int(x) for x in rng.integers(lo, hi, nirrep)]


def _dpd(tb, rng, irrep, nirrep, lens, device=None):
    import torch
    T = tb.DpdTensor(irrep, nirrep, lens)
    data = rng.uniform(-1, 1, max(1, T.size()))
    T.data = torch.from_numpy(data).to(device) if device is not None else data
    return T


def _np(T):
    return T.data.cpu().numpy() if hasattr(T.data, "cpu") else T.data


@pytest.mark.parametrize("case", ["transpose", "trace", "replicate", "mismatch", "beta0"])
def test_add(cuda, case):
    import tblis_b200 as tb
    rng = np.random.default_rng(["transpose", "trace", "replicate", "mismatch", "beta0"].index(case))
    n = 4
    a, b, c = _lens(rng, n), _lens(rng, n), _lens(rng, n)
    if case in ("transpose", "mismatch", "beta0"):
        lA, iA, lB, iB = [a, b, c], "abc", [c, a, b], "cab"
    elif case == "trace":
        lA, iA, lB, iB = [a, b, c], "abc", [b, a], "ba"
    else:
        lA, iA, lB, iB = [a, b], "ab", [b, c, a], "bca"
    irrA, irrB = (1, 1) if case != "mismatch" else (1, 2)
    if case == "trace":
        irrB = 3
    A = _dpd(tb, rng, irrA, n, lA, cuda if case == "transpose" else None)
    B = _dpd(tb, rng, irrB, n, lB, cuda if case == "transpose" else None)
    alpha, beta = 0.75, (0.0 if case == "beta0" else -1.25)
    wantB = _np(B).copy()
    oracle.ref_dpd_add(n, alpha, irrA, lA, _np(A).copy(), iA, beta, irrB, lB, wantB, iB)
    tb.dpd_add(alpha, A, iA, beta, B, iB)
    got = _np(B)
    assert np.linalg.norm(got - wantB) <= 1e-14 * max(1.0, np.linalg.norm(wantB)), case


def test_dot(cuda):
    import tblis_b200 as tb
    rng = np.random.default_rng(11)
    n = 8
    a, b, c = _lens(rng, n, 0, 4), _lens(rng, n, 1, 4), _lens(rng, n, 1, 3)
    A = _dpd(tb, rng, 5, n, [a, b, c])
    B = _dpd(tb, rng, 5, n, [c, a, b])
    want = oracle.ref_dpd_dot(n, 5, [a, b, c], A.data, "abc", 5, [c, a, b], B.data, "cab")
    got = tb.dpd_dot(A, "abc", B, "cab")
    assert abs(got - want) <= 1e-13 * max(1.0, abs(want))


@pytest.mark.parametrize("op", sorted(REDUCE))
def test_reduce(cuda, op):
    import tblis_b200 as tb
    rng = np.random.default_rng(REDUCE[op])
    n = 4
    lens = [_lens(rng, n), _lens(rng, n), _lens(rng, n)]
    A = _dpd(tb, rng, 2, n, lens)
    want, wi = oracle.ref_dpd_reduce(REDUCE[op], n, 2, lens, A.data, "abc")
    got, gi = tb.dpd_reduce(REDUCE[op], A, "abc")
    assert abs(got - want) <= 1e-13 * max(1.0, abs(want))
    if op not in ("SUM", "SUM_ABS", "NORM_2"):
        assert gi == wi


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_unary(cuda, kind):
    import tblis_b200 as tb
    rng = np.random.default_rng(20 + kind)
    n = 2
    lens = [_lens(rng, n), _lens(rng, n), _lens(rng, n), _lens(rng, n)]
    A = _dpd(tb, rng, 1, n, lens)
    want = A.data.copy()
    oracle.ref_dpd_unary(kind, 0.3, -2.0, n, 1, lens, want, "abcd")
    if kind == 0:
        tb.dpd_scale(0.3, A, "abcd")
    elif kind == 1:
        tb.dpd_set(0.3, A, "abcd")
    else:
        tb.dpd_shift(0.3, -2.0, A, "abcd")
    assert np.linalg.norm(A.data - want) <= 1e-14 * max(1.0, np.linalg.norm(want))
