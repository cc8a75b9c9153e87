"""CPU pin of the oracle's dense-form restatement (orc_dpd_block_to_full /
orc_dpd_full_to_block, src/internal/1t/dpd/util.hpp:70-133).

The reference's FULL DPD contraction (src/internal/3t/dpd/mult.cxx:28-74) is
block_to_full of A, B and C, one dense contraction, then full_to_block of C.
Running the same three steps with the restatement and numpy's einsum must
give the reference's FULL result. The restatement also inverts itself: a DPD
tensor survives the round trip, and block_to_full covers exactly the
symmetry-allowed blocks (everything else is zero)."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built")

CASES = [
    # nirrep, (irrep_A, lens_A, idx_A), (irrep_B, lens_B, idx_B), idx_C
    (2, (0, [[3, 2], [2, 3], [1, 2]], "abe"), (1, [[1, 2], [2, 1], [1, 2]], "ecd"), "abcd"),
    (4, (1, [[2, 1, 3, 2], [3, 1, 2, 1]], "ae"), (2, [[3, 1, 2, 1], [1, 2, 2, 3]], "eb"), "ab"),
    (4, (0, [[2, 1, 2, 1], [1, 2, 1, 2], [2, 2, 1, 1], [1, 1, 2, 2]], "abef"),
        (0, [[2, 2, 1, 1], [1, 1, 2, 2], [2, 1, 1, 2], [1, 2, 2, 1]], "efij"), "abij"),
]


def _lens_of(label, idx_list, lens_list):
    for idx, lens in zip(idx_list, lens_list):
        if label in idx:
            return lens[idx.index(label)]
    raise KeyError(label)


@pytest.mark.parametrize("case", range(len(CASES)))
def test_full_contraction_through_restatement_matches_reference(case):
    nirrep, (ia, la, xa), (ib, lb, xb), xc = CASES[case]
    lc = [_lens_of(c, [xa, xb], [la, lb]) for c in xc]
    ic = ia ^ ib
    rng = np.random.default_rng(case)
    A = rng.uniform(-1, 1, oracle.orc_dpd_size(ia, nirrep, la, 5))
    B = rng.uniform(-1, 1, oracle.orc_dpd_size(ib, nirrep, lb, 5))
    C0 = rng.uniform(-1, 1, oracle.orc_dpd_size(ic, nirrep, lc, 5))
    # the reference's FULL path
    want = C0.copy()
    prev = oracle.ref_dpd_impl(2)
    try:
        oracle.ref_dpd_mult(nirrep, 0.75, ia, la, A, xa, ib, lb, B, xb, 0.5, ic, lc, want, xc)
    finally:
        oracle.ref_dpd_impl(prev)
    # the same steps with the restatement
    FA = oracle.orc_dpd_block_to_full(ia, nirrep, la, A)
    FB = oracle.orc_dpd_block_to_full(ib, nirrep, lb, B)
    FC = oracle.orc_dpd_block_to_full(ic, nirrep, lc, C0)
    FC = 0.75 * np.einsum("%s,%s->%s" % (xa, xb, xc), FA, FB) + 0.5 * FC
    got = C0.copy()
    oracle.orc_dpd_full_to_block(ic, nirrep, lc, FC, got)
    assert np.linalg.norm(got - want) <= 1e-13 * max(1.0, np.linalg.norm(want))


@pytest.mark.parametrize("case", range(len(CASES)))
def test_round_trip_and_zeros_outside_blocks(case):
    nirrep, (ia, la, _), _, _ = CASES[case]
    size = oracle.orc_dpd_size(ia, nirrep, la, 5)
    data = np.arange(1, size + 1, dtype=np.float64)
    F = oracle.orc_dpd_block_to_full(ia, nirrep, la, data)
    assert np.count_nonzero(F) == size and F.sum() == data.sum()
    back = np.zeros(size)
    oracle.orc_dpd_full_to_block(ia, nirrep, la, F, back)
    assert np.array_equal(back, data)
