"""CPU tests: DPD block layout (offsets, lengths, strides) of the product and
of the oracle restatement, pinned bit for bit against the golden vectors of
the reference's MArray test suite and against MArray itself (built from the
reference sources into oracle/_ref)."""
import itertools
import json
import os

import numpy as np
import pytest

import oracle

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "dpd_layout_golden.json")))


@pytest.mark.parametrize("j", range(6))
def test_golden_layouts(j):
    import tblis_b200 as tb
    layout = GOLDEN["layouts"][j]
    t = tb.DpdTensor(GOLDEN["irrep"], GOLDEN["nirrep"], GOLDEN["lens"], layout=layout)
    assert t.size() == 168
    assert oracle.orc_dpd_size(GOLDEN["irrep"], GOLDEN["nirrep"], GOLDEN["lens"], layout) == 168
    for i, irr in enumerate(GOLDEN["blocks"]):
        want = (GOLDEN["block_offsets"][j][i], GOLDEN["block_lengths"][i], GOLDEN["block_strides"][j][i])
        assert t.block(irr) == (want[0], want[1], want[2]), (layout, irr)
        assert oracle.orc_dpd_block(GOLDEN["irrep"], GOLDEN["nirrep"], GOLDEN["lens"], layout, irr) == \
            (want[0], want[1], want[2]), (layout, irr)


def _blocks(nirrep, ndim, irrep):
    """Allowed blocks in the order oracle.ref_dpd_layout lists them (the
    second dimension's irrep fastest, the first closing the XOR)."""
    for rev in itertools.product(range(nirrep), repeat=ndim - 1):
        tail = list(reversed(rev))
        x = irrep
        for t in tail:
            x ^= t
        yield [x] + list(tail)


@pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built")
@pytest.mark.parametrize("seed", range(24))
def test_random_layouts_match_marray(seed):
    import tblis_b200 as tb
    rng = np.random.default_rng(seed)
    nirrep = int(rng.choice([1, 2, 4, 8]))
    ndim = int(rng.integers(1, 5 if nirrep < 8 else 4))
    irrep = int(rng.integers(0, nirrep))
    lens = [[int(rng.integers(0, 5)) for _ in range(nirrep)] for _ in range(ndim)]
    for layout in range(6):
        total, offs, strides = oracle.ref_dpd_layout(irrep, nirrep, lens, layout)
        t = tb.DpdTensor(irrep, nirrep, lens, layout=layout)
        assert t.size() == total
        assert oracle.orc_dpd_size(irrep, nirrep, lens, layout) == total
        for b, irr in enumerate(_blocks(nirrep, ndim, irrep)):
            off, bl, bs = t.block(irr)
            assert off == offs[b] and bs == list(strides[b]), (layout, irr)
            assert bl == [lens[d][irr[d]] for d in range(ndim)]
            assert oracle.orc_dpd_block(irrep, nirrep, lens, layout, irr) == (off, bl, bs)


def test_block_rejects_forbidden_irreps():
    import tblis_b200 as tb
    t = tb.DpdTensor(1, 2, GOLDEN["lens"])
    with pytest.raises(tb.TblisError):
        t.block([0, 0, 0, 0])
