"""The reference's indexed-DPD contraction (tblis::mult over
indexed_dpd_varray_view, built from its own sources) against the numpy
restatement of its FULL form, on the label mixes the GPU tests use: pins the
semantics (beta through the C entries' factors, factor weighting, index
matching, slicing of dense dimensions by indexed labels) before the GPU path
is compared. Both the reference's default block path and its FULL path."""
import numpy as np
import pytest

import oracle
from tests.idx_dpd_helpers import cases, restated_mult


@pytest.mark.parametrize("name,build", cases())
@pytest.mark.parametrize("beta", [0.0, 1.0, 0.5])
@pytest.mark.parametrize("impl", [0, 2])
def test_reference_matches_full_form(name, build, beta, impl):
    if not oracle.have_ref():
        pytest.skip("reference library not built here")
    rng = np.random.default_rng(sum(map(ord, name)))
    n, A, iA, B, iB, C, iC = build(rng)
    want = restated_mult(n, 0.7, A, iA, B, iB, beta, C, iC)
    oracle.ref_indexed_dpd_mult(n, 0.7, A, iA, B, iB, beta, C, iC, impl=impl)
    assert np.linalg.norm(C["data"] - want) <= 1e-13 * max(1.0, np.linalg.norm(want))
