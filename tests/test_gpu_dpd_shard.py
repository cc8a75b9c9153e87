"""GPU parity of the sharded DPD contraction on one GPU: every rank's share
(tblis_b200_dpd_mult_shard) runs in turn on the same C, and the shares
assemble the reference's whole DPD contraction (its FULL path); one share alone changes
only its own blocks. (Several GPUs are not available here; the rank logic
itself is tested with gloo ranks on CPU.)"""
import numpy as np
import pytest
import torch

import oracle
from tests.test_dpd_shard import CASES, _reference, _tensors

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built")]


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("nranks", [2, 3, 8])
def test_shares_assemble_the_reference(cuda, case, nranks):
    import tblis_b200 as tb
    (iA, iB, iC), irr, (A, B, C), (a, b, c) = _tensors(case, seed=5)
    want = _reference(irr, (A, B, C), (a, b, c), (iA, iB, iC), 0.5, -1.5)
    A.data, B.data = torch.from_numpy(a).to(cuda), torch.from_numpy(b).to(cuda)
    C.data = torch.from_numpy(c.copy()).to(cuda)
    owner, _ = tb.dpd_shard_plan(A, iA, B, iB, C, iC, nranks)
    for r in range(nranks):
        before = C.data.cpu().numpy()
        tb.dpd_mult_shard(0.5, A, iA, B, iB, -1.5, C, iC, rank=r, nranks=nranks)
        torch.cuda.synchronize()
        after = C.data.cpu().numpy()
        # blocks of other ranks are untouched by this share
        for t, o in owner.items():
            if o == r:
                continue
            off, Ls, S = C.block(t)
            if np.prod(Ls) == 0:
                continue
            idx = off + (np.asarray(S)[:, None] * np.indices(Ls).reshape(len(Ls), -1)).sum(0)
            assert np.array_equal(after[idx], before[idx]), (t, o, r)
    got = C.data.cpu().numpy()
    assert np.linalg.norm(got - want) <= 1e-13 * np.linalg.norm(want)
