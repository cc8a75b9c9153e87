"""GPU parity of the sharded contraction: every rank's slab (run one after
another on one GPU; the slabs are independent launches, nothing waits on
another rank) assembles the contraction the oracle computes."""
import numpy as np
import pytest

import oracle
from tests.helpers import normwise_rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nranks", [2, 3, 8])
@pytest.mark.parametrize("case", [("abef", "efij", "abij", (24, 20, 24, 20, 6, 5)),
                                  ("aeim", "mbej", "aibj", (20, 9, 6, 7, 18, 5))])
def test_slabs_assemble_the_contraction(cuda, nranks, case):
    import torch
    import tblis_b200 as tb
    iA, iB, iC, ext = case
    L = dict(zip(sorted(set(iA + iB + iC)), ext))
    rng = np.random.default_rng(nranks)
    A = rng.uniform(-1, 1, [L[c] for c in iA])
    B = rng.uniform(-1, 1, [L[c] for c in iB])
    C = rng.uniform(-1, 1, [L[c] for c in iC])
    want = C.copy()
    oracle.orc_mult(0.75, A, iA, B, iB, -0.5, want, iC)
    dA, dB, dC = (torch.from_numpy(x).to(cuda) for x in (A, B, C))
    for r in range(nranks):
        tb.mult_shard(0.75, dA, iA, dB, iB, -0.5, dC, iC, rank=r, nranks=nranks)
    torch.cuda.synchronize()
    assert normwise_rel(dC.cpu().numpy(), want) <= 1e-14


def test_complex_slabs(cuda):
    import torch
    import tblis_b200 as tb
    rng = np.random.default_rng(4)
    A = rng.uniform(-1, 1, (30, 12)) + 1j * rng.uniform(-1, 1, (30, 12))
    B = rng.uniform(-1, 1, (12, 17)) + 1j * rng.uniform(-1, 1, (12, 17))
    C = rng.uniform(-1, 1, (30, 17)) + 1j * rng.uniform(-1, 1, (30, 17))
    want = (0.5 - 1j) * (A @ B) + (0.25 + 0.5j) * C
    dA, dB, dC = (torch.from_numpy(x).to(cuda) for x in (A, B, C))
    for r in range(4):
        tb.mult_shard(0.5 - 1j, dA, "ak", dB, "kb", 0.25 + 0.5j, dC, "ab", rank=r, nranks=4)
    torch.cuda.synchronize()
    assert normwise_rel(dC.cpu().numpy(), want) <= 1e-14
