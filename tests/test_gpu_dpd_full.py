"""GPU tests of the dense form of a DPD tensor and back
(tblis_b200_dpd_block_to_full / tblis_b200_dpd_full_to_block, the reference's
block_to_full / full_to_block, src/internal/1t/dpd/util.hpp:70-133).

Both are plain copies, so results must equal the oracle's restatement bit for
bit. The oracle takes every block's offset and strides from the reference's
own MArray layout. The dense tensors carry NaN before block_to_full (it
must zero what no block covers) and have permuted strides in some cases."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

CASES = [
    # (nirrep, irrep, lens per dimension per irrep)
    (2, 0, [[2, 3], [3, 1], [2, 2]]),
    (2, 1, [[4, 2], [1, 3]]),
    (4, 0, [[2, 1, 3, 2], [3, 2, 1, 2], [1, 2, 2, 3], [2, 2, 1, 1]]),
    (4, 3, [[3, 0, 2, 1], [2, 2, 0, 3], [1, 3, 2, 2]]),
    (8, 0, [[3, 2, 1, 2, 3, 1, 2, 2], [2, 1, 3, 1, 2, 2, 1, 3], [1, 2, 2, 1, 3, 1, 2, 1]]),
    (8, 5, [[2, 1, 2, 3, 1, 2, 1, 1], [1, 2, 1, 2, 2, 1, 3, 1]]),
]


def _dense(torch, cuda, dims, permuted, fill):
    if permuted:
        t = torch.full(list(reversed(dims)), fill, dtype=torch.float64, device=cuda)
        return t.permute(*reversed(range(len(dims))))
    return torch.full(dims, fill, dtype=torch.float64, device=cuda)


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("permuted", [False, True])
def test_block_to_full_matches_oracle(cuda, case, permuted):
    import torch
    import tblis_b200 as tb
    nirrep, irrep, lens = CASES[case]
    rng = np.random.default_rng(40 + case)
    size = oracle.orc_dpd_size(irrep, nirrep, lens, 5)
    data = rng.uniform(-1, 1, max(size, 1))[:size]
    A = tb.DpdTensor(irrep, nirrep, lens, torch.from_numpy(data.copy()).to(cuda))
    dims = [sum(r) for r in lens]
    F = _dense(torch, cuda, dims, permuted, float("nan"))
    tb.dpd_block_to_full(A, F)
    torch.cuda.synchronize()
    want = oracle.orc_dpd_block_to_full(irrep, nirrep, lens, data)
    assert np.array_equal(F.cpu().numpy(), want)


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("permuted", [False, True])
def test_full_to_block_matches_oracle(cuda, case, permuted):
    import torch
    import tblis_b200 as tb
    nirrep, irrep, lens = CASES[case]
    rng = np.random.default_rng(60 + case)
    size = oracle.orc_dpd_size(irrep, nirrep, lens, 5)
    dims = [sum(r) for r in lens]
    full = rng.uniform(-1, 1, dims)
    F = _dense(torch, cuda, dims, permuted, 0.0)
    F.copy_(torch.from_numpy(full))
    data = np.full(size, 7.0)
    A = tb.DpdTensor(irrep, nirrep, lens, torch.from_numpy(data.copy()).to(cuda))
    tb.dpd_full_to_block(F, A)
    torch.cuda.synchronize()
    want = data.copy()
    oracle.orc_dpd_full_to_block(irrep, nirrep, lens, full, want)
    assert np.array_equal(A.data.cpu().numpy(), want)


@pytest.mark.parametrize("dtype", ["float32", "complex64", "complex128"])
def test_round_trip_every_type(cuda, dtype):
    import torch
    import tblis_b200 as tb
    nirrep, irrep, lens = CASES[2]
    size = oracle.orc_dpd_size(irrep, nirrep, lens, 5)
    tdt = getattr(torch, dtype)
    g = torch.Generator(device=cuda)
    g.manual_seed(3)
    if tdt.is_complex:
        src = torch.complex(torch.rand(size, generator=g, device=cuda), torch.rand(size, generator=g, device=cuda))
        src = src.to(tdt)
    else:
        src = torch.rand(size, generator=g, device=cuda, dtype=tdt)
    A = tb.DpdTensor(irrep, nirrep, lens, src.clone())
    F = torch.zeros([sum(r) for r in lens], dtype=tdt, device=cuda)
    tb.dpd_block_to_full(A, F)
    B = tb.DpdTensor(irrep, nirrep, lens, torch.zeros_like(src))
    tb.dpd_full_to_block(F, B)
    torch.cuda.synchronize()
    assert torch.equal(B.data, src)
    # everything outside the blocks is zero: the block sums add up to the whole
    assert torch.allclose(F.sum(), src.sum(), rtol=1e-5)


def test_host_dense_tensor_is_staged(cuda):
    import torch
    import tblis_b200 as tb
    nirrep, irrep, lens = CASES[4]
    size = oracle.orc_dpd_size(irrep, nirrep, lens, 5)
    data = np.random.default_rng(8).uniform(-1, 1, size)
    A = tb.DpdTensor(irrep, nirrep, lens, torch.from_numpy(data.copy()).to(cuda))
    F = np.full([sum(r) for r in lens], np.nan)
    tb.dpd_block_to_full(A, F)
    assert np.array_equal(F, oracle.orc_dpd_block_to_full(irrep, nirrep, lens, data))


def test_bad_shapes_and_types_raise(cuda):
    import torch
    import tblis_b200 as tb
    nirrep, irrep, lens = CASES[0]
    size = oracle.orc_dpd_size(irrep, nirrep, lens, 5)
    A = tb.DpdTensor(irrep, nirrep, lens, torch.zeros(size, dtype=torch.float64, device=cuda))
    dims = [sum(r) for r in lens]
    with pytest.raises(tb.TblisError) as e:
        tb.dpd_block_to_full(A, torch.zeros([dims[0] + 1] + dims[1:], dtype=torch.float64, device=cuda))
    assert e.value.code == 1
    with pytest.raises(tb.TblisError) as e:
        tb.dpd_block_to_full(A, torch.zeros(dims, dtype=torch.float32, device=cuda))
    assert e.value.code == 2
