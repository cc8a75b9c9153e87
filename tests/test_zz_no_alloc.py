"""GPU tests of tblis_b200_tensor_mult_noalloc, the allocation-free entry point.

Some callers cannot let the library call cudaMalloc: their device memory
belongs to another allocator that reserved the GPU up front, or their loop
must not hit the device-wide synchronisation an allocation can cause. This
entry point keeps all of its scratch in one fixed device array that every call
shares. Each contraction below is checked against the C oracle (the
restatement of the reference's mult_ref, pinned to the reference itself) within
the plain-FP64 tolerance of every contraction test (1e-13 normwise relative),
and against tblis_tensor_mult's own result, on two calls in a row: the second
call finds the shared array holding the first call's data.

This file is named to be collected last, so a run that stops at the first
failure has run every other test before it."""
import ctypes

import numpy as np
import pytest

import oracle
from tests.helpers import normwise_rel

pytestmark = pytest.mark.gpu
TOL = 1e-13
SCRATCH = 32 << 20


def _noalloc(tb, alpha, A, idx_A, B, idx_B, beta, C, idx_C):
    a, b, c = tb._View(A, alpha), tb._View(B), tb._View(C, beta)
    fn = tb.lib.tblis_b200_tensor_mult_noalloc
    fn.restype = ctypes.c_int
    rc = fn(a.ref, idx_A.encode(), b.ref, idx_B.encode(), c.ref, idx_C.encode())
    if rc:
        msg = tb.lib.tblis_b200_last_error_string().decode()
        tb.lib.tblis_b200_clear_error()
        raise tb.TblisError(rc, msg)


CASES = [
    # (idx_A, idx_B, idx_C, lengths) -- 24^4 needs split-K partials in the scratch array
    ("abef", "efij", "abij", {"a": 24, "b": 24, "e": 24, "f": 24, "i": 24, "j": 24}),
    ("aeim", "mbej", "aibj", {"a": 40, "e": 24, "i": 8, "m": 8, "b": 40, "j": 8}),
    ("abc", "cbd", "ad", {"a": 300, "b": 7, "c": 9, "d": 260}),
    # a batch label in all three tensors
    ("zak", "zkb", "zab", {"z": 5, "a": 33, "k": 70, "b": 29}),
]


def _make(torch, cuda, g, idx, lens):
    shape = [lens[c] for c in idx]
    return torch.empty(list(reversed(shape)), dtype=torch.float64, device=cuda) \
        .uniform_(-1, 1, generator=g).permute(*reversed(range(len(shape))))


@pytest.mark.parametrize("case", range(len(CASES)))
def test_noalloc_matches_oracle_and_default_entry_point_twice(cuda, case):
    import torch
    import tblis_b200 as tb
    idx_A, idx_B, idx_C, lens = CASES[case]
    g = torch.Generator(device=cuda)
    g.manual_seed(100 + case)
    A, B = _make(torch, cuda, g, idx_A, lens), _make(torch, cuda, g, idx_B, lens)
    hA, hB = A.cpu().numpy(), B.cpu().numpy()
    for call in range(2):
        C0 = _make(torch, cuda, g, idx_C, lens)
        want = C0.cpu().numpy().copy()
        oracle.orc_mult(0.75, hA, idx_A, hB, idx_B, 0.5, want, idx_C)
        default = C0.clone()
        tb.mult(0.75, A, idx_A, B, idx_B, 0.5, default, idx_C)
        got = C0.clone()
        _noalloc(tb, 0.75, A, idx_A, B, idx_B, 0.5, got, idx_C)
        torch.cuda.synchronize()
        err = normwise_rel(got.cpu().numpy(), want)
        assert err <= TOL, (case, call, err)
        assert normwise_rel(got.cpu().numpy(), default.cpu().numpy()) <= TOL, (case, call)


@pytest.mark.parametrize("alpha,klen,beta", [(0.0, 7, 0.5), (0.0, 7, 0.0), (1.5, 0, 2.0), (1.5, 0, 0.0)])
def test_noalloc_no_product_sets_or_scales_c(cuda, alpha, klen, beta):
    """alpha == 0 or an empty contracted extent: C = beta*C, or C = 0
    without reading C (a NaN in C must not survive beta == 0)."""
    import torch
    import tblis_b200 as tb
    g = torch.Generator(device=cuda)
    g.manual_seed(7)
    A = torch.empty((9, klen), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g)
    B = torch.empty((klen, 6), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g)
    for call in range(2):
        C = torch.empty((9, 6), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g)
        if beta == 0.0:
            C[2, 3] = float("nan")
        want = C.cpu().numpy().copy()
        oracle.orc_mult(alpha, A.cpu().numpy(), "ak", B.cpu().numpy(), "kb", beta, want, "ab")
        _noalloc(tb, alpha, A, "ak", B, "kb", beta, C, "ab")
        torch.cuda.synchronize()
        got = C.cpu().numpy()
        assert np.isfinite(got).all()
        assert np.array_equal(got, want), (alpha, klen, beta, call)


def _choose_splits(M, N, K, L, sms):
    """The FP64 kernel's split-K choice (64x64 tiles, three resident per SM,
    16-wide k blocks), restated here to size the next test."""
    tiles = -(-M // 64) * -(-N // 64) * L
    kt = -(-K // 16)
    slots = 3 * sms
    if tiles >= slots or kt < 8:
        return 1
    return max(1, min(-(-slots // tiles), kt // 4, 32))


def test_noalloc_reduces_split_k_to_fit(cuda):
    """A long K with few output tiles: the default split-K partials plus the
    scatter vectors would overflow the 32 MiB array, so the entry point must
    use fewer splits. A is one column broadcast along k (stride 0), so
    C[a, c] = x[a] * sum_k B[k, c] is known in closed form."""
    import torch
    import tblis_b200 as tb
    M, N, K = 1280, 64, 1_200_000
    sms = torch.cuda.get_device_properties(cuda).multi_processor_count
    splits = _choose_splits(M, N, K, 1, sms)
    tables = (2 * M + 2 * K + 2 * N + 3 + 2 * (-(-K // 16))) * 8
    assert splits > 1 and tables + splits * M * N * 8 > SCRATCH and tables < SCRATCH
    g = torch.Generator(device=cuda)
    g.manual_seed(11)
    x = torch.empty(M, dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g)
    A = x.as_strided((M, K), (1, 0))
    B = torch.empty((K, N), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g)
    want = torch.outer(x, B.sum(0)).cpu().numpy()
    for call in range(2):
        C = torch.full((M, N), float("nan"), dtype=torch.float64, device=cuda)
        _noalloc(tb, 1.0, A, "ak", B, "kb", 0.0, C, "ab")
        torch.cuda.synchronize()
        assert normwise_rel(C.cpu().numpy(), want) <= TOL, call


def test_noalloc_rejects_host_data_and_reports_limit(cuda):
    import tblis_b200 as tb
    tb.lib.tblis_b200_noalloc_scratch_bytes.restype = ctypes.c_size_t
    assert tb.lib.tblis_b200_noalloc_scratch_bytes() == SCRATCH
    A = np.ones((4, 5))
    B = np.ones((5, 3))
    C = np.zeros((4, 3))
    with pytest.raises(tb.TblisError) as e:
        _noalloc(tb, 1.0, A, "ab", B, "bc", 0.0, C, "ac")
    assert e.value.code == 1


def test_noalloc_rejects_oversized_tables(cuda):
    import torch
    import tblis_b200 as tb
    # scatter vectors of an m=3M, k=1M, n=2 view need (2m+2k+2n+...)*8 bytes > 32 MiB;
    # A broadcasts one 3M-element column along k (stride 0), so nothing large is allocated
    A = torch.zeros(3_000_000, dtype=torch.float64, device=cuda).as_strided((3_000_000, 1_000_000), (1, 0))
    B = torch.zeros((1_000_000, 2), dtype=torch.float64, device=cuda)
    C = torch.zeros((3_000_000, 2), dtype=torch.float64, device=cuda)
    C.fill_(3.0)
    with pytest.raises(tb.TblisError) as e:
        _noalloc(tb, 1.0, A, "ab", B, "bc", 0.0, C, "ac")
    assert e.value.code == 5
    # a failed call leaves C as it was
    assert bool((C == 3.0).all())
