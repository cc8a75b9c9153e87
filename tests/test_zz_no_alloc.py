"""GPU test of tblis_b200_tensor_mult_noalloc, the allocation-free entry point
for callers that cannot let the library call cudaMalloc (their device memory
belongs to another allocator, or they must not trigger the device-wide
synchronisation an allocation can cause). Its output must match
tblis_tensor_mult's on the same inputs within the plain-FP64 tolerance used by
every contraction test (1e-13 normwise relative), on two calls in a row (the
second call finds the shared scratch array holding the first call's data).

This file is named to be collected last, so a run that stops at the first
failure has run every other test before it."""
import ctypes

import numpy as np
import pytest

from tests.helpers import normwise_rel

pytestmark = pytest.mark.gpu
TOL = 1e-13


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
    # (idx_A, idx_B, idx_C, shapes) -- 24^4 needs split-K partials in the scratch array
    ("abef", "efij", "abij", {"a": 24, "b": 24, "e": 24, "f": 24, "i": 24, "j": 24}),
    ("aeim", "mbej", "aibj", {"a": 40, "e": 24, "i": 8, "m": 8, "b": 40, "j": 8}),
    ("abc", "cbd", "ad", {"a": 300, "b": 7, "c": 9, "d": 260}),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_noalloc_matches_default_entry_point_twice(cuda, case):
    import torch
    import tblis_b200 as tb
    idx_A, idx_B, idx_C, lens = CASES[case]
    g = torch.Generator(device=cuda)
    g.manual_seed(100 + case)

    def make(idx):
        shape = [lens[c] for c in idx]
        return torch.empty(list(reversed(shape)), dtype=torch.float64, device=cuda) \
            .uniform_(-1, 1, generator=g).permute(*reversed(range(len(shape))))

    A, B = make(idx_A), make(idx_B)
    for call in range(2):
        C0 = make(idx_C)
        want = C0.clone()
        tb.mult(0.75, A, idx_A, B, idx_B, 0.5, want, idx_C)
        got = C0.clone()
        _noalloc(tb, 0.75, A, idx_A, B, idx_B, 0.5, got, idx_C)
        torch.cuda.synchronize()
        err = normwise_rel(got.cpu().numpy(), want.cpu().numpy())
        assert err <= TOL, (case, call, err)


def test_noalloc_rejects_host_data_and_reports_limit(cuda):
    import tblis_b200 as tb
    tb.lib.tblis_b200_noalloc_scratch_bytes.restype = ctypes.c_size_t
    assert tb.lib.tblis_b200_noalloc_scratch_bytes() == 32 << 20
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
    with pytest.raises(tb.TblisError) as e:
        _noalloc(tb, 1.0, A, "ab", B, "bc", 0.0, C, "ac")
    assert e.value.code == 5
