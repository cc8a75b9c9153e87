"""The scatter-table cache under churn: more distinct contraction shapes than
it holds (512 live tables), so evicted tables retire and are freed in a
batch once 256 have retired, while later contractions keep running. Every
result is checked, before and after the purge."""
import pytest

pytestmark = pytest.mark.gpu


def test_more_shapes_than_the_cache_holds(cuda):
    import torch
    import tblis_b200 as tb
    g = torch.Generator(device=cuda)
    g.manual_seed(3)
    worst = 0.0
    for i in range(800):
        m, n, k = i % 37 + 1, i // 37 + 1, 3 + i % 5
        A = torch.empty((m, k), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g)
        B = torch.empty((k, n), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g)
        C = torch.empty((m, n), dtype=torch.float64, device=cuda).uniform_(-1, 1, generator=g)
        want = 0.5 * (A @ B) - 1.25 * C
        tb.mult(0.5, A, "ac", B, "cb", -1.25, C, "ab")
        err = ((C - want).abs().max() / want.abs().max().clamp_min(1.0)).item()
        worst = max(worst, err)
        assert err <= 1e-14, (i, m, n, k, err)
    torch.cuda.synchronize()
    assert worst <= 1e-14
