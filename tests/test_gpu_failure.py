"""Failure detection of the Ozaki kernels, tested without any GPU fault.

Every wait of the slice GEMM and of the moduli GEMM on an mbarrier is
bounded. tblis_b200_ozaki_inject_wait_timeout makes those kernels skip the
operand copies of one k step (one pipeline stage for the moduli kernel) and
shortens the bound, so the wait for that stage runs out: the kernel records
the timeout, drains the copies it issued, frees its tensor memory and
returns. The test checks that tblis_b200_synchronize reports TB_ERR_TIMEOUT
(6) once, and that the same contraction then runs correctly on the same
context (nothing was left hung or corrupted)."""
import ctypes

import numpy as np
import pytest

import oracle
from tests.helpers import normwise_rel

pytestmark = pytest.mark.gpu


def _inject(tb, step, seconds):
    fn = tb.lib.tblis_b200_ozaki_inject_wait_timeout
    fn.argtypes = [ctypes.c_int, ctypes.c_double]
    fn.restype = ctypes.c_int
    assert fn(step, seconds) == 0


@pytest.mark.parametrize("method,slices", [(2, 4), (6, 12)])
def test_bounded_wait_runs_out_and_context_recovers(cuda, method, slices):
    import torch
    import tblis_b200 as tb
    rng = np.random.default_rng(5)
    A = rng.uniform(-1, 1, (300, 2048))
    B = rng.uniform(-1, 1, (2048, 260))
    ref = np.zeros((300, 260))
    oracle.orc_mult(1.0, A, "ik", B, "kj", 0.0, ref, "ij")
    dA, dB = torch.from_numpy(A).to(cuda), torch.from_numpy(B).to(cuda)
    dC = torch.zeros((300, 260), dtype=torch.float64, device=cuda)
    tb.synchronize()
    try:
        _inject(tb, 3, 0.05)
        tb.mult_ex(1.0, dA, "ik", dB, "kj", 0.0, dC, "ij", method=method, slices=slices)
        with pytest.raises(tb.TblisError) as e:
            tb.synchronize()
        assert e.value.code == 6
    finally:
        _inject(tb, -1, 0.0)
    # reported once, then the context works as before
    tb.synchronize()
    dC.zero_()
    rep = tb.mult_ex(1.0, dA, "ik", dB, "kj", 0.0, dC, "ij", method=method, slices=slices)
    tb.synchronize()
    assert rep["method"] == method
    assert normwise_rel(dC.cpu().numpy(), ref) <= 1e-9


# The packed grouped FP64 GEMM (batches, DPD, indexed DPD) has the same
# bounded waits. It runs only where the tuner picks it, so the check runs in a
# child process with that path forced (TBLIS_B200_GEMM_VARIANT=5): a batch of
# three contractions, one run with a stage whose copies never come, then the
# same batch again on the same context.
_PACKED_TIMEOUT = r"""
import ctypes
import numpy as np
import torch
import tblis_b200 as tb
import oracle
from tests.helpers import normwise_rel

dev = torch.device("cuda:0")
rng = np.random.default_rng(9)
shapes = [(96, 80, 2048), (64, 64, 1024), (130, 70, 1500)]
host, items = [], []
for m, n, k in shapes:
    A, B = rng.uniform(-1, 1, (m, k)), rng.uniform(-1, 1, (k, n))
    ref = np.zeros((m, n))
    oracle.orc_mult(1.0, A, "ik", B, "kj", 0.0, ref, "ij")
    C = torch.zeros((m, n), dtype=torch.float64, device=dev)
    host.append(ref)
    items.append((1.0, torch.from_numpy(A).to(dev), "ik", torch.from_numpy(B).to(dev), "kj", 0.0, C, "ij"))
batch = tb.PreparedBatch(items)
batch.run()
tb.synchronize()
inject = tb.lib.tblis_b200_grouped_inject_wait_timeout
inject.argtypes = [ctypes.c_int, ctypes.c_double]
inject.restype = ctypes.c_int
assert inject(3, 0.05) == 0
try:
    batch.run()
    try:
        tb.synchronize()
        raise SystemExit("no timeout reported")
    except tb.TblisError as e:
        assert e.code == 6, e.code
finally:
    assert inject(-1, 0.0) == 0
tb.synchronize()                  # reported once
for it in items:
    it[6].zero_()
batch.run()
tb.synchronize()
for it, ref in zip(items, host):
    err = normwise_rel(it[6].cpu().numpy(), ref)
    assert err <= 1e-13, err
print("packed timeout ok")
"""


def test_packed_grouped_wait_runs_out_and_context_recovers(cuda):
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ)
    env["TBLIS_B200_GEMM_VARIANT"] = "5"
    r = subprocess.run([sys.executable, "-c", _PACKED_TIMEOUT], cwd=root, env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-3000:])
    assert "packed timeout ok" in r.stdout
