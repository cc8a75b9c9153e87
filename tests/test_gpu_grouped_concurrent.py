"""Grouped FP64 launches stay exact while other kernels run beside them.

A batch of 4-index contractions (the shape of the 10,000-member benchmark
batch, extents 4..32, every operand in a random index order) runs on one
stream while unrelated kernels (an elementwise pass and a random gather over
a 1 GiB vector) run on another, so that their blocks share SMs with the
grouped GEMM. Every member is checked against torch's FP64 einsum.

This guards the packed path's stage ring: its bulk copies (async proxy)
refill shared memory that the MMA warps read with ordinary loads, and the
refill has to be ordered after those loads by a proxy fence. Without the
fence, runs next to other kernels gave wrong warp tiles (thousands of
members of 10,000 beside the gather) while runs alone were exact. The batch
runs in a child process per path, with TBLIS_B200_GEMM_VARIANT naming it
(5 = packed, 4 = per-thread gathers), so each path is covered whatever the
tuner would pick."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import random, sys
sys.path.insert(0, sys.argv[1])
import torch
import tblis_b200 as tb
dev = torch.device("cuda:0")
rnd = random.Random(0)
g = torch.Generator(device=dev)
g.manual_seed(43)
items = []
for _ in range(4000):
    l = {c: rnd.randint(4, 32) for c in "abefij"}
    ia = "".join(rnd.sample("abef", 4)); ib = "".join(rnd.sample("efij", 4)); ic = "".join(rnd.sample("abij", 4))
    mk = lambda ix: torch.empty([l[c] for c in ix], dtype=torch.float64, device=dev).uniform_(-1, 1, generator=g)
    items.append((1.0, mk(ia), ia, mk(ib), ib, 0.0, mk(ic), ic))
wants = [torch.einsum("%s,%s->%s" % (ia, ib, ic), a, b) for (_, a, ia, b, ib, _, _, ic) in items]
s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
tb.set_stream(s1.cuda_stream)
prepared = tb.PreparedBatch(items)
with torch.cuda.stream(s1):
    rep = prepared.run()
torch.cuda.synchronize()
x = torch.randn(1 << 28, device=dev, dtype=torch.float32)
idx = torch.randint(0, 1 << 28, (1 << 26,), device=dev)
for mode in ("elementwise", "gather"):
    for _ in range(2):
        for it in items:
            it[6].fill_(float("nan"))
        torch.cuda.synchronize()
        with torch.cuda.stream(s2):
            for _ in range(40):
                y = x * 1.0001 + 0.5 if mode == "elementwise" else x[idx]
        with torch.cuda.stream(s1):
            prepared.run()
        torch.cuda.synchronize()
        tb.synchronize()
        bad = sum(1 for it, w in zip(items, wants)
                  if not ((it[6] - w).norm() / w.norm()).item() <= 1e-13)
        print("variant", rep["n"], mode, "bad", bad, flush=True)
'''


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["5", "4"])
def test_grouped_batch_exact_beside_other_kernels(cuda, variant):
    env = dict(os.environ)
    env["TBLIS_B200_GEMM_VARIANT"] = variant
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("variant")]
    assert len(lines) == 4, r.stdout[-2000:]
    for ln in lines:
        assert ln.split()[1] == variant, ln
        assert ln.endswith(" bad 0"), ln
