"""Both grouped FP64 code paths, each forced in turn.

A grouped plan (DPD irrep GEMMs, indexed-DPD triples, batches of
contractions) runs on whichever path its autotuner timed fastest: the packed
path (a pack kernel gathers the operand panels once, then a warp-specialised
persistent GEMM streams them with bulk copies) or the kernel whose threads
gather their own tiles through the scatter vectors. The tuner's choice depends
on the shapes, so a plain run of the parity tests may exercise only one of
them. These tests rerun the batch and DPD parity suites in a child process
with TBLIS_B200_GEMM_VARIANT naming one path (5 = packed, 4 = 64x64
per-thread gathers), so both stay checked against the oracle and the
reference whatever the tuner picks."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["5", "4"])
def test_grouped_parity_suites_on_each_path(cuda, variant):
    env = dict(os.environ)
    env["TBLIS_B200_GEMM_VARIANT"] = variant
    cmd = [sys.executable, "-m", "pytest", "-q", "-x", "-m", "gpu", "-p", "no:cacheprovider",
           os.path.join("tests", "test_gpu_batch.py"), os.path.join("tests", "test_gpu_dpd.py"),
           os.path.join("tests", "test_gpu_dpd_abc.py")]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=1800)
    assert r.returncode == 0, (variant, r.stdout[-3000:], r.stderr[-2000:])
    assert " passed" in r.stdout, r.stdout[-1000:]
