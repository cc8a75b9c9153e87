"""Link-time drop-in, shown with programs written against TBLIS's own headers.

tests/cxx/dropin_c.c and dropin_cxx.cxx include TBLIS's src/tblis.h (with its
MArray and TCI headers) and are linked against libtblis_b200.so alone (the
build recipe is tests/cxx/Makefile; both also static_assert the byte layout
of tblis_scalar and tblis_tensor from TBLIS's basic_types.h against the
numbers abi_ours.c checks in include/tblis_b200.h). They run TBLIS's C ABI
and its inline C++ templates on host buffers and write their inputs and
results; this test recomputes every result with the oracle and compares:
contractions within the FP64 tolerance (1e-13 normwise relative; 1e-12 for
the Ozaki configuration), level-1 results exactly or within rounding."""
import os
import struct
import subprocess

import numpy as np
import pytest

import oracle
from tests.helpers import normwise_rel

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "tests", "cxx", "_bin")


def _run(tmp_path, name):
    exe = os.path.join(BIN, name)
    assert os.path.exists(exe), "drop-in program not built (make -C tests/cxx REF=... MARRAY=...)"
    out = str(tmp_path / (name + ".bin"))
    env = dict(os.environ)
    env.pop("LD_PRELOAD", None)
    subprocess.run([exe, out], check=True, env=env, timeout=300)
    rec = {}
    with open(out, "rb") as f:
        while True:
            tag = f.read(16)
            if not tag:
                break
            (n,) = struct.unpack("<q", f.read(8))
            rec[tag.rstrip(b"\0").decode()] = np.frombuffer(f.read(8 * n), dtype=np.float64).copy()
    return rec


def _view(flat, lens, strides):
    return np.lib.stride_tricks.as_strided(flat, shape=lens, strides=[8 * s for s in strides])


def test_abi_layout_of_this_header_compiles():
    # the object exists only if its static_asserts held at build time
    assert os.path.exists(os.path.join(BIN, "abi_ours.o"))


def test_c_program_against_tblis_header(cuda, tmp_path):
    r = _run(tmp_path, "dropin_c")
    lenA, strA = [7, 6, 5, 4], [126, 21, 4, 1]
    lenB, strB = [5, 4, 3, 6], [1, 5, 20, 60]
    lenC, strC = [7, 6, 3, 6], [1, 7, 42, 126]
    A = _view(r["A"], lenA, strA)
    B = _view(r["B"], lenB, strB)
    want = r["C0"].copy()
    oracle.orc_mult(0.5, A, "abef", B, "efij", 2.0, _view(want, lenC, strC), "abij")
    assert normwise_rel(r["C"], want) <= 1e-13
    # C's scalar reset to 1 and conj to 0 (src/iface/3t/mult.cxx:162-163)
    assert r["Cscalar"][0] == 1.0 and r["Cscalar"][1] == 0.0
    assert r["has_cfg"][0] == 1.0
    assert normwise_rel(r["C_ozaki"], want) <= 1e-12
    C = _view(r["C"], lenC, strC)
    D = np.zeros(r["D"].shape)
    oracle.orc_add(1.5, C, "abij", 0.0, _view(D, [3, 6, 7, 6], [1, 3, 18, 126]), "ijab")
    assert np.array_equal(r["D"], D)
    assert abs(r["dot"][0] - oracle.orc_dot(A, "abef", A, "abef")) <= 1e-13 * abs(r["dot"][0])
    nrm, _ = oracle.orc_reduce(6, C, "abij")
    assert abs(r["norm2"][0] - nrm) <= 1e-14 * nrm
    mx, idx = oracle.orc_reduce(3, C, "abij")
    assert r["maxabs"][0] == mx and int(r["maxabs"][1]) == idx
    assert np.array_equal(r["Cscaled"], -0.25 * r["C"])


def test_cxx_templates_against_tblis_header(cuda, tmp_path):
    r = _run(tmp_path, "dropin_cxx")
    # MArray's default layout is row-major
    A = r["A"].reshape(6, 7, 5, 4)
    B = r["B"].reshape(7, 4, 5, 3)
    want = r["C0"].reshape(6, 5, 5, 3).copy()
    oracle.orc_mult(0.75, A, "aebf", B, "efij", -0.5, want, "abij")
    C = r["C"].reshape(6, 5, 5, 3)
    assert normwise_rel(C, want) <= 1e-13
    D = np.zeros((3, 5, 5, 6))
    oracle.orc_add(2.0, C, "abij", 0.0, D, "jiba")
    assert np.array_equal(r["D"].reshape(3, 5, 5, 6), D)
    want_dot = oracle.orc_dot(C.transpose(3, 1, 0, 2), "jbai", C, "abij")
    assert abs(r["dot"][0] - want_dot) <= 1e-13 * abs(want_dot)
    mx, idx = oracle.orc_reduce(2, C, "abij")
    assert r["max"][0] == mx and int(r["max"][1]) == idx
    assert np.array_equal(r["Cscaled"], 3.0 * r["C"])
