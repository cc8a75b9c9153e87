"""GPU parity of the C++ overload tblis::mult over MArray dpd_varray_view
(libtblis_b200_cxx.so, src/iface/3t/mult.h:56-60), called through its mangled
name by a C++ driver exactly as a TBLIS C++ program calls it: every MArray
storage layout and permuted views, against the reference's own DPD
contraction on the same data."""
import ctypes
import os

import numpy as np
import pytest
from numpy.lib.stride_tricks import as_strided

import oracle

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "tests", "cxx", "_bin", "libdpd_driver.so")
_sz = ctypes.c_ssize_t


@pytest.fixture(scope="module")
def driver(cuda):
    assert os.path.exists(DRIVER), "C++ test driver not built (make -C tests/cxx MARRAY=...)"
    lib = ctypes.CDLL(DRIVER, mode=ctypes.RTLD_LOCAL)
    lib.driver_dpd_mult.restype = ctypes.c_int
    return lib


def tuples(irrep, nirrep, ndim):
    """Allowed irrep tuples in the order MArray's layout query lists them
    (oracle.ref_dpd_layout): dimension 1 fastest, dimension 0 closing the XOR."""
    out = []
    for b in range(nirrep ** (ndim - 1)):
        rest = [(b // nirrep ** i) % nirrep for i in range(ndim - 1)]
        x = irrep
        for r in rest:
            x ^= r
        out.append((x,) + tuple(rest))
    return out


def random_blocks(rng, irrep, nirrep, lens):
    return {t: rng.uniform(-1, 1, [lens[d][t[d]] for d in range(len(lens))])
            for t in tuples(irrep, nirrep, len(lens))}


def store(irrep, nirrep, lens, layout, blocks):
    """Flat storage of the blocks in MArray's layout `layout` (the geometry
    comes from MArray itself)."""
    total, offs, strides = oracle.ref_dpd_layout(irrep, nirrep, lens, layout)
    flat = np.zeros(max(total, 1))
    for b, t in enumerate(tuples(irrep, nirrep, len(lens))):
        shape = [lens[d][t[d]] for d in range(len(lens))]
        if np.prod(shape) == 0:
            continue
        v = as_strided(flat[offs[b]:], shape=shape, strides=[8 * s for s in strides[b]])
        v[...] = blocks[t]
    return flat


def load(irrep, nirrep, lens, layout, flat):
    total, offs, strides = oracle.ref_dpd_layout(irrep, nirrep, lens, layout)
    out = {}
    for b, t in enumerate(tuples(irrep, nirrep, len(lens))):
        shape = [lens[d][t[d]] for d in range(len(lens))]
        if np.prod(shape) == 0:
            continue
        out[t] = np.array(as_strided(flat[offs[b]:], shape=shape, strides=[8 * s for s in strides[b]]))
    return out


def flat_lens(lens):
    return (_sz * sum(len(r) for r in lens))(*[x for r in lens for x in r])


def call(driver, nirrep, alpha, A, B, beta, C):
    """Each of A, B, C: dict(irrep, lens, layout, perm, data, idx)."""
    args = [ctypes.c_uint(nirrep), ctypes.c_double(alpha)]
    for i, T in enumerate((A, B, C)):
        if i == 2:
            args.append(ctypes.c_double(beta))
        perm = None if T["perm"] is None else (ctypes.c_uint * len(T["perm"]))(*T["perm"])
        args += [ctypes.c_uint(T["irrep"]), ctypes.c_uint(len(T["lens"])), flat_lens(T["lens"]),
                 ctypes.c_int(T["layout"]), perm, ctypes.c_void_p(T["data"].ctypes.data), T["idx"].encode()]
    return driver.driver_dpd_mult(*args)


def rel(got, want):
    num = sum(np.sum((got[t] - want[t]) ** 2) for t in want)
    den = sum(np.sum(want[t] ** 2) for t in want)
    return np.sqrt(num / den)


def ladder_case(seed, nirrep=4):
    rng = np.random.default_rng(seed)
    occ = [int(x) for x in rng.integers(1, 5, nirrep)]
    vir = [int(x) for x in rng.integers(2, 8, nirrep)]
    lA, lB, lC = [vir, vir, vir, vir], [vir, vir, occ, occ], [vir, vir, occ, occ]
    bA = random_blocks(rng, 0, nirrep, lA)
    bB = random_blocks(rng, 0, nirrep, lB)
    bC = random_blocks(rng, 0, nirrep, lC)
    return lA, lB, lC, bA, bB, bC


def reference(nirrep, alpha, lA, bA, iA, lB, bB, iB, beta, lC, bC, iC, irreps=(0, 0, 0)):
    """The reference's DPD contraction on default-layout (5) storage."""
    a = store(irreps[0], nirrep, lA, 5, bA)
    b = store(irreps[1], nirrep, lB, 5, bB)
    c = store(irreps[2], nirrep, lC, 5, bC)
    oracle.ref_dpd_mult(nirrep, alpha, irreps[0], lA, a, iA, irreps[1], lB, b, iB, beta, irreps[2], lC, c, iC)
    return load(irreps[2], nirrep, lC, 5, c)


@pytest.mark.parametrize("layout", range(6))
def test_every_storage_layout(driver, layout):
    nirrep = 4
    lA, lB, lC, bA, bB, bC = ladder_case(100 + layout, nirrep)
    want = reference(nirrep, 0.75, lA, bA, "abef", lB, bB, "efij", 0.5, lC, bC, "abij")
    A = dict(irrep=0, lens=lA, layout=layout, perm=None, data=store(0, nirrep, lA, layout, bA), idx="abef")
    B = dict(irrep=0, lens=lB, layout=layout, perm=None, data=store(0, nirrep, lB, layout, bB), idx="efij")
    C = dict(irrep=0, lens=lC, layout=layout, perm=None, data=store(0, nirrep, lC, layout, bC), idx="abij")
    assert call(driver, nirrep, 0.75, A, B, 0.5, C) == 0
    got = load(0, nirrep, lC, layout, C["data"])
    assert rel(got, want) <= 1e-13


@pytest.mark.parametrize("seed", range(4))
def test_permuted_views(driver, seed):
    """A view permuted by p with its labels permuted alike is the same tensor:
    the result must match the unpermuted reference call."""
    nirrep = 4
    rng = np.random.default_rng(200 + seed)
    lA, lB, lC, bA, bB, bC = ladder_case(200 + seed, nirrep)
    want = reference(nirrep, 1.0, lA, bA, "abef", lB, bB, "efij", 0.0, lC, bC, "abij")
    pA = [int(x) for x in rng.permutation(4)]
    pC = [int(x) for x in rng.permutation(4)]
    A = dict(irrep=0, lens=lA, layout=5, perm=pA, data=store(0, nirrep, lA, 5, bA),
             idx="".join("abef"[p] for p in pA))
    B = dict(irrep=0, lens=lB, layout=5, perm=None, data=store(0, nirrep, lB, 5, bB), idx="efij")
    C = dict(irrep=0, lens=lC, layout=5, perm=pC, data=store(0, nirrep, lC, 5, bC),
             idx="".join("abij"[p] for p in pC))
    assert call(driver, nirrep, 1.0, A, B, 0.0, C) == 0
    got = load(0, nirrep, lC, 5, C["data"])
    assert rel(got, want) <= 1e-13


def test_ring_term_with_nonzero_irreps(driver):
    """Ring-type labels interleave in the layout tree (segmented-K groups) and
    the tensors carry non-zero irreps."""
    nirrep = 2
    rng = np.random.default_rng(300)
    o = [3, 2]
    v = [4, 5]
    lA, lB, lC = [v, v, o, o], [o, v, v, o], [v, o, v, o]
    bA = random_blocks(rng, 1, nirrep, lA)
    bB = random_blocks(rng, 1, nirrep, lB)
    bC = random_blocks(rng, 0, nirrep, lC)
    want = reference(nirrep, 1.0, lA, bA, "aeim", lB, bB, "mbej", 1.0, lC, bC, "aibj", irreps=(1, 1, 0))
    A = dict(irrep=1, lens=lA, layout=5, perm=None, data=store(1, nirrep, lA, 5, bA), idx="aeim")
    B = dict(irrep=1, lens=lB, layout=5, perm=None, data=store(1, nirrep, lB, 5, bB), idx="mbej")
    C = dict(irrep=0, lens=lC, layout=5, perm=None, data=store(0, nirrep, lC, 5, bC), idx="aibj")
    assert call(driver, nirrep, 1.0, A, B, 1.0, C) == 0
    got = load(0, nirrep, lC, 5, C["data"])
    assert rel(got, want) <= 1e-13
