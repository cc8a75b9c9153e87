"""GPU parity of the DPD (irrep block-sparse) contraction: tblis_b200_dpd_mult
against the reference's own C++ DPD contraction (tblis::mult over
dpd_varray_view, built from the reference sources) on the same seeded
storage. Tolerance: plain FP64, 1e-13 normwise relative."""
import numpy as np
import pytest

import oracle

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built")]
TOL = 1e-13


def _rel(x, ref):
    d = np.linalg.norm(x - ref)
    n = np.linalg.norm(ref)
    return d / n if n else d


def _run(cuda, nirrep, idx, lens, irreps, alpha, beta, seed):
    """idx: (idx_A, idx_B, idx_C); lens: label -> per-irrep lengths."""
    import torch
    import tblis_b200 as tb
    rng = np.random.default_rng(seed)
    tens = []
    for ix, irr in zip(idx, irreps):
        L = [lens[c] for c in ix]
        t = tb.DpdTensor(irr, nirrep, L)
        n = t.size()
        data = rng.uniform(-1, 1, n)
        tens.append((t, L, data))
    (tA, LA, dA), (tB, LB, dB), (tC, LC, dC) = tens
    ref = dC.copy()
    oracle.ref_dpd_mult(nirrep, alpha, irreps[0], LA, dA, idx[0], irreps[1], LB, dB, idx[1],
                        beta, irreps[2], LC, ref, idx[2])
    gA = torch.from_numpy(dA).to(cuda)
    gB = torch.from_numpy(dB).to(cuda)
    gC = torch.from_numpy(dC.copy()).to(cuda)
    tA.data, tB.data, tC.data = gA, gB, gC
    rep = tb.dpd_mult(alpha, tA, idx[0], tB, idx[1], beta, tC, idx[2])
    torch.cuda.synchronize()
    return gC.cpu().numpy(), ref, rep


def _lens(rng, labels, nirrep, lo=0, hi=5):
    return {c: [int(rng.integers(lo, hi + 1)) for _ in range(nirrep)] for c in labels}


@pytest.mark.parametrize("nirrep", [1, 2, 4, 8])
@pytest.mark.parametrize("seed", range(3))
def test_ladder_blocks(cuda, nirrep, seed):
    rng = np.random.default_rng(100 * nirrep + seed)
    lens = _lens(rng, "abefij", nirrep, 0, 4 if nirrep == 8 else 6)
    got, ref, rep = _run(cuda, nirrep, ("abef", "efij", "abij"), lens, (0, 0, 0), 1.0, 0.0, seed)
    assert _rel(got, ref) <= TOL
    assert rep["m"] <= nirrep


@pytest.mark.parametrize("seed", range(4))
def test_ring_blocks_nonzero_irreps(cuda, seed):
    """C[aibj] = alpha*A[aeim]*B[mbej] + beta*C with irrep(A)=1, irrep(B)=1 ->
    irrep(C)=0, in the permuted label orders of the ring term."""
    rng = np.random.default_rng(7 + seed)
    lens = _lens(rng, "aeimbj", 4, 1, 5)
    got, ref, rep = _run(cuda, 4, ("aeim", "mbej", "aibj"), lens, (1, 1, 0), 0.5, 0.75, seed)
    assert _rel(got, ref) <= TOL


def test_matrix_and_mixed_irreps(cuda):
    rng = np.random.default_rng(3)
    lens = _lens(rng, "ikj", 2, 1, 9)
    got, ref, _ = _run(cuda, 2, ("ik", "kj", "ij"), lens, (1, 0, 1), 2.0, -1.0, 3)
    assert _rel(got, ref) <= TOL


def test_irrep_check_quirk_is_reproduced(cuda):
    """irrep(A)=2, irrep(B)=0, irrep(C)=2: the reference's check
    `A.irrep()^B.irrep() != C.irrep()` (src/iface/3t/mult.cxx:270) reads as
    A.irrep()^(B.irrep()!=C.irrep()) = 3, so C is only scaled by beta."""
    rng = np.random.default_rng(4)
    lens = _lens(rng, "ikj", 4, 1, 4)
    got, ref, rep = _run(cuda, 4, ("ik", "kj", "ij"), lens, (2, 0, 2), 1.0, 0.5, 4)
    assert _rel(got, ref) <= TOL
    assert rep["kernels"] >= 1


def test_dpd_ladder_small_d2h(cuda):
    """The D2h ladder term C[abij] = A[abef]*B[efij] (8 irreps, total irrep 0)
    at reduced per-irrep extents."""
    occ = [2, 1, 2, 1, 2, 1, 1, 1]
    vir = [6, 3, 5, 4, 6, 2, 4, 3]
    lens = {"a": vir, "b": vir, "e": vir, "f": vir, "i": occ, "j": occ}
    got, ref, rep = _run(cuda, 8, ("abef", "efij", "abij"), lens, (0, 0, 0), 1.0, 0.0, 11)
    assert _rel(got, ref) <= TOL
    assert rep["m"] == 8 and rep["flops"] > 0


def test_repeat_call_replays_cached_plan(cuda):
    import torch
    import tblis_b200 as tb
    rng = np.random.default_rng(5)
    lens = _lens(rng, "abefij", 2, 1, 6)
    for seed in (21, 22):      # same shapes: cached plan and graph, new data
        got, ref, rep = _run(cuda, 2, ("abef", "efij", "abij"), lens, (0, 0, 0), 1.0, 1.0, seed)
        assert _rel(got, ref) <= TOL
