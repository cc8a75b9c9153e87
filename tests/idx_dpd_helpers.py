"""Indexed-DPD test helpers: random tensors in MArray's indexed_dpd_varray
storage (entries back to back, default layout) and a plain numpy restatement
of the contraction in its FULL form (src/internal/3t/indexed_dpd/mult.cxx:68-114
with block_to_full / full_to_block, src/internal/1t/indexed_dpd/util.hpp:14-113),
used to pin the reference's behaviour before comparing the GPU path with it."""

import numpy as np
from numpy.lib.stride_tricks import as_strided

import oracle


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


def dense_irrep(T):
    x = T["irrep"]
    for r in T["idx_irreps"]:
        x ^= r
    return x


def dense_geometry(T, nirrep):
    """(entry size, {tuple: (offset, shape, strides)}) of the dense part."""
    nd = len(T["lens"]) - len(T["idx_irreps"])
    lens = T["lens"][:nd]
    di = dense_irrep(T)
    total, offs, strides = oracle.ref_dpd_layout(di, nirrep, lens, 5)
    geo = {}
    for b, t in enumerate(tuples(di, nirrep, nd)):
        shape = [lens[d][t[d]] for d in range(nd)]
        if np.prod(shape) > 0:
            geo[t] = (int(offs[b]), shape, [int(s) for s in strides[b]])
    return total, geo


def block_view(flat, off, shape, strides):
    return as_strided(flat[off:], shape=shape, strides=[flat.itemsize * s for s in strides])


def make(rng, nirrep, irrep, lens, idx_irreps, indices, factors=None):
    T = {"irrep": irrep, "lens": lens, "idx_irreps": idx_irreps, "indices": indices}
    n = max(1, len(indices)) if idx_irreps else 1
    size, _ = dense_geometry(T, nirrep)
    T["data"] = rng.uniform(-1, 1, n * size)
    T["factors"] = list(factors) if factors is not None else [1.0] * n
    return T


def full(T, nirrep):
    """block_to_full: the dense tensor over all irreps, entries scaled by
    their factors and placed at their index values."""
    nd = len(T["lens"]) - len(T["idx_irreps"])
    ext = [sum(r) for r in T["lens"]]
    off = [np.concatenate([[0], np.cumsum(r)[:-1]]).astype(int) for r in T["lens"]]
    F = np.zeros(ext, dtype=np.result_type(T["data"].dtype, np.float64))
    size, geo = dense_geometry(T, nirrep)
    entries = T["indices"] if T["idx_irreps"] else [[]]
    for e, ix in enumerate(entries):
        for t, (o, shape, st) in geo.items():
            blk = block_view(T["data"][e * size:], o, shape, st)
            sl = [slice(off[d][t[d]], off[d][t[d]] + shape[d]) for d in range(nd)]
            sl += [off[nd + i][T["idx_irreps"][i]] + ix[i] for i in range(len(ix))]
            F[tuple(sl)] = T["factors"][e] * blk
    return F


def restated_mult(nirrep, alpha, A, idx_A, B, idx_B, beta, C, idx_C):
    """C's storage after the contraction, in the FULL form."""
    out = C["data"].astype(np.result_type(C["data"].dtype, np.float64))
    size, geo = dense_geometry(C, nirrep)
    entries = C["indices"] if C["idx_irreps"] else [[]]
    # beta goes through the entries' factors (src/internal/1t/indexed_dpd/
    # scale.cxx, set.cxx): beta == 1 leaves C as is, beta == 0 or a zero
    # factor sets the entry to zero, otherwise entry e is scaled by f_e*beta
    for e in range(len(entries)):
        seg = out[e * size:(e + 1) * size]
        if beta == 0.0 or C["factors"][e] == 0.0:
            seg[:] = 0.0
        elif beta != 1.0:
            seg *= C["factors"][e] * beta
    C2 = alpha * np.einsum("%s,%s->%s" % (idx_A, idx_B, idx_C), full(A, nirrep), full(B, nirrep))
    nd = len(C["lens"]) - len(C["idx_irreps"])
    off = [np.concatenate([[0], np.cumsum(r)[:-1]]).astype(int) for r in C["lens"]]
    for e, ix in enumerate(entries):
        for t, (o, shape, st) in geo.items():
            blk = block_view(out[e * size:], o, shape, st)
            sl = [slice(off[d][t[d]], off[d][t[d]] + shape[d]) for d in range(nd)]
            sl += [off[nd + i][C["idx_irreps"][i]] + ix[i] for i in range(len(ix))]
            blk += C["factors"][e] * C2[tuple(sl)]
    return out


# contraction cases: (name, nirrep, label strings, builder)
def cases():
    out = []

    def ladder_indexed_j(rng):
        # C[abij] (j indexed) = A[abef] (dense) * B[efij] (j indexed)
        n = 2
        v, o = [3, 2], [2, 3]
        A = make(rng, n, 0, [v, v, v, v], [], [])
        B = make(rng, n, 1, [v, v, o, o], [1], [[0], [2]], factors=[0.5, -1.5])
        C = make(rng, n, 1, [v, v, o, o], [1], [[0], [1], [2]], factors=[1.0, 2.0, -0.25])
        return n, A, "abef", B, "efij", C, "abij"
    out.append(("ladder_indexed_j", ladder_indexed_j))

    def contracted_indexed(rng):
        # C[abij] = A[abem] (m indexed) * B[emij] (m indexed): contraction over entries
        n = 2
        v, o = [3, 2], [2, 2]
        A = make(rng, n, 1, [v, v, v, o], [1], [[0], [1]], factors=[1.0, 0.75])
        B = make(rng, n, 1, [v, o, o, o], [1], [[1], [0]], factors=[-1.0, 2.0])
        C = make(rng, n, 0, [v, v, o, o], [], [])
        return n, A, "abem", B, "emij", C, "abij"
    out.append(("contracted_indexed", contracted_indexed))

    def sliced_dense(rng):
        # i indexed in A, dense in C: each A entry writes one slice of C
        n = 4
        v, o = [2, 1, 2, 1], [1, 2, 1, 2]
        A = make(rng, n, 1, [v, v, o], [1], [[0], [1]], factors=[1.5, -0.5])
        B = make(rng, n, 2, [v, v], [], [])
        C = make(rng, n, 3, [v, v, o], [], [])
        return n, A, "aei", B, "eb", C, "abi"
    out.append(("sliced_dense", sliced_dense))

    def all_indexed_c(rng):
        # C[ai] with i indexed, one entry each in B and C
        n = 2
        v, o = [2, 3], [3, 1]
        A = make(rng, n, 0, [v, v], [], [])
        B = make(rng, n, 1, [v, o], [1], [[0]], factors=[2.0])
        C = make(rng, n, 1, [v, o], [1], [[0]], factors=[0.5])
        return n, A, "ae", B, "ei", C, "ai"
    out.append(("all_indexed_c", all_indexed_c))

    def scalar_slice(rng):
        # j indexed in A and dense in C: each A entry fills one element of C
        n = 2
        e, j = [2, 3], [2, 2]
        A = make(rng, n, 1, [e, j], [1], [[0], [1]], factors=[1.0, 3.0])
        B = make(rng, n, 0, [e], [], [])
        C = make(rng, n, 1, [j], [], [])
        return n, A, "ej", B, "e", C, "j"
    out.append(("scalar_slice", scalar_slice))
    return out
