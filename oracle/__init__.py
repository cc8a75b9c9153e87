"""oracle -- TEST INFRASTRUCTURE ONLY.

ctypes access to (1) the C restatement of the TBLIS reference algorithms
(oracle/tblis_oracle.c, built to oracle/_build/libtblis_oracle.so) and (2) the
reference library itself, compiled from its own sources by oracle/Makefile into
oracle/_ref/ (libtblis_ref.so plus librefshim.so, a shim exposing the block
scatter builder, the DPD layout and the C++ DPD entry point).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this package, and only as the checker or the timed CPU
baseline. The product (tblis_b200) never imports it.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(_HERE, "_build", "libtblis_oracle.so")
REF_SO = os.path.join(_HERE, "_ref", "libtblis_ref.so")
SHIM_SO = os.path.join(_HERE, "_ref", "librefshim.so")

_P = ctypes.POINTER
_sz = ctypes.c_ssize_t

_orc = None
_ref = None
_shim = None


class Scalar(ctypes.Structure):
    _fields_ = [("data", ctypes.c_double * 2), ("type", ctypes.c_int)]


class Tensor(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("conj", ctypes.c_int), ("scalar", Scalar),
                ("data", ctypes.c_void_p), ("ndim", ctypes.c_uint),
                ("len", _P(_sz)), ("stride", _P(_sz))]


def orc():
    """The C restatement (always available once built)."""
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError("oracle not built: make -C oracle oracle")
        _orc = ctypes.CDLL(ORACLE_SO)
        _orc.orc_tensor_reduce_d.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_uint, _P(_sz), _P(_sz),
                                             ctypes.c_void_p, ctypes.c_char_p, _P(ctypes.c_double), _P(_sz)]
        for f in ("orc_tensor_mult_d", "orc_tensor_add_d", "orc_tensor_dot_d", "orc_tensor_mult_sample_d",
                  "orc_mult_groups_build", "orc_tensor_scale_d", "orc_tensor_set_d", "orc_tensor_shift_d"):
            getattr(_orc, f).restype = ctypes.c_int
    return _orc


def have_ref():
    return os.path.exists(REF_SO) and os.path.exists(SHIM_SO)


def ref():
    """The reference TBLIS library built from its own sources."""
    global _ref, _shim
    if _ref is None:
        _ref = ctypes.CDLL(REF_SO)   # local: its static libstdc++ must not interpose
        _shim = ctypes.CDLL(SHIM_SO)
        _shim.refshim_dpd_layout.restype = ctypes.c_long
    return _ref


def shim():
    ref()
    return _shim


# ---- array helpers ------------------------------------------------------------------

def _lens_strides(a):
    n = a.ndim
    L = (_sz * max(n, 1))(*a.shape)
    S = (_sz * max(n, 1))(*[s // a.itemsize for s in a.strides])
    return L, S


def _lab(s):
    return s.encode() if isinstance(s, str) else s


_TYPE_OF = {np.dtype(np.float32): 0, np.dtype(np.float64): 1,
            np.dtype(np.complex64): 2, np.dtype(np.complex128): 3}
_DTYPE_OF = {v: k for k, v in _TYPE_OF.items()}


def _set_scalar(sc, value, type_):
    """Write value into a tblis_scalar's 16-byte union as the given type."""
    sc.type = type_
    raw = np.zeros(2, dtype=np.float64)
    raw.view(_DTYPE_OF[type_])[0] = value
    sc.data[0], sc.data[1] = raw[0], raw[1]


def _scalar_value(sc):
    raw = np.array([sc.data[0], sc.data[1]], dtype=np.float64)
    v = raw.view(_DTYPE_OF[sc.type])[0]
    return complex(v) if sc.type >= 2 else float(v)


def _tensor(a, alpha=1.0, keep=None, conj=False):
    L, S = _lens_strides(a)
    t = Tensor()
    t.type = _TYPE_OF[a.dtype]
    t.conj = 1 if conj else 0
    _set_scalar(t.scalar, alpha, t.type)
    t.data = a.ctypes.data
    t.ndim = a.ndim
    t.len = ctypes.cast(L, _P(_sz))
    t.stride = ctypes.cast(S, _P(_sz))
    if keep is not None:
        keep.extend([L, S])
    return t


# ---- the C restatement ----------------------------------------------------------------

def orc_mult(alpha, A, idx_A, B, idx_B, beta, C, idx_C):
    """C = alpha*A*B + beta*C in place (numpy float64 arrays, any strides)."""
    lA, sA = _lens_strides(A)
    lB, sB = _lens_strides(B)
    lC, sC = _lens_strides(C)
    rc = orc().orc_tensor_mult_d(ctypes.c_double(alpha), A.ndim, lA, sA, ctypes.c_void_p(A.ctypes.data), _lab(idx_A),
                                 B.ndim, lB, sB, ctypes.c_void_p(B.ctypes.data), _lab(idx_B),
                                 ctypes.c_double(beta), C.ndim, lC, sC, ctypes.c_void_p(C.ctypes.data), _lab(idx_C))
    if rc:
        raise ValueError("oracle mult failed: %d" % rc)


def orc_mult_sample(alpha, A, idx_A, B, idx_B, beta, C, idx_C, sample_idx):
    """alpha*sum A*B + beta*C at the given multi-indices of C (rows of sample_idx)."""
    sample_idx = np.ascontiguousarray(sample_idx, dtype=np.int64)
    out = np.empty(sample_idx.shape[0], dtype=np.float64)
    lA, sA = _lens_strides(A)
    lB, sB = _lens_strides(B)
    lC, sC = _lens_strides(C)
    rc = orc().orc_tensor_mult_sample_d(
        ctypes.c_double(alpha), A.ndim, lA, sA, ctypes.c_void_p(A.ctypes.data), _lab(idx_A),
        B.ndim, lB, sB, ctypes.c_void_p(B.ctypes.data), _lab(idx_B),
        ctypes.c_double(beta), C.ndim, lC, sC, ctypes.c_void_p(C.ctypes.data), _lab(idx_C),
        _sz(sample_idx.shape[0]), ctypes.c_void_p(sample_idx.ctypes.data), ctypes.c_void_p(out.ctypes.data))
    if rc:
        raise ValueError("oracle sample failed: %d" % rc)
    return out


def orc_add(alpha, A, idx_A, beta, B, idx_B):
    lA, sA = _lens_strides(A)
    lB, sB = _lens_strides(B)
    rc = orc().orc_tensor_add_d(ctypes.c_double(alpha), A.ndim, lA, sA, ctypes.c_void_p(A.ctypes.data), _lab(idx_A),
                                ctypes.c_double(beta), B.ndim, lB, sB, ctypes.c_void_p(B.ctypes.data), _lab(idx_B))
    if rc:
        raise ValueError("oracle add failed: %d" % rc)


def orc_dot(A, idx_A, B, idx_B, alpha_A=1.0, alpha_B=1.0):
    lA, sA = _lens_strides(A)
    lB, sB = _lens_strides(B)
    r = ctypes.c_double()
    rc = orc().orc_tensor_dot_d(ctypes.c_double(alpha_A), A.ndim, lA, sA, ctypes.c_void_p(A.ctypes.data), _lab(idx_A),
                                ctypes.c_double(alpha_B), B.ndim, lB, sB, ctypes.c_void_p(B.ctypes.data), _lab(idx_B),
                                ctypes.byref(r))
    if rc:
        raise ValueError("oracle dot failed: %d" % rc)
    return r.value


def orc_reduce(op, A, idx_A, alpha=1.0):
    lA, sA = _lens_strides(A)
    r = ctypes.c_double()
    i = _sz()
    rc = orc().orc_tensor_reduce_d(op, alpha, A.ndim, lA, sA, ctypes.c_void_p(A.ctypes.data), _lab(idx_A),
                                   ctypes.byref(r), ctypes.byref(i))
    if rc:
        raise ValueError("oracle reduce failed: %d" % rc)
    return r.value, i.value


def orc_unary(kind, A, alpha=1.0, shift=0.0):
    """kind: 'set' (A = alpha), 'scale' (A *= alpha), 'shift' (A = shift + alpha*A)."""
    lA, sA = _lens_strides(A)
    p = ctypes.c_void_p(A.ctypes.data)
    if kind == "set":
        return orc().orc_tensor_set_d(ctypes.c_double(alpha), A.ndim, lA, sA, p)
    if kind == "scale":
        return orc().orc_tensor_scale_d(ctypes.c_double(alpha), A.ndim, lA, sA, p)
    return orc().orc_tensor_shift_d(ctypes.c_double(shift), ctypes.c_double(alpha), A.ndim, lA, sA, p)


def orc_fill_block_scatter(lens, strides, BS, off, size, pack_3d):
    n = len(lens)
    L = (_sz * max(n, 1))(*lens)
    S = (_sz * max(n, 1))(*strides)
    scat = np.zeros(max(size, 1), dtype=np.int64)
    bs = np.zeros(max(size, 1), dtype=np.int64)
    orc().orc_fill_block_scatter(n, L, S, _sz(BS), _sz(off), _sz(size), ctypes.c_void_p(scat.ctypes.data),
                                 ctypes.c_void_p(bs.ctypes.data), int(pack_3d))
    return scat[:size], bs[:size]


def orc_mult_groups(A, idx_A, B, idx_B, C, idx_C):
    """Group split of the restatement: dict of label strings after fold."""
    class G(ctypes.Structure):
        M = 16
        _fields_ = ([("n_AB", ctypes.c_uint), ("n_AC", ctypes.c_uint), ("n_BC", ctypes.c_uint), ("n_ABC", ctypes.c_uint)]
                    + [(n, ctypes.c_char * 16) for n in ("idx_AB", "idx_AC", "idx_BC", "idx_ABC")]
                    + [(n, _sz * 16) for n in ("len_AB", "len_AC", "len_BC", "len_ABC", "sA_AB", "sB_AB",
                                               "sA_AC", "sC_AC", "sB_BC", "sC_BC", "sA_ABC", "sB_ABC", "sC_ABC")])
    lA, sA = _lens_strides(A)
    lB, sB = _lens_strides(B)
    lC, sC = _lens_strides(C)
    g = G()
    rc = orc().orc_mult_groups_build(A.ndim, lA, sA, _lab(idx_A), B.ndim, lB, sB, _lab(idx_B),
                                     C.ndim, lC, sC, _lab(idx_C), ctypes.byref(g))
    if rc:
        raise ValueError("oracle groups failed: %d" % rc)
    out = {}
    for grp in ("AB", "AC", "BC", "ABC"):
        n = getattr(g, "n_" + grp)
        out[grp] = bytes(getattr(g, "idx_" + grp)[:n]).decode("latin1")
        out["len_" + grp] = list(getattr(g, "len_" + grp)[:n])
    return out


# ---- the reference itself -----------------------------------------------------------------

def ref_mult(alpha, A, idx_A, B, idx_B, beta, C, idx_C, threads=None, conj_A=False, conj_B=False):
    """The reference's tblis_tensor_mult (double or dcomplex numpy arrays)."""
    keep = []
    r = ref()
    if threads:
        r.tblis_set_num_threads(int(threads))
    tA = _tensor(A, alpha, keep, conj_A)
    tB = _tensor(B, 1.0, keep, conj_B)
    tC = _tensor(C, beta, keep)
    r.tblis_tensor_mult(None, None, ctypes.byref(tA), _lab(idx_A), ctypes.byref(tB), _lab(idx_B),
                        ctypes.byref(tC), _lab(idx_C))


def ref_add(alpha, A, idx_A, beta, B, idx_B, threads=None, conj_A=False, conj_B=False):
    keep = []
    r = ref()
    if threads:
        r.tblis_set_num_threads(int(threads))
    tA = _tensor(A, alpha, keep, conj_A)
    tB = _tensor(B, beta, keep, conj_B)
    r.tblis_tensor_add(None, None, ctypes.byref(tA), _lab(idx_A), ctypes.byref(tB), _lab(idx_B))


def ref_dot(A, idx_A, B, idx_B, conj_A=False, conj_B=False):
    """The reference's tblis_tensor_dot (a float, or a complex for complex arrays)."""
    keep = []
    tA = _tensor(A, 1.0, keep, conj_A)
    tB = _tensor(B, 1.0, keep, conj_B)
    s = Scalar()
    s.type = tA.type
    ref().tblis_tensor_dot(None, None, ctypes.byref(tA), _lab(idx_A), ctypes.byref(tB), _lab(idx_B), ctypes.byref(s))
    return _scalar_value(s)


def ref_reduce(op, A, idx_A, alpha=1.0, conj=False):
    keep = []
    tA = _tensor(A, alpha, keep, conj)
    s = Scalar()
    s.type = tA.type
    i = _sz(-1)
    ref().tblis_tensor_reduce(None, None, op, ctypes.byref(tA), _lab(idx_A), ctypes.byref(s), ctypes.byref(i))
    return _scalar_value(s), i.value


def ref_unary(kind, A, idx_A, alpha=1.0, value=0.0, conj=False):
    """The reference's tblis_tensor_scale (kind 1: A = alpha*op(A)), set
    (0: A = value) and shift (2: A = value + alpha*op(A)), in place."""
    keep = []
    tA = _tensor(A, alpha, keep, conj)
    v = Scalar()
    _set_scalar(v, value, tA.type)
    r = ref()
    if kind == 0:
        r.tblis_tensor_set(None, None, ctypes.byref(v), ctypes.byref(tA), _lab(idx_A))
    elif kind == 1:
        r.tblis_tensor_scale(None, None, ctypes.byref(tA), _lab(idx_A))
    else:
        r.tblis_tensor_shift(None, None, ctypes.byref(v), ctypes.byref(tA), _lab(idx_A))


def ref_fill_block_scatter(lens, strides, BS, off, size, pack_3d):
    n = len(lens)
    L = (_sz * max(n, 1))(*lens)
    S = (_sz * max(n, 1))(*strides)
    scat = np.zeros(max(size, 1), dtype=np.int64)
    bs = np.zeros(max(size, 1), dtype=np.int64)
    shim().refshim_fill_block_scatter(n, L, S, _sz(BS), _sz(off), _sz(size), ctypes.c_void_p(scat.ctypes.data),
                                      ctypes.c_void_p(bs.ctypes.data), int(pack_3d))
    return scat[:size], bs[:size]


def ref_dpd_layout(irrep, nirrep, lens, layout=5):
    """(total_size, block_offsets[nblock], block_strides[nblock][ndim]) from MArray."""
    ndim = len(lens)
    flat = (_sz * (ndim * nirrep))(*[x for row in lens for x in row])
    nb = nirrep ** (ndim - 1)
    offs = np.zeros(nb, dtype=np.int64)
    strides = np.zeros(nb * ndim, dtype=np.int64)
    total = shim().refshim_dpd_layout(irrep, nirrep, ndim, flat, layout, ctypes.c_void_p(offs.ctypes.data),
                                      ctypes.c_void_p(strides.ctypes.data), ctypes.c_long(nb))
    return total, offs, strides.reshape(nb, ndim)


def _dpd_blocks_ref(irrep, nirrep, lens):
    """(irreps, offset, strides) of every stored block of a default-layout DPD
    tensor, from the reference's MArray layout (ref_dpd_layout); the block
    order is the one refshim_dpd_layout walks: irreps of dimensions 1.. (the
    first fastest), dimension 0 closing the XOR."""
    ndim = len(lens)
    total, offs, strides = ref_dpd_layout(irrep, nirrep, lens, 5)
    out = []
    for b in range(len(offs)):
        irr = [0] * ndim
        t, x = b, irrep
        for i in range(1, ndim):
            irr[i] = t % nirrep
            t //= nirrep
            x ^= irr[i]
        irr[0] = x
        out.append((irr, int(offs[b]), [int(v) for v in strides[b]]))
    return total, out


def orc_dpd_block_to_full(irrep, nirrep, lens, data):
    """The dense form of a default-layout DPD tensor, restating
    src/internal/1t/dpd/util.hpp:70-102 (block_to_full): dimension d has the
    sum of the lengths over the irreps, irrep x starting after the lengths of
    the irreps below it; zero everywhere, then every stored block copied into
    its region. Block geometry from the reference's MArray layout."""
    dims = [sum(r) for r in lens]
    full = np.zeros(dims, dtype=data.dtype)
    _, blocks = _dpd_blocks_ref(irrep, nirrep, lens)
    for irr, off, strides in blocks:
        bl = [lens[d][irr[d]] for d in range(len(lens))]
        if 0 in bl:
            continue
        blk = np.lib.stride_tricks.as_strided(data[off:], shape=bl, strides=[data.itemsize * s for s in strides])
        sl = tuple(slice(sum(lens[d][:irr[d]]), sum(lens[d][:irr[d]]) + bl[d]) for d in range(len(lens)))
        full[sl] = blk
    return full


def orc_dpd_full_to_block(irrep, nirrep, lens, full, data):
    """The reverse, restating src/internal/1t/dpd/util.hpp:104-133
    (full_to_block): every stored block of `data` (updated in place) gets a
    copy of its region of `full`."""
    _, blocks = _dpd_blocks_ref(irrep, nirrep, lens)
    for irr, off, strides in blocks:
        bl = [lens[d][irr[d]] for d in range(len(lens))]
        if 0 in bl:
            continue
        blk = np.lib.stride_tricks.as_strided(data[off:], shape=bl, strides=[data.itemsize * s for s in strides])
        sl = tuple(slice(sum(lens[d][:irr[d]]), sum(lens[d][:irr[d]]) + bl[d]) for d in range(len(lens)))
        blk[...] = full[sl]


# ---- DPD ----------------------------------------------------------------------------------

def orc_dpd_block(irrep, nirrep, lens, layout, irreps):
    """(offset, lengths, strides) of one block from the C restatement."""
    ndim = len(lens)
    flat = (_sz * (ndim * nirrep))(*[x for row in lens for x in row])
    irr = (ctypes.c_uint * ndim)(*irreps)
    bl = (_sz * ndim)()
    bs = (_sz * ndim)()
    off = _sz()
    rc = orc().orc_dpd_block(irrep, nirrep, ndim, flat, layout, irr, bl, bs, ctypes.byref(off))
    if rc:
        raise ValueError("oracle dpd_block failed: %d" % rc)
    return off.value, list(bl), list(bs)


def orc_dpd_size(irrep, nirrep, lens, layout):
    ndim = len(lens)
    flat = (_sz * (ndim * nirrep))(*[x for row in lens for x in row])
    f = orc().orc_dpd_size
    f.restype = _sz
    return f(irrep, nirrep, ndim, flat, layout)


def ref_dpd_mult(nirrep, alpha, irrep_A, lens_A, A, idx_A, irrep_B, lens_B, B, idx_B,
                 beta, irrep_C, lens_C, C, idx_C):
    """The reference's own C++ DPD contraction (tblis::mult over
    dpd_varray_view, default layout) on flat numpy storage; C updated in place."""
    def flat(lens):
        return (_sz * (len(lens) * nirrep))(*[x for row in lens for x in row])
    rc = shim().refshim_dpd_mult(
        nirrep, ctypes.c_double(alpha), irrep_A, len(lens_A), flat(lens_A), ctypes.c_void_p(A.ctypes.data), _lab(idx_A),
        irrep_B, len(lens_B), flat(lens_B), ctypes.c_void_p(B.ctypes.data), _lab(idx_B),
        ctypes.c_double(beta), irrep_C, len(lens_C), flat(lens_C), ctypes.c_void_p(C.ctypes.data), _lab(idx_C))
    if rc:
        raise ValueError("reference dpd mult failed")


def _idx_args(nirrep, T, lab):
    ndim = len(T["lens"])
    nidim = len(T["idx_irreps"])
    flat = (_sz * (ndim * nirrep))(*[x for row in T["lens"] for x in row])
    irr = (ctypes.c_uint * max(1, nidim))(*T["idx_irreps"])
    idx = [x for t in T["indices"] for x in t]
    nidx = max(1, len(T["indices"])) if nidim else 1
    ix = (_sz * max(1, len(idx)))(*idx)
    f = (ctypes.c_double * nidx)(*T["factors"])
    return [ctypes.c_uint(T["irrep"]), ctypes.c_uint(ndim), flat, ctypes.c_uint(nidim), irr, ctypes.c_long(nidx),
            ix, ctypes.c_void_p(T["data"].ctypes.data), f, _lab(lab)]


def ref_indexed_dpd_add(nirrep, alpha, A, idx_A, beta, B, idx_B):
    """The reference's tblis::add over indexed_dpd_varray_view; B's data updated."""
    shim().refshim_indexed_dpd_add(ctypes.c_uint(nirrep), ctypes.c_double(alpha), *_idx_args(nirrep, A, idx_A),
                                   ctypes.c_double(beta), *_idx_args(nirrep, B, idx_B))


def ref_indexed_dpd_dot(nirrep, A, idx_A, B, idx_B):
    f = shim().refshim_indexed_dpd_dot
    f.restype = ctypes.c_double
    return f(ctypes.c_uint(nirrep), *_idx_args(nirrep, A, idx_A), *_idx_args(nirrep, B, idx_B))


def ref_indexed_dpd_reduce(op, nirrep, A, idx_A):
    r = ctypes.c_double()
    i = ctypes.c_long()
    shim().refshim_indexed_dpd_reduce(ctypes.c_int(op), ctypes.c_uint(nirrep), *_idx_args(nirrep, A, idx_A),
                                      ctypes.byref(r), ctypes.byref(i))
    return r.value, i.value


def ref_indexed_dpd_unary(kind, alpha, beta, nirrep, A, idx_A):
    shim().refshim_indexed_dpd_unary(ctypes.c_int(kind), ctypes.c_double(alpha), ctypes.c_double(beta),
                                     ctypes.c_uint(nirrep), *_idx_args(nirrep, A, idx_A))


def ref_indexed_dpd_mult(nirrep, alpha, A, idx_A, B, idx_B, beta, C, idx_C, impl=2):
    """The reference's own indexed-DPD contraction (tblis::mult over
    indexed_dpd_varray_view). Each tensor is a dict: irrep (overall), lens
    [ndim][nirrep], idx_irreps, indices [nidx][nidim], data (numpy, nidx x
    dense size, default layout), factors. C's data is updated in place.
    impl: 0 = the reference's default block path, 1 = BLOCKED, 2 = FULL (the
    dense round trip its own tests take as the answer, test/3t/mult.cxx:176-232)."""
    def args(T):
        ndim = len(T["lens"])
        nidim = len(T["idx_irreps"])
        flat = (_sz * (ndim * nirrep))(*[x for row in T["lens"] for x in row])
        irr = (ctypes.c_uint * max(1, nidim))(*T["idx_irreps"])
        idx = [x for t in T["indices"] for x in t]
        nidx = max(1, len(T["indices"])) if nidim else 1
        ix = (_sz * max(1, len(idx)))(*idx)
        f = (ctypes.c_double * nidx)(*T["factors"])
        return [ctypes.c_uint(T["irrep"]), ctypes.c_uint(ndim), flat, ctypes.c_uint(nidim), irr, ctypes.c_long(nidx),
                ix, ctypes.c_void_p(T["data"].ctypes.data), f]
    a = args(A) + [_lab(idx_A)]
    b = args(B) + [_lab(idx_B)]
    c = args(C) + [_lab(idx_C)]
    rc = shim().refshim_indexed_dpd_mult(ctypes.c_uint(nirrep), ctypes.c_double(alpha), *a, *b,
                                         ctypes.c_double(beta), *c, ctypes.c_int(impl))
    if rc:
        raise ValueError("reference indexed dpd mult failed")


def ref_dense_impl(impl):
    """Selects the reference's dense contraction implementation: 0 = its
    default BLIS-based path, 2 = REFERENCE (mult_ref,
    src/internal/3t/dense/mult.cxx:653-720), which applies conjugation flags
    (the default path asserts them off). Returns the previous value."""
    return shim().refshim_set_dense_impl(int(impl))


def ref_dpd_impl(impl):
    """Selects the reference's DPD contraction implementation for the plain
    DPD entry points: 0 = its default block path (BLIS), 1 = BLOCKED, 2 =
    FULL (dense round trip). Returns the previous value."""
    return shim().refshim_set_dpd_impl(int(impl))


def _dpd_flat(nirrep, lens):
    return (_sz * (len(lens) * nirrep))(*[x for row in lens for x in row])


def _value_buf(value, dtype):
    """A 16-byte buffer holding value as one element of dtype."""
    b = np.zeros(2, dtype=np.float64)
    b.view(np.dtype(dtype))[0] = value
    return b


def ref_dpd_mult_typed(nirrep, alpha, irrep_A, lens_A, A, idx_A, irrep_B, lens_B, B, idx_B,
                       beta, irrep_C, lens_C, C, idx_C):
    """The reference's tblis::mult over dpd_varray_view for the element type of
    the numpy storage (float32, float64, complex64, complex128); C in place."""
    t = _TYPE_OF[C.dtype]
    a, b = _value_buf(alpha, C.dtype), _value_buf(beta, C.dtype)
    rc = shim().refshim_dpd_mult_t(
        t, nirrep, ctypes.c_void_p(a.ctypes.data), irrep_A, len(lens_A), _dpd_flat(nirrep, lens_A),
        ctypes.c_void_p(A.ctypes.data), _lab(idx_A), irrep_B, len(lens_B), _dpd_flat(nirrep, lens_B),
        ctypes.c_void_p(B.ctypes.data), _lab(idx_B), ctypes.c_void_p(b.ctypes.data), irrep_C, len(lens_C),
        _dpd_flat(nirrep, lens_C), ctypes.c_void_p(C.ctypes.data), _lab(idx_C))
    if rc:
        raise ValueError("reference dpd mult failed")


def ref_dpd_level1_typed(op, nirrep, irrep_A, lens_A, A, idx_A, irrep_B=0, lens_B=None, B=None, idx_B="",
                         alpha=1.0, beta=0.0):
    """The reference's DPD level-1 operation for A's element type. op: "add"
    (B = alpha*A + beta*B), "dot", "scale" (A *= alpha), "set" (A = alpha),
    "shift" (A = alpha + beta*A), or ("reduce", r). Returns the dot value, a
    (value, idx) pair for a reduction, else None; A / B updated in place."""
    codes = {"add": 0, "dot": 1, "scale": 2, "set": 3, "shift": 4}
    code = 10 + op[1] if isinstance(op, tuple) else codes[op]
    a, b = _value_buf(alpha, A.dtype), _value_buf(beta, A.dtype)
    res = np.zeros(2, dtype=np.float64)
    i = ctypes.c_long(-1)
    lb = _dpd_flat(nirrep, lens_B) if lens_B is not None else None
    rc = shim().refshim_dpd_level1_t(
        _TYPE_OF[A.dtype], code, nirrep, ctypes.c_void_p(a.ctypes.data), ctypes.c_void_p(b.ctypes.data),
        irrep_A, len(lens_A), _dpd_flat(nirrep, lens_A), ctypes.c_void_p(A.ctypes.data), _lab(idx_A),
        irrep_B, len(lens_B) if lens_B is not None else 0, lb,
        ctypes.c_void_p(B.ctypes.data) if B is not None else None, _lab(idx_B),
        ctypes.c_void_p(res.ctypes.data), ctypes.byref(i))
    if rc:
        raise ValueError("reference dpd level-1 failed")
    v = res.view(A.dtype)[0]
    v = complex(v) if np.dtype(A.dtype).kind == "c" else float(v)
    if code == 1:
        return v
    if code >= 10:
        return v, i.value
    return None


def ref_dpd_add(nirrep, alpha, irrep_A, lens_A, A, idx_A, beta, irrep_B, lens_B, B, idx_B):
    """The reference's tblis::add over dpd_varray_view (default layout storage)."""
    rc = shim().refshim_dpd_add(nirrep, ctypes.c_double(alpha), irrep_A, len(lens_A), _dpd_flat(nirrep, lens_A),
                                ctypes.c_void_p(A.ctypes.data), _lab(idx_A), ctypes.c_double(beta), irrep_B,
                                len(lens_B), _dpd_flat(nirrep, lens_B), ctypes.c_void_p(B.ctypes.data), _lab(idx_B))
    if rc:
        raise ValueError("reference dpd add failed")


def ref_dpd_dot(nirrep, irrep_A, lens_A, A, idx_A, irrep_B, lens_B, B, idx_B):
    f = shim().refshim_dpd_dot
    f.restype = ctypes.c_double
    return f(nirrep, irrep_A, len(lens_A), _dpd_flat(nirrep, lens_A), ctypes.c_void_p(A.ctypes.data), _lab(idx_A),
             irrep_B, len(lens_B), _dpd_flat(nirrep, lens_B), ctypes.c_void_p(B.ctypes.data), _lab(idx_B))


def ref_dpd_reduce(op, nirrep, irrep_A, lens_A, A, idx_A):
    r = ctypes.c_double()
    i = ctypes.c_long()
    shim().refshim_dpd_reduce(int(op), nirrep, irrep_A, len(lens_A), _dpd_flat(nirrep, lens_A),
                              ctypes.c_void_p(A.ctypes.data), _lab(idx_A), ctypes.byref(r), ctypes.byref(i))
    return r.value, i.value


def ref_dpd_unary(kind, alpha, beta, nirrep, irrep_A, lens_A, A, idx_A):
    """kind 0: A *= alpha; 1: A = alpha; 2: A = alpha + beta*A (reference, in place)."""
    shim().refshim_dpd_unary(int(kind), ctypes.c_double(alpha), ctypes.c_double(beta), nirrep, irrep_A,
                             len(lens_A), _dpd_flat(nirrep, lens_A), ctypes.c_void_p(A.ctypes.data), _lab(idx_A))
