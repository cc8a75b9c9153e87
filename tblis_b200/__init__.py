"""tblis_b200 -- Python mirror of TBLIS's tensor interface over the B200 C ABI.

The functions mirror the reference's C++ wrappers (src/iface/3t/mult.h:28-38,
src/iface/1t/add.h:27-35, src/iface/1t/dot.h, src/iface/1t/reduce.h:28-60,
src/iface/1t/scale.h, set.h, shift.h): same names, same argument order and
meaning (alpha/beta carried as tensor scalars, index strings as labels), and
every call goes through ``libtblis_b200.so``'s C ABI (``tblis_tensor_*``), which
runs hand-written sm_100a kernels. There is no CPU fallback: importing fails if
the shared library is missing, and calls fail if no CUDA device is visible.

Tensors may be torch tensors (device or host) or numpy arrays (host); host
data is staged to the GPU by the library around the call.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libtblis_b200.so")

if not os.path.exists(_LIB_PATH):
    raise ImportError(
        "tblis_b200: %s is not built (run `make -C tblis_b200` or __graft_entry__.build())"
        % _LIB_PATH)

lib = ctypes.CDLL(_LIB_PATH)

TYPE_FLOAT, TYPE_DOUBLE, TYPE_SCOMPLEX, TYPE_DCOMPLEX = 0, 1, 2, 3
REDUCE_SUM, REDUCE_SUM_ABS, REDUCE_MAX, REDUCE_MAX_ABS = 0, 1, 2, 3
REDUCE_MIN, REDUCE_MIN_ABS, REDUCE_NORM_2 = 4, 5, 6
REDUCE_NORM_1, REDUCE_NORM_INF = REDUCE_SUM_ABS, REDUCE_MAX_ABS


class tblis_scalar(ctypes.Structure):
    """src/util/basic_types.h:154-175 (16-byte value union + type tag)."""
    _fields_ = [("data", ctypes.c_double * 2), ("type", ctypes.c_int)]


class tblis_tensor(ctypes.Structure):
    """src/util/basic_types.h:471-479."""
    _fields_ = [("type", ctypes.c_int), ("conj", ctypes.c_int), ("scalar", tblis_scalar),
                ("data", ctypes.c_void_p), ("ndim", ctypes.c_uint),
                ("len", ctypes.POINTER(ctypes.c_ssize_t)),
                ("stride", ctypes.POINTER(ctypes.c_ssize_t))]


class tblis_b200_opts(ctypes.Structure):
    _fields_ = [("method", ctypes.c_int), ("slices", ctypes.c_int), ("tolerance", ctypes.c_double)]


class tblis_b200_report(ctypes.Structure):
    _fields_ = [("method", ctypes.c_int), ("slices", ctypes.c_int), ("est_error", ctypes.c_double),
                ("flops", ctypes.c_double), ("m", ctypes.c_int64), ("n", ctypes.c_int64),
                ("k", ctypes.c_int64), ("l", ctypes.c_int64), ("kernels", ctypes.c_int)]


assert ctypes.sizeof(tblis_scalar) == 24 and ctypes.sizeof(tblis_tensor) == 64

_P = ctypes.POINTER
lib.tblis_tensor_mult.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _P(tblis_tensor), ctypes.c_char_p,
                                  _P(tblis_tensor), ctypes.c_char_p, _P(tblis_tensor), ctypes.c_char_p]
lib.tblis_tensor_add.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _P(tblis_tensor), ctypes.c_char_p,
                                 _P(tblis_tensor), ctypes.c_char_p]
lib.tblis_tensor_dot.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _P(tblis_tensor), ctypes.c_char_p,
                                 _P(tblis_tensor), ctypes.c_char_p, _P(tblis_scalar)]
lib.tblis_tensor_reduce.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, _P(tblis_tensor),
                                    ctypes.c_char_p, _P(tblis_scalar), _P(ctypes.c_ssize_t)]
lib.tblis_tensor_scale.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _P(tblis_tensor), ctypes.c_char_p]
lib.tblis_tensor_set.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _P(tblis_scalar), _P(tblis_tensor),
                                 ctypes.c_char_p]
lib.tblis_tensor_shift.argtypes = lib.tblis_tensor_set.argtypes
lib.tblis_get_config.argtypes = [ctypes.c_char_p]
lib.tblis_get_config.restype = ctypes.c_void_p
lib.tblis_b200_last_error.restype = ctypes.c_int
lib.tblis_b200_last_error_string.restype = ctypes.c_char_p
lib.tblis_b200_tensor_mult_ex.argtypes = [ctypes.c_void_p, _P(tblis_tensor), ctypes.c_char_p,
                                          _P(tblis_tensor), ctypes.c_char_p, _P(tblis_tensor),
                                          ctypes.c_char_p, _P(tblis_b200_opts), _P(tblis_b200_report)]
lib.tblis_b200_tensor_mult_ex.restype = ctypes.c_int
lib.tblis_b200_fill_block_scatter.argtypes = [ctypes.c_uint, _P(ctypes.c_ssize_t), _P(ctypes.c_ssize_t),
                                              ctypes.c_ssize_t, ctypes.c_ssize_t, ctypes.c_ssize_t,
                                              _P(ctypes.c_ssize_t), _P(ctypes.c_ssize_t), ctypes.c_int]
lib.tblis_b200_mult_groups.argtypes = [_P(tblis_tensor), ctypes.c_char_p, _P(tblis_tensor),
                                       ctypes.c_char_p, _P(tblis_tensor), ctypes.c_char_p,
                                       ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                       ctypes.c_char_p, _P(ctypes.c_int64)]
lib.tblis_b200_mult_groups.restype = ctypes.c_int
lib.tblis_b200_kernel_count.restype = ctypes.c_int64
lib.tblis_b200_kernel_timer.argtypes = [ctypes.c_int]
lib.tblis_b200_kernel_timer_read.argtypes = [ctypes.c_char_p, _P(ctypes.c_double), _P(ctypes.c_int64)]
lib.tblis_b200_set_stream.argtypes = [ctypes.c_void_p]
lib.tblis_b200_get_stream.restype = ctypes.c_void_p
lib.tblis_b200_config_set_tolerance.argtypes = [ctypes.c_void_p, ctypes.c_double]


class TblisError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("tblis_b200 error %d: %s" % (code, msg))
        self.code = code


def _check():
    code = lib.tblis_b200_last_error()
    if code:
        msg = lib.tblis_b200_last_error_string().decode()
        lib.tblis_b200_clear_error()
        raise TblisError(code, msg)


def _labels(idx):
    if isinstance(idx, bytes):
        return idx
    return idx.encode()


def _dtype_code(x):
    name = str(getattr(x, "dtype", ""))
    if name.endswith("float64"):
        return TYPE_DOUBLE, 8
    if name.endswith("float32"):
        return TYPE_FLOAT, 4
    if name.endswith("complex128"):
        return TYPE_DCOMPLEX, 16
    if name.endswith("complex64"):
        return TYPE_SCOMPLEX, 8
    raise TypeError("tblis_b200: unsupported dtype %s" % name)


class _View:
    """A tblis_tensor describing a torch tensor or numpy array (no copy)."""

    def __init__(self, x, scalar=1.0, conj=False):
        self.obj = x
        code, esize = _dtype_code(x)
        if hasattr(x, "data_ptr"):          # torch
            shape = tuple(x.shape)
            strides = tuple(x.stride())
            ptr = x.data_ptr()
        else:                                # numpy
            shape = tuple(x.shape)
            strides = tuple(s // esize for s in x.strides)
            ptr = x.ctypes.data
        n = len(shape)
        self.len = (ctypes.c_ssize_t * max(n, 1))(*shape)
        self.stride = (ctypes.c_ssize_t * max(n, 1))(*strides)
        t = tblis_tensor()
        t.type = code
        t.conj = 1 if conj else 0
        t.scalar = _make_scalar(scalar, code)
        t.data = ptr
        t.ndim = n
        t.len = self.len          # ctypes converts the arrays to the pointer fields
        t.stride = self.stride
        self.t = t

    @property
    def ref(self):
        return ctypes.byref(self.t)


def get_config(name):
    """src/util/configs.h:11 -- a configuration handle by name (or None)."""
    p = lib.tblis_get_config(name.encode())
    return p


def mult(alpha, A, idx_A, B, idx_B, beta, C, idx_C, cfg=None, conj_A=False, conj_B=False):
    """C[idx_C] = alpha*A[idx_A]*B[idx_B] + beta*C[idx_C] (src/iface/3t/mult.h:28-38);
    conj_A / conj_B conjugate complex operands."""
    a, b, c = _View(A, alpha, conj_A), _View(B, 1.0, conj_B), _View(C, beta)
    lib.tblis_tensor_mult(None, cfg, a.ref, _labels(idx_A), b.ref, _labels(idx_B), c.ref, _labels(idx_C))
    _check()


def mult_ex(alpha, A, idx_A, B, idx_B, beta, C, idx_C, method=0, slices=0, tolerance=0.0, cfg=None,
            conj_A=False, conj_B=False):
    """mult with an explicit method and a report dict. Methods: 1 = FP64 DMMA,
    2 = Ozaki INT8 (slices or moduli, whichever needs less INT8 work; a given
    slice count forces slices), 3 = Ozaki BF16 slices (slice count from the
    tolerance unless given), 4 = one TF32 pass, 5 = one BF16 pass, 6 = Ozaki
    INT8 over moduli (scheme II; `slices` counts the moduli). The report's
    method is 6 when method 2 chose moduli."""
    a, b, c = _View(A, alpha, conj_A), _View(B, 1.0, conj_B), _View(C, beta)
    o = tblis_b200_opts(method, slices, tolerance)
    r = tblis_b200_report()
    lib.tblis_b200_tensor_mult_ex(cfg, a.ref, _labels(idx_A), b.ref, _labels(idx_B), c.ref,
                                  _labels(idx_C), ctypes.byref(o), ctypes.byref(r))
    _check()
    return {f: getattr(r, f) for f, _ in tblis_b200_report._fields_}


def add(alpha, A, idx_A, beta, B, idx_B, conj_A=False, conj_B=False):
    """B[idx_B] = alpha*op(A[idx_A]) + beta*op(B[idx_B]) (src/iface/1t/add.h:27-35);
    op conjugates a complex operand whose flag is set."""
    a, b = _View(A, alpha, conj_A), _View(B, beta, conj_B)
    lib.tblis_tensor_add(None, None, a.ref, _labels(idx_A), b.ref, _labels(idx_B))
    _check()


def dot(A, idx_A, B, idx_B, conj_A=False, conj_B=False):
    """sum over all labels of op(A)*op(B) (src/iface/1t/dot.h)."""
    a, b = _View(A, 1.0, conj_A), _View(B, 1.0, conj_B)
    r = tblis_scalar()
    lib.tblis_tensor_dot(None, None, a.ref, _labels(idx_A), b.ref, _labels(idx_B), ctypes.byref(r))
    _check()
    return _scalar_value(r, a.t.type)


def reduce(op, A, idx_A, conj=False):
    """(value, offset) of a reduction (src/iface/1t/reduce.h:47-53)."""
    a = _View(A, 1.0, conj)
    r = tblis_scalar()
    r.type = a.t.type
    idx = ctypes.c_ssize_t(-1)
    lib.tblis_tensor_reduce(None, None, int(op), a.ref, _labels(idx_A), ctypes.byref(r), ctypes.byref(idx))
    _check()
    return _scalar_value(r, a.t.type), idx.value


def scale(alpha, A, idx_A, conj=False):
    """A = alpha*op(A) (src/iface/1t/scale.h)."""
    a = _View(A, alpha, conj)
    lib.tblis_tensor_scale(None, None, a.ref, _labels(idx_A))
    _check()


def set(alpha, A, idx_A):  # noqa: A001 -- mirrors tblis::set
    """A = alpha (src/iface/1t/set.h)."""
    a = _View(A)
    s = _make_scalar(alpha, a.t.type)
    lib.tblis_tensor_set(None, None, ctypes.byref(s), a.ref, _labels(idx_A))
    _check()


def shift(alpha, beta, A, idx_A, conj=False):
    """A = alpha + beta*op(A) (src/iface/1t/shift.h)."""
    a = _View(A, beta, conj)
    s = _make_scalar(alpha, a.t.type)
    lib.tblis_tensor_shift(None, None, ctypes.byref(s), a.ref, _labels(idx_A))
    _check()


lib.tblis_b200_shard_plan.restype = ctypes.c_int
lib.tblis_b200_tensor_mult_shard.restype = ctypes.c_int


def shard_plan(A, idx_A, B, idx_B, C, idx_C, nranks, rank):
    """(label, begin, end) of rank's slab of C when the contraction is split
    over nranks processes (label '' when there is nothing to cut: rank 0 then
    owns all of C). Host-only: needs no GPU."""
    a, b, c = _View(A), _View(B), _View(C)
    lab = ctypes.c_char()
    beg, end = ctypes.c_ssize_t(), ctypes.c_ssize_t()
    lib.tblis_b200_shard_plan(a.ref, _labels(idx_A), b.ref, _labels(idx_B), c.ref, _labels(idx_C),
                              int(nranks), int(rank), ctypes.byref(lab), ctypes.byref(beg), ctypes.byref(end))
    _check()
    label = lab.value.decode() if lab.value != b"\x00" else ""
    return label, beg.value, end.value


def _rank_world(rank, nranks, group):
    if rank is None or nranks is None:
        import torch.distributed as dist
        return dist.get_rank(group), dist.get_world_size(group)
    return rank, nranks


def mult_shard(alpha, A, idx_A, B, idx_B, beta, C, idx_C, rank=None, nranks=None, gather=False, group=None,
               cfg=None):
    """This rank's slab of C = alpha*A*B + beta*C (tblis_b200_tensor_mult_shard);
    rank / nranks default to the torch.distributed group's. gather=True then
    hands every slab to every rank (gather_shards), so each holds all of C."""
    rank, nranks = _rank_world(rank, nranks, group)
    a, b, c = _View(A, alpha), _View(B), _View(C, beta)
    r = tblis_b200_report()
    lib.tblis_b200_tensor_mult_shard(cfg, a.ref, _labels(idx_A), b.ref, _labels(idx_B), c.ref, _labels(idx_C),
                                     int(nranks), int(rank), ctypes.byref(r))
    _check()
    if gather:
        gather_shards(A, idx_A, B, idx_B, C, idx_C, rank, nranks, group)
    return {f: getattr(r, f) for f, _ in tblis_b200_report._fields_}


def _slab(C, idx_C, label, begin, end):
    """The view of torch tensor C restricted to label in [begin, end)."""
    dims = [d for d, c in enumerate(idx_C) if c == label]
    if len(dims) != 1:
        raise ValueError("gather_shards: the cut label must appear once in C")
    return C.narrow(dims[0], begin, end - begin)


def gather_shards(A, idx_A, B, idx_B, C, idx_C, rank=None, nranks=None, group=None):
    """Every rank broadcasts its slab of C (torch tensor, same shape on every
    rank) in rank order; afterwards all ranks hold the whole C. Over NCCL on
    GPUs, gloo on CPU tensors."""
    import torch.distributed as dist
    rank, nranks = _rank_world(rank, nranks, group)
    for r in range(nranks):
        label, b, e = shard_plan(A, idx_A, B, idx_B, C, idx_C, nranks, r)
        view = C if not label else _slab(C, idx_C, label, b, e)
        if view.numel() == 0:
            continue
        buf = view.contiguous() if r == rank else view.new_empty(view.shape).contiguous()
        dist.broadcast(buf, src=dist.get_global_rank(group, r) if group is not None else r, group=group)
        if r != rank:
            view.copy_(buf)


def _make_scalar(v, code):
    s = tblis_scalar()
    s.type = code
    if code == TYPE_DOUBLE:
        s.data[0] = float(v)
    elif code == TYPE_DCOMPLEX:
        s.data[0] = complex(v).real
        s.data[1] = complex(v).imag
    else:
        f = ctypes.cast(ctypes.byref(s), _P(ctypes.c_float))
        if code == TYPE_SCOMPLEX:
            f[0] = complex(v).real
            f[1] = complex(v).imag
        else:
            f[0] = float(v)
    return s


def _scalar_value(s, code):
    f = ctypes.cast(ctypes.byref(s), _P(ctypes.c_float))
    if code == TYPE_DOUBLE:
        return s.data[0]
    if code == TYPE_DCOMPLEX:
        return complex(s.data[0], s.data[1])
    if code == TYPE_SCOMPLEX:
        return complex(f[0], f[1])
    return f[0]


def kernel_count():
    """Kernels this library launched in this process."""
    return lib.tblis_b200_kernel_count()


def kernel_timer(enable):
    """Start (True) or stop (False) per-launch device timing of the contraction
    and transpose kernels; either call clears the records."""
    lib.tblis_b200_kernel_timer(1 if enable else 0)


def kernel_time(kernel):
    """(total device ms, launches) of one kernel name since kernel_timer(True)."""
    ms, n = ctypes.c_double(0), ctypes.c_int64(0)
    if lib.tblis_b200_kernel_timer_read(kernel.encode(), ctypes.byref(ms), ctypes.byref(n)):
        _check()
    return ms.value, n.value


def set_stream(stream_handle):
    """Make the library enqueue on a cudaStream_t (int handle); 0 = default stream."""
    lib.tblis_b200_set_stream(ctypes.c_void_p(stream_handle))


def synchronize():
    lib.tblis_b200_synchronize()
    _check()


# ---- DPD tensors and batches ---------------------------------------------------------------

class tblis_b200_dpd_tensor(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("conj", ctypes.c_int), ("scalar", tblis_scalar),
                ("data", ctypes.c_void_p), ("ndim", ctypes.c_uint), ("nirrep", ctypes.c_uint),
                ("irrep", ctypes.c_uint), ("len", ctypes.POINTER(ctypes.c_ssize_t)), ("layout", ctypes.c_int)]


lib.tblis_b200_dpd_mult.argtypes = [_P(tblis_b200_dpd_tensor), ctypes.c_char_p, _P(tblis_b200_dpd_tensor),
                                    ctypes.c_char_p, _P(tblis_b200_dpd_tensor), ctypes.c_char_p,
                                    _P(tblis_b200_report)]
lib.tblis_b200_dpd_mult.restype = ctypes.c_int
lib.tblis_b200_dpd_block.argtypes = [_P(tblis_b200_dpd_tensor), _P(ctypes.c_uint), _P(ctypes.c_ssize_t),
                                     _P(ctypes.c_ssize_t), _P(ctypes.c_ssize_t)]
lib.tblis_b200_dpd_block.restype = ctypes.c_int
lib.tblis_b200_dpd_size.argtypes = [_P(tblis_b200_dpd_tensor)]
lib.tblis_b200_dpd_size.restype = ctypes.c_ssize_t
lib.tblis_b200_tensor_mult_batch.restype = ctypes.c_int


class DpdTensor:
    """A DPD tensor (MArray dpd_varray layout) over a flat torch/numpy buffer.

    lens: [ndim][nirrep] lengths per irrep; irrep: the tensor's irrep;
    layout: MArray dpd_layout type (default 5 = PREFIX_ROW_MAJOR)."""

    def __init__(self, irrep, nirrep, lens, data=None, layout=5):
        self.irrep, self.nirrep, self.layout = int(irrep), int(nirrep), int(layout)
        self.lens = [list(map(int, r)) for r in lens]
        self.data = data
        # element type from the buffer (float32 / float64 / complex64 / complex128)
        self.code = _dtype_code(data)[0] if data is not None else TYPE_DOUBLE
        self._len = (ctypes.c_ssize_t * (len(self.lens) * self.nirrep))(*[x for r in self.lens for x in r])

    def struct(self, scalar=1.0):
        t = tblis_b200_dpd_tensor()
        t.type = self.code
        t.conj = 0
        t.scalar = _make_scalar(scalar, self.code)
        if self.data is None:
            t.data = None
        elif hasattr(self.data, "data_ptr"):
            t.data = self.data.data_ptr()
        else:
            t.data = self.data.ctypes.data
        t.ndim = len(self.lens)
        t.nirrep = self.nirrep
        t.irrep = self.irrep
        t.len = ctypes.cast(self._len, _P(ctypes.c_ssize_t))
        t.layout = self.layout
        return t

    def size(self):
        t = self.struct()
        n = lib.tblis_b200_dpd_size(ctypes.byref(t))
        _check()
        return n

    def block(self, irreps):
        """(offset, lengths, strides) of one block, as dpd_varray_view(irreps)."""
        t = self.struct()
        n = len(self.lens)
        irr = (ctypes.c_uint * n)(*irreps)
        L = (ctypes.c_ssize_t * n)()
        S = (ctypes.c_ssize_t * n)()
        off = ctypes.c_ssize_t()
        lib.tblis_b200_dpd_block(ctypes.byref(t), irr, L, S, ctypes.byref(off))
        _check()
        return off.value, list(L), list(S)


def dpd_mult(alpha, A, idx_A, B, idx_B, beta, C, idx_C):
    """C = alpha*A*B + beta*C over DPD tensors (src/iface/3t/mult.h:59-72)."""
    a, b, c = A.struct(alpha), B.struct(), C.struct(beta)
    r = tblis_b200_report()
    lib.tblis_b200_dpd_mult(ctypes.byref(a), _labels(idx_A), ctypes.byref(b), _labels(idx_B), ctypes.byref(c),
                            _labels(idx_C), ctypes.byref(r))
    _check()
    return {f: getattr(r, f) for f, _ in tblis_b200_report._fields_}


lib.tblis_b200_dpd_shard_plan.restype = ctypes.c_int
lib.tblis_b200_dpd_mult_shard.restype = ctypes.c_int


def dpd_shard_plan(A, idx_A, B, idx_B, C, idx_C, nranks):
    """(owner, flops): the rank that computes each C block of a DPD
    contraction split over nranks processes, keyed by the block's irrep
    tuple, and each rank's FLOPs (tblis_b200_dpd_shard_plan; host-only: needs
    no GPU). Units of work are the irrep GEMMs (irrep of the contracted
    labels), placed longest first onto the least loaded rank."""
    import itertools
    a, b, c = A.struct(), B.struct(), C.struct()
    n, nd = C.nirrep, len(C.lens)
    owner = (ctypes.c_int * (n ** nd))()
    flops = (ctypes.c_double * int(nranks))()
    lib.tblis_b200_dpd_shard_plan(ctypes.byref(a), _labels(idx_A), ctypes.byref(b), _labels(idx_B), ctypes.byref(c),
                                  _labels(idx_C), int(nranks), owner, flops)
    _check()
    out = {}
    for t in itertools.product(range(n), repeat=nd):
        k = sum(t[d] * n ** d for d in range(nd))
        if owner[k] >= 0:
            out[t] = owner[k]
    return out, list(flops)


def dpd_mult_shard(alpha, A, idx_A, B, idx_B, beta, C, idx_C, rank=None, nranks=None, gather=False, group=None):
    """This rank's blocks of C = alpha*A*B + beta*C over DPD tensors
    (tblis_b200_dpd_mult_shard); the others stay as they are. rank / nranks
    default to the torch.distributed group's; gather=True then hands every
    rank's blocks to every rank (dpd_gather_shards)."""
    rank, nranks = _rank_world(rank, nranks, group)
    a, b, c = A.struct(alpha), B.struct(), C.struct(beta)
    r = tblis_b200_report()
    lib.tblis_b200_dpd_mult_shard(ctypes.byref(a), _labels(idx_A), ctypes.byref(b), _labels(idx_B), ctypes.byref(c),
                                  _labels(idx_C), int(nranks), int(rank), ctypes.byref(r))
    _check()
    if gather:
        dpd_gather_shards(A, idx_A, B, idx_B, C, idx_C, rank, nranks, group)
    return {f: getattr(r, f) for f, _ in tblis_b200_report._fields_}


def dpd_gather_shards(A, idx_A, B, idx_B, C, idx_C, rank=None, nranks=None, group=None):
    """Every rank broadcasts the elements of its blocks of C (C.data: a flat
    torch tensor of the same layout on every rank) in rank order; afterwards
    all ranks hold the whole C. Over NCCL on GPUs, gloo on CPU tensors."""
    import numpy as np
    import torch
    import torch.distributed as dist
    rank, nranks = _rank_world(rank, nranks, group)
    owner, _ = dpd_shard_plan(A, idx_A, B, idx_B, C, idx_C, nranks)
    per_rank = [[] for _ in range(nranks)]
    for t, r in owner.items():
        off, L, S = C.block(t)
        if np.prod(L) == 0:
            continue
        grid = np.indices(L).reshape(len(L), -1)
        per_rank[r].append(off + (np.asarray(S)[:, None] * grid).sum(0))
    flat = C.data.view(-1)
    for r in range(nranks):
        if not per_rank[r]:
            continue
        idx = torch.from_numpy(np.concatenate(per_rank[r]).astype(np.int64)).to(flat.device)
        buf = flat.index_select(0, idx) if r == rank else flat.new_empty(idx.numel())
        dist.broadcast(buf, src=dist.get_global_rank(group, r) if group is not None else r, group=group)
        if r != rank:
            flat.index_copy_(0, idx, buf)


class tblis_b200_dpd_block_table(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("conj", ctypes.c_int), ("scalar", tblis_scalar),
                ("data", ctypes.c_void_p), ("ndim", ctypes.c_uint), ("nirrep", ctypes.c_uint),
                ("irrep", ctypes.c_uint), ("len", _P(ctypes.c_ssize_t)), ("offset", _P(ctypes.c_ssize_t)),
                ("stride", _P(ctypes.c_ssize_t))]


_DT = _P(tblis_b200_dpd_block_table)
lib.tblis_b200_dpd_add.argtypes = [_DT, ctypes.c_char_p, _DT, ctypes.c_char_p]
lib.tblis_b200_dpd_dot.argtypes = [_DT, ctypes.c_char_p, _DT, ctypes.c_char_p, _P(tblis_scalar)]
lib.tblis_b200_dpd_reduce.argtypes = [ctypes.c_int, _DT, ctypes.c_char_p, _P(tblis_scalar),
                                      _P(ctypes.c_ssize_t)]
lib.tblis_b200_dpd_scale.argtypes = [_DT, ctypes.c_char_p]
lib.tblis_b200_dpd_set.argtypes = [_P(tblis_scalar), _DT, ctypes.c_char_p]
lib.tblis_b200_dpd_shift.argtypes = [_P(tblis_scalar), _DT, ctypes.c_char_p]
lib.tblis_b200_dpd_block_to_full.argtypes = [_DT, _P(tblis_tensor)]
lib.tblis_b200_dpd_full_to_block.argtypes = [_P(tblis_tensor), _DT]


def _dpd_table(T, scalar=1.0):
    """The block table of a DpdTensor (every stored block's offset and
    strides, irrep tuples numbered with dimension 0 fastest)."""
    nd, n = len(T.lens), T.nirrep
    nt = n ** nd
    off = [-1] * nt
    st = [0] * (nt * nd)
    for t in range(nt):
        irr = [(t // n ** d) % n for d in range(nd)]
        x = 0
        ext = 1
        for d in range(nd):
            x ^= irr[d]
            ext *= T.lens[d][irr[d]]
        if x != T.irrep or ext == 0:
            continue
        o, _, strides = T.block(irr)
        off[t] = o
        st[t * nd:(t + 1) * nd] = strides
    keep = [(ctypes.c_ssize_t * (nd * n))(*[x for r in T.lens for x in r]), (ctypes.c_ssize_t * nt)(*off),
            (ctypes.c_ssize_t * max(1, len(st)))(*st)]
    b = tblis_b200_dpd_block_table()
    b.type = T.code
    b.conj = 0
    b.scalar = _make_scalar(scalar, T.code)
    b.data = T.data.data_ptr() if hasattr(T.data, "data_ptr") else T.data.ctypes.data
    b.ndim, b.nirrep, b.irrep = nd, n, T.irrep
    b.len = ctypes.cast(keep[0], _P(ctypes.c_ssize_t))
    b.offset = ctypes.cast(keep[1], _P(ctypes.c_ssize_t))
    b.stride = ctypes.cast(keep[2], _P(ctypes.c_ssize_t))
    return b, keep


def dpd_block_to_full(A, F):
    """F = the dense form of the DPD tensor A (block_to_full,
    src/internal/1t/dpd/util.hpp:70-102): F's length in dimension d is the
    sum of A's lengths over the irreps; F is zeroed, then each stored block of
    A is copied into its region (irrep x after the irreps below it)."""
    a, ka = _dpd_table(A)
    f = _View(F)
    lib.tblis_b200_dpd_block_to_full(ctypes.byref(a), f.ref)
    _check()


def dpd_full_to_block(F, A):
    """Every stored block of the DPD tensor A gets its region of the dense
    tensor F (full_to_block, src/internal/1t/dpd/util.hpp:104-133)."""
    a, ka = _dpd_table(A)
    f = _View(F)
    lib.tblis_b200_dpd_full_to_block(f.ref, ctypes.byref(a))
    _check()


def dpd_add(alpha, A, idx_A, beta, B, idx_B):
    """B = alpha*A + beta*B over DPD tensors (tblis::add over dpd_varray_view)."""
    a, ka = _dpd_table(A, alpha)
    b, kb = _dpd_table(B, beta)
    lib.tblis_b200_dpd_add(ctypes.byref(a), _labels(idx_A), ctypes.byref(b), _labels(idx_B))
    _check()


def dpd_dot(A, idx_A, B, idx_B):
    a, ka = _dpd_table(A)
    b, kb = _dpd_table(B)
    r = tblis_scalar()
    lib.tblis_b200_dpd_dot(ctypes.byref(a), _labels(idx_A), ctypes.byref(b), _labels(idx_B), ctypes.byref(r))
    _check()
    return _scalar_value(r, A.code)


def dpd_reduce(op, A, idx_A):
    """(value, offset from the data) of a reduction over the stored elements."""
    a, ka = _dpd_table(A)
    r = tblis_scalar()
    i = ctypes.c_ssize_t(-1)
    lib.tblis_b200_dpd_reduce(int(op), ctypes.byref(a), _labels(idx_A), ctypes.byref(r), ctypes.byref(i))
    _check()
    return _scalar_value(r, A.code), i.value


def dpd_scale(alpha, A, idx_A):
    a, ka = _dpd_table(A, alpha)
    lib.tblis_b200_dpd_scale(ctypes.byref(a), _labels(idx_A))
    _check()


def dpd_set(alpha, A, idx_A):
    a, ka = _dpd_table(A)
    s = _make_scalar(alpha, A.code)
    lib.tblis_b200_dpd_set(ctypes.byref(s), ctypes.byref(a), _labels(idx_A))
    _check()


def dpd_shift(alpha, beta, A, idx_A):
    """A = alpha + beta*A over the stored elements."""
    a, ka = _dpd_table(A, beta)
    s = _make_scalar(alpha, A.code)
    lib.tblis_b200_dpd_shift(ctypes.byref(s), ctypes.byref(a), _labels(idx_A))
    _check()


class tblis_b200_indexed_dpd_tensor(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("scalar", tblis_scalar), ("ndim", ctypes.c_uint),
                ("dense_ndim", ctypes.c_uint), ("nirrep", ctypes.c_uint), ("dense_irrep", ctypes.c_uint),
                ("len", _P(ctypes.c_ssize_t)), ("idx_irrep", _P(ctypes.c_uint)), ("nidx", ctypes.c_ssize_t),
                ("indices", _P(ctypes.c_ssize_t)), ("data", _P(ctypes.c_void_p)), ("factor", ctypes.c_void_p),
                ("offset", _P(ctypes.c_ssize_t)), ("stride", _P(ctypes.c_ssize_t))]


lib.tblis_b200_indexed_dpd_mult.argtypes = [_P(tblis_b200_indexed_dpd_tensor), ctypes.c_char_p,
                                            _P(tblis_b200_indexed_dpd_tensor), ctypes.c_char_p,
                                            _P(tblis_b200_indexed_dpd_tensor), ctypes.c_char_p,
                                            _P(tblis_b200_report)]
lib.tblis_b200_indexed_dpd_mult.restype = ctypes.c_int


class IndexedDpdTensor:
    """An indexed DPD tensor as MArray's indexed_dpd_varray holds it: the
    first ndim - len(idx_irreps) dimensions are dense DPD dimensions, the
    others are indexed with fixed irreps; `indices` lists the index tuples of
    the stored entries, `data` holds their dense storage back to back (entry
    size = dense_size(), MArray layout `layout`), `factors` their scalars.

    irrep: the overall irrep (dense irrep XOR the indexed irreps), as
    indexed_dpd_varray(irrep, nirrep, len, idx_irrep, idx) takes it."""

    def __init__(self, irrep, nirrep, lens, idx_irreps, indices, data=None, factors=None, layout=5):
        self.nirrep = int(nirrep)
        self.lens = [list(map(int, r)) for r in lens]
        self.idx_irreps = [int(x) for x in idx_irreps]
        self.ndim = len(self.lens)
        self.dense_ndim = self.ndim - len(self.idx_irreps)
        self.irrep = int(irrep)
        self.dense_irrep = self.irrep
        for r in self.idx_irreps:
            self.dense_irrep ^= r
        self.indices = [list(map(int, t)) for t in indices] if self.idx_irreps else [[]]
        self.nidx = max(1, len(self.indices))
        self.factors = [1.0] * self.nidx if factors is None else [complex(f) for f in factors]
        self.layout = int(layout)
        self.data = data
        # element type from the buffer (float32 / float64 / complex64 / complex128)
        self.code, self.esize = _dtype_code(data) if data is not None else (TYPE_DOUBLE, 8)
        dense = DpdTensor(self.dense_irrep, self.nirrep, self.lens[:self.dense_ndim], layout=self.layout)
        self._dense_size = dense.size()
        # block table of one entry: every irrep tuple of the dense dims, dim 0 fastest
        nt = self.nirrep ** self.dense_ndim
        off = [-1] * nt
        strides = [0] * (nt * self.dense_ndim)
        for t in range(nt):
            irr = [(t // self.nirrep ** d) % self.nirrep for d in range(self.dense_ndim)]
            x = 0
            for r in irr:
                x ^= r
            ext = 1
            for d in range(self.dense_ndim):
                ext *= self.lens[d][irr[d]]
            if x != self.dense_irrep or ext == 0:
                continue
            o, _, st = dense.block(irr)
            off[t] = o
            strides[t * self.dense_ndim:(t + 1) * self.dense_ndim] = st
        self._len = (ctypes.c_ssize_t * (self.ndim * self.nirrep))(*[x for r in self.lens for x in r])
        self._irr = (ctypes.c_uint * max(1, len(self.idx_irreps)))(*self.idx_irreps)
        flat_idx = [x for t in self.indices for x in t]
        self._idx = (ctypes.c_ssize_t * max(1, len(flat_idx)))(*flat_idx)
        self._off = (ctypes.c_ssize_t * nt)(*off)
        self._str = (ctypes.c_ssize_t * max(1, len(strides)))(*strides)

    def dense_size(self):
        """Stored elements of one entry."""
        return self._dense_size

    def struct(self, scalar=1.0):
        t = tblis_b200_indexed_dpd_tensor()
        t.type = self.code
        t.scalar = _make_scalar(scalar, self.code)
        t.ndim, t.dense_ndim, t.nirrep, t.dense_irrep = self.ndim, self.dense_ndim, self.nirrep, self.dense_irrep
        t.len = ctypes.cast(self._len, _P(ctypes.c_ssize_t))
        t.idx_irrep = ctypes.cast(self._irr, _P(ctypes.c_uint))
        t.nidx = self.nidx
        t.indices = ctypes.cast(self._idx, _P(ctypes.c_ssize_t))
        base = self.data.data_ptr() if hasattr(self.data, "data_ptr") else self.data.ctypes.data
        self._ptrs = (ctypes.c_void_p * self.nidx)(*[base + self.esize * e * self._dense_size
                                                     for e in range(self.nidx)])
        t.data = ctypes.cast(self._ptrs, _P(ctypes.c_void_p))
        # the factors as elements of the tensor's type
        if self.code == TYPE_DOUBLE:
            self._fac = (ctypes.c_double * self.nidx)(*[f.real for f in self.factors])
        elif self.code == TYPE_FLOAT:
            self._fac = (ctypes.c_float * self.nidx)(*[f.real for f in self.factors])
        else:
            part = ctypes.c_double if self.code == TYPE_DCOMPLEX else ctypes.c_float
            self._fac = (part * (2 * self.nidx))(*[x for f in self.factors for x in (f.real, f.imag)])
        t.factor = ctypes.cast(self._fac, ctypes.c_void_p)
        t.offset = ctypes.cast(self._off, _P(ctypes.c_ssize_t))
        t.stride = ctypes.cast(self._str, _P(ctypes.c_ssize_t))
        return t


_IT = _P(tblis_b200_indexed_dpd_tensor)
lib.tblis_b200_indexed_dpd_add.argtypes = [_IT, ctypes.c_char_p, _IT, ctypes.c_char_p]
lib.tblis_b200_indexed_dpd_dot.argtypes = [_IT, ctypes.c_char_p, _IT, ctypes.c_char_p, _P(tblis_scalar)]
lib.tblis_b200_indexed_dpd_reduce.argtypes = [ctypes.c_int, _IT, ctypes.c_char_p, _P(tblis_scalar),
                                              _P(ctypes.c_ssize_t)]
lib.tblis_b200_indexed_dpd_scale.argtypes = [_IT, ctypes.c_char_p]
lib.tblis_b200_indexed_dpd_set.argtypes = [_P(tblis_scalar), _IT, ctypes.c_char_p]
lib.tblis_b200_indexed_dpd_shift.argtypes = [_P(tblis_scalar), _IT, ctypes.c_char_p]




def indexed_dpd_add(alpha, A, idx_A, beta, B, idx_B):
    """B = alpha*A + beta*B over indexed DPD tensors (tblis::add over indexed_dpd_varray_view)."""
    a, b = A.struct(alpha), B.struct(beta)
    lib.tblis_b200_indexed_dpd_add(ctypes.byref(a), _labels(idx_A), ctypes.byref(b), _labels(idx_B))
    _check()


def indexed_dpd_dot(A, idx_A, B, idx_B):
    a, b = A.struct(), B.struct()
    r = tblis_scalar()
    lib.tblis_b200_indexed_dpd_dot(ctypes.byref(a), _labels(idx_A), ctypes.byref(b), _labels(idx_B),
                                   ctypes.byref(r))
    _check()
    return _scalar_value(r, A.code)


def indexed_dpd_reduce(op, A, idx_A):
    a = A.struct()
    r = tblis_scalar()
    i = ctypes.c_ssize_t(-1)
    lib.tblis_b200_indexed_dpd_reduce(int(op), ctypes.byref(a), _labels(idx_A), ctypes.byref(r), ctypes.byref(i))
    _check()
    return _scalar_value(r, A.code), i.value


def indexed_dpd_scale(alpha, A, idx_A):
    a = A.struct(alpha)
    lib.tblis_b200_indexed_dpd_scale(ctypes.byref(a), _labels(idx_A))
    _check()


def indexed_dpd_set(alpha, A, idx_A):
    a = A.struct()
    s = _make_scalar(alpha, A.code)
    lib.tblis_b200_indexed_dpd_set(ctypes.byref(s), ctypes.byref(a), _labels(idx_A))
    _check()


def indexed_dpd_shift(alpha, beta, A, idx_A):
    a = A.struct(beta)
    s = _make_scalar(alpha, A.code)
    lib.tblis_b200_indexed_dpd_shift(ctypes.byref(s), ctypes.byref(a), _labels(idx_A))
    _check()


def indexed_dpd_mult(alpha, A, idx_A, B, idx_B, beta, C, idx_C):
    """C = alpha*A*B + beta*C over indexed DPD tensors (src/iface/3t/mult.h:92-110)."""
    a, b, c = A.struct(alpha), B.struct(), C.struct(beta)
    r = tblis_b200_report()
    lib.tblis_b200_indexed_dpd_mult(ctypes.byref(a), _labels(idx_A), ctypes.byref(b), _labels(idx_B),
                                    ctypes.byref(c), _labels(idx_C), ctypes.byref(r))
    _check()
    return {f: getattr(r, f) for f, _ in tblis_b200_report._fields_}


class PreparedBatch:
    """The C-ABI arrays of a batch built once, so repeated runs of the same
    tensors (an iterative solver's step) cost one library call."""

    def __init__(self, items):
        n = len(items)
        self.views = []
        self.TA = (tblis_tensor * n)()
        self.TB = (tblis_tensor * n)()
        self.TC = (tblis_tensor * n)()
        self.IA = (ctypes.c_char_p * n)()
        self.IB = (ctypes.c_char_p * n)()
        self.IC = (ctypes.c_char_p * n)()
        for i, (alpha, A, ia, B, ib, beta, C, ic) in enumerate(items):
            va, vb, vc = _View(A, alpha), _View(B), _View(C, beta)
            self.views.append((va, vb, vc))
            self.TA[i], self.TB[i], self.TC[i] = va.t, vb.t, vc.t
            self.IA[i], self.IB[i], self.IC[i] = _labels(ia), _labels(ib), _labels(ic)
        self.betas = [float(it[5]) for it in items]
        self.n = n

    def run(self):
        # the library resets C's scalar after each call: restore beta
        for i, b in enumerate(self.betas):
            self.TC[i].scalar.data[0] = b
        r = tblis_b200_report()
        lib.tblis_b200_tensor_mult_batch(self.n, self.TA, self.IA, self.TB, self.IB, self.TC, self.IC,
                                         ctypes.byref(r))
        _check()
        return {f: getattr(r, f) for f, _ in tblis_b200_report._fields_}


def mult_batch(items):
    """items: list of (alpha, A, idx_A, B, idx_B, beta, C, idx_C) with device
    tensors; all run in one grouped launch."""
    return PreparedBatch(items).run()


def _mult_batch_unprepared(items):
    n = len(items)
    views = []
    TA = (tblis_tensor * n)()
    TB = (tblis_tensor * n)()
    TC = (tblis_tensor * n)()
    IA = (ctypes.c_char_p * n)()
    IB = (ctypes.c_char_p * n)()
    IC = (ctypes.c_char_p * n)()
    for i, (alpha, A, ia, B, ib, beta, C, ic) in enumerate(items):
        va, vb, vc = _View(A, alpha), _View(B), _View(C, beta)
        views.append((va, vb, vc))
        TA[i], TB[i], TC[i] = va.t, vb.t, vc.t
        IA[i], IB[i], IC[i] = _labels(ia), _labels(ib), _labels(ic)
    r = tblis_b200_report()
    lib.tblis_b200_tensor_mult_batch(n, TA, IA, TB, IB, TC, IC, ctypes.byref(r))
    _check()
    return {f: getattr(r, f) for f, _ in tblis_b200_report._fields_}


# ---- serving -----------------------------------------------------------------------------------

class tblis_b200_server_stats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_int64), ("failed", ctypes.c_int64), ("batches", ctypes.c_int64),
                ("queued", ctypes.c_int64), ("mean_batch", ctypes.c_double),
                ("max_concurrent_batches", ctypes.c_int), ("p50_ms", ctypes.c_double),
                ("p99_ms", ctypes.c_double), ("max_ms", ctypes.c_double), ("ozaki", ctypes.c_int64),
                ("shape_hits", ctypes.c_int64), ("shape_misses", ctypes.c_int64)]


lib.tblis_b200_server_create.argtypes = [ctypes.c_size_t, ctypes.c_int]
lib.tblis_b200_server_create.restype = ctypes.c_void_p
lib.tblis_b200_server_destroy.argtypes = [ctypes.c_void_p]
lib.tblis_b200_server_submit.argtypes = [ctypes.c_void_p, _P(tblis_tensor), ctypes.c_char_p, _P(tblis_tensor),
                                         ctypes.c_char_p, _P(tblis_tensor), ctypes.c_char_p, ctypes.c_double]
lib.tblis_b200_server_submit.restype = ctypes.c_int64
lib.tblis_b200_server_poll.argtypes = [ctypes.c_void_p, ctypes.c_int64, _P(ctypes.c_double)]
lib.tblis_b200_server_wait.argtypes = [ctypes.c_void_p, ctypes.c_int64, _P(ctypes.c_double)]
lib.tblis_b200_server_get_stats.argtypes = [ctypes.c_void_p, _P(tblis_b200_server_stats)]


class Server:
    """Continuous-batching contraction server over device-resident operands
    (see tblis_b200_server_* in include/tblis_b200.h)."""

    def __init__(self, hbm_budget_bytes=150 << 30, slots=4):
        self.h = lib.tblis_b200_server_create(int(hbm_budget_bytes), int(slots))
        _check()
        if not self.h:
            raise TblisError(3, "server creation failed")
        self._live = {}

    def submit(self, alpha, A, idx_A, B, idx_B, beta, C, idx_C, tolerance=1e-13):
        a, b, c = _View(A, alpha), _View(B), _View(C, beta)
        rid = lib.tblis_b200_server_submit(self.h, a.ref, _labels(idx_A), b.ref, _labels(idx_B), c.ref,
                                           _labels(idx_C), float(tolerance))
        if rid < 0:
            _check()
            raise TblisError(1, "submit failed")
        self._live[rid] = (a, b, c)
        return rid

    def wait(self, rid):
        lat = ctypes.c_double(0)
        rc = lib.tblis_b200_server_wait(self.h, rid, ctypes.byref(lat))
        self._live.pop(rid, None)
        if rc:
            _check()
            raise TblisError(rc, "request failed")
        return lat.value

    def poll(self, rid):
        lat = ctypes.c_double(0)
        rc = lib.tblis_b200_server_poll(self.h, rid, ctypes.byref(lat))
        if rc == 1:
            return False, None
        self._live.pop(rid, None)
        if rc:
            _check()
            raise TblisError(rc, "request failed")
        return True, lat.value

    def stats(self):
        s = tblis_b200_server_stats()
        lib.tblis_b200_server_get_stats(self.h, ctypes.byref(s))
        _check()
        return {f: getattr(s, f) for f, _ in tblis_b200_server_stats._fields_}

    def close(self):
        if self.h:
            lib.tblis_b200_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
