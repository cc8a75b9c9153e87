"""Seeded random strided tensors and contractions for the parity tests.

Mirrors the style of the reference's randomized tests (test/test.hpp:401-443,
test/test.cxx:716-1333): random labels split into AB/AC/BC/ABC groups, random
lengths, every operand stored in a random dimension order with optional
padding, values uniform(-1, 1).
"""
import numpy as np

LABELS = "abcdefghijklmnopqrstuvwxyz"


def strided_empty(shape, order=None, pad=0, rng=None, dtype=np.float64):
    """A numpy array view of `shape` whose storage is ordered by `order`
    (order[0] fastest) with `pad` extra elements per dimension."""
    n = len(shape)
    if order is None:
        order = list(range(n))
    strides = [0] * n
    s = 1
    for d in order:
        strides[d] = s
        s *= shape[d] + (pad if shape[d] > 1 else 0)
    size = max(s, 1)
    base = np.zeros(size, dtype=dtype)
    view = np.lib.stride_tricks.as_strided(base, shape=tuple(shape),
                                           strides=tuple(x * base.itemsize for x in strides))
    return base, view, strides


def random_tensor(shape, rng, order=None, pad=0, fill=True):
    base, view, strides = strided_empty(shape, order, pad, rng)
    if fill:
        base[:] = rng.uniform(-1.0, 1.0, base.size)
    return base, view, strides


def random_contraction(rng, max_len=7, max_labels=(3, 3, 3, 2), pad_prob=0.3):
    """Returns (idx_A, idx_B, idx_C, lens) for a random contraction."""
    counts = [int(rng.integers(0, m + 1)) for m in max_labels]
    while sum(counts[:3]) == 0:
        counts = [int(rng.integers(0, m + 1)) for m in max_labels]
    labs = list(LABELS)
    rng.shuffle(labs)
    groups = []
    p = 0
    for c in counts:
        groups.append(labs[p:p + c])
        p += c
    AB, AC, BC, ABC = groups
    lens = {l: int(rng.integers(1, max_len + 1)) for l in AB + AC + BC + ABC}
    idx_A = AB + AC + ABC
    idx_B = AB + BC + ABC
    idx_C = AC + BC + ABC
    for lst in (idx_A, idx_B, idx_C):
        rng.shuffle(lst)
    return "".join(idx_A), "".join(idx_B), "".join(idx_C), lens


def make_operand(idx, lens, rng, pad_prob=0.3):
    shape = [lens[c] for c in idx]
    order = list(rng.permutation(len(shape)))
    pad = int(rng.integers(1, 3)) if rng.random() < pad_prob else 0
    return random_tensor(shape, rng, order, pad)


def normwise_rel(x, ref):
    d = np.linalg.norm((np.asarray(x) - np.asarray(ref)).ravel())
    n = np.linalg.norm(np.asarray(ref).ravel())
    return d / n if n > 0 else d


def to_device(base, view, strides, torch, device):
    """A torch device tensor with the same storage layout as the numpy view."""
    tb = torch.from_numpy(base.copy()).to(device)
    return tb, torch.as_strided(tb, tuple(view.shape), tuple(strides))


def view_of(base_np, shape, strides):
    return np.lib.stride_tricks.as_strided(base_np, shape=tuple(shape),
                                           strides=tuple(s * base_np.itemsize for s in strides))
