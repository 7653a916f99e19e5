"""Shapes of the learned proposal: the coupling masks and the flat parameter
layout of libchili_b200 (include/chili_gpu.h, "learned proposal"), mirrored
on the host so that parameters can be moved between the library and Python
(checkpoints, tests)."""
import numpy as np

HIDDEN = 128
BINS = 16
PER_DIM = 3 * BINS + 1
ALPHA_HIDDEN = 64


def masks(dims, layers):
    """True = conditioning dimension of layer l; every layer transforms at
    most 5 dimensions."""
    idx = np.arange(dims)
    out = []
    if dims <= 10:
        pats = [idx % 2 == 0, idx % 2 == 1, idx < dims // 2, idx >= dims // 2,
                ((idx + 1) // 2) % 2 == 0, ((idx + 1) // 2) % 2 == 1]
        for l in range(layers):
            m = pats[l % 6]
            if m.all() or not m.any():
                m = idx % 2 == (l % 2)
            out.append(m)
    else:
        for l in range(layers):
            m = np.ones(dims, dtype=bool)
            m[(5 * l + np.arange(5)) % dims] = False
            out.append(m)
    return out


def n_features(n_ext):
    n_out = n_ext - 2
    return n_out * (n_out - 1) // 2 + n_out


def w2_name(l, k):
    """The k-th square hidden matrix of coupling layer l."""
    return f"W2_{l}" if k == 0 else f"W2_{l}_{k}"


def layout(dims, nch, n_ext, layers=6, hidden=HIDDEN, depth=2):
    """[(name, offset, shape)] in the library's order: per coupling layer
    W1 [hidden][da], E [nch][hidden], depth - 1 square matrices
    [hidden][hidden], W3 [db*49][hidden]; then the channel-weight network."""
    out, off = [], 0
    H = hidden
    for l, m in enumerate(masks(dims, layers)):
        da, db = int(m.sum()), int((~m).sum())
        items = [(f"W1_{l}", (H, da)), (f"E_{l}", (nch, H))]
        items += [(w2_name(l, k), (H, H)) for k in range(depth - 1)]
        items.append((f"W3_{l}", (db * PER_DIM, H)))
        for name, shape in items:
            out.append((name, off, shape))
            off += int(np.prod(shape))
    F, A = n_features(n_ext), ALPHA_HIDDEN
    for name, shape in (("A1", (A, F)), ("c1", (A,)), ("A2", (A, A)), ("c2", (A,)), ("A3", (nch, A)), ("c3", (nch,))):
        out.append((name, off, shape))
        off += int(np.prod(shape))
    return out


def unflatten(flat, lay):
    return {name: np.asarray(flat[off:off + int(np.prod(shape))], dtype=np.float64).reshape(shape)
            for name, off, shape in lay}


def flatten(params, lay):
    n = lay[-1][1] + int(np.prod(lay[-1][2]))
    out = np.zeros(n, dtype=np.float32)
    for name, off, shape in lay:
        out[off:off + int(np.prod(shape))] = np.asarray(params[name], dtype=np.float32).reshape(-1)
    return out
