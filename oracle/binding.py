"""Shared ctypes binding of the two CPU oracles:
  oracle/_ref/libchili_ref.so  the UNMODIFIED Chili reference (ref_driver.cc), prefix ref_
  oracle/libchili_oracle.so    the C restatement (port/chili_oracle.c),       prefix orc_
Both export the same entry points (the reference additionally its own
mt19937-driven loops, the port the Philox uniforms of the CUDA library).

TEST INFRASTRUCTURE ONLY (tests/, smoke(), bench.py's CPU legs).
"""
import ctypes as C
import os

import numpy as np

from chili_b200 import abi  # the shared ABI structs

HERE = os.path.dirname(os.path.abspath(__file__))


class OracleLib:
    def __init__(self, path, prefix):
        self.path = path
        self.prefix = prefix
        self._lib = None

    def available(self):
        return os.path.exists(self.path)

    def __call__(self):
        if self._lib is None:
            self._lib = _load(self.path, self.prefix)
        return self._lib


class _Prefixed:
    """Maps ref_xxx attribute names onto the library's own prefix."""

    def __init__(self, lib, prefix):
        self._l = lib
        self._p = prefix

    def __getattr__(self, name):
        return getattr(self._l, self._p + name[4:] if name.startswith("ref_") else name)


def _load(path, prefix):
    L = C.CDLL(path)
    vp, i32, i64, dbl, u32 = C.c_void_p, C.c_int, C.c_int64, C.c_double, C.c_uint
    P = C.POINTER
    sigs = {
        "ref_am_map": ([i32, i32, vp, vp, i64, vp, vp], None),
        "ref_am_weight": ([i32, i32, vp, vp, i64, vp, vp], None),
        "ref_am_adapt": ([i32, i32, vp, dbl, vp, vp], None),
        "ref_am_split": ([i32, i32, vp, i32, vp], None),
        "ref_vegas_iterate": ([i32, i32, vp, dbl, i32, vp, i32, i64, vp, P(abi.Stats), vp], None),
        "ref_vegas_run": ([i32, i32, dbl, vp, i32, u32, i64, i32, P(abi.Stats)], None),
        "ref_mc_create": ([P(abi.ChannelDesc), i32, P(abi.Cuts), dbl, i32, i32,
                           P(abi.MultiChannelParams)], vp),
        "ref_mc_destroy": ([vp], None),
        "ref_mc_ndims": ([vp], i32),
        "ref_mc_set_integrand": ([vp, i32, vp, i32, i32], None),
        "ref_mc_set_cuts": ([vp, dbl, dbl, dbl, dbl], None),
        "ref_mc_set_grids": ([vp, vp], None),
        "ref_mc_get_grids": ([vp, vp], None),
        "ref_mc_set_alpha": ([vp, vp], None),
        "ref_mc_get_alpha": ([vp, vp, vp, vp], None),
        "ref_fsm_generate": ([vp, i32, vp, i64, vp], None),
        "ref_fsm_weight": ([vp, i32, vp, i64, vp, vp], None),
        "ref_select": ([vp, i32, vp, i64, vp], None),
        "ref_mc_weight": ([vp, vp, vp, i64, vp, vp, vp], None),
        "ref_mc_iterate": ([vp, vp, i64, i32, P(abi.Stats), P(abi.MCIterInfo)], i32),
        "ref_mc_get_training": ([vp, vp, vp], None),
        "ref_mc_train": ([vp, vp, vp], None),
        "ref_mc_set_defer": ([vp, i32], None),
        "ref_mc_set_fixed_budget": ([vp, i32], None),
        "ref_mc_save": ([vp, C.c_char_p], i32),
        "ref_mc_load": ([vp, C.c_char_p], i32),
        "ref_mc_dropped_dim0": ([vp], C.c_uint64),
        "ref_mc_run_native": ([vp, u32, i32, P(abi.Stats)], None),
        "ref_random_uniforms": ([u32, i64, vp], None),
        "ref_vegas_optimize": ([i32, i32, dbl, vp, i32, u32, i64, i64, dbl, dbl, i64, i32, vp, P(i64), P(i64),
                                P(abi.Stats), vp, i64], i32),
        "ref_evaluate_batch": ([vp, i32, vp, i64, vp], None),
        "ref_philox_uniforms": ([C.c_uint64, C.c_uint64, i64, i32, vp], None),
        "ref_philox_stream_uniforms": ([C.c_uint64, C.c_uint64, i64, i32, C.c_uint32, vp], None),
        "ref_mc_point_values": ([vp, vp, i64, vp, vp, vp], None),
        "ref_construct_channels": ([dbl, vp, i32, vp, i32, vp, i32, vp, i32, P(abi.Cuts), i32, vp, i64, P(i64),
                                    vp, P(i32), vp, P(i32), i32], i32),
    }
    for name, (args, res) in sigs.items():
        real = prefix + name[4:]
        if not hasattr(L, real):
            continue
        fn = getattr(L, real)
        fn.argtypes = args
        fn.restype = res
    return _Prefixed(L, prefix)


REF = OracleLib(os.path.join(HERE, "_ref", "libchili_ref.so"), "ref_")
PORT = OracleLib(os.path.join(HERE, "libchili_oracle.so"), "orc_")


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def am_map(edges, u, oracle=REF):
    dims, b1 = edges.shape
    u = np.ascontiguousarray(u, dtype=np.float64)
    x = np.empty_like(u)
    jac = np.empty(u.shape[0])
    oracle().ref_am_map(dims, b1 - 1, _p(np.ascontiguousarray(edges)), _p(u), u.shape[0], _p(x), _p(jac))
    return x, jac


def am_weight(edges, x, oracle=REF):
    dims, b1 = edges.shape
    x = np.ascontiguousarray(x, dtype=np.float64)
    w = np.empty(x.shape[0])
    b = np.empty(x.shape, dtype=np.int32)
    oracle().ref_am_weight(dims, b1 - 1, _p(np.ascontiguousarray(edges)), _p(x), x.shape[0], _p(w), _p(b))
    return w, b


def am_adapt(edges, alpha, train, oracle=REF):
    dims, b1 = edges.shape
    out = np.empty_like(edges)
    oracle().ref_am_adapt(dims, b1 - 1, _p(np.ascontiguousarray(edges)), alpha,
                       _p(np.ascontiguousarray(train, dtype=np.float64)), _p(out))
    return out


def am_split(edges, nsplit, oracle=REF):
    dims, b1 = edges.shape
    out = np.empty((dims, nsplit * (b1 - 1) + 1))
    oracle().ref_am_split(dims, b1 - 1, _p(np.ascontiguousarray(edges)), nsplit, _p(out))
    return out


def vegas_iterate(edges, alpha, params, u, adapt=True, oracle=REF):
    """One Vegas::operator() on the given uniforms; returns (stats, train, new_edges)."""
    dims, b1 = edges.shape
    e = np.array(edges, dtype=np.float64, copy=True)
    p = np.ascontiguousarray(params, dtype=np.float64)
    u = np.ascontiguousarray(u, dtype=np.float64)
    st = abi.Stats()
    tr = np.empty(dims * (b1 - 1))
    oracle().ref_vegas_iterate(dims, b1 - 1, _p(e), alpha, 1 if adapt else 0, _p(p), p.size, u.shape[0], _p(u),
                            C.byref(st), _p(tr))
    return st, tr, e


def vegas_run(dims, bins, alpha, params, seed, ncalls, niter, oracle=REF):
    p = np.ascontiguousarray(params, dtype=np.float64)
    st = abi.Stats()
    oracle().ref_vegas_run(dims, bins, alpha, _p(p), p.size, seed, ncalls, niter, C.byref(st))
    return st


def random_uniforms(seed, n, oracle=REF):
    """The reference's own uniform stream (Random::Instance() seeded with
    `seed`, n draws; the reference build only)."""
    out = np.empty(n)
    oracle().ref_random_uniforms(seed, n, _p(out))
    return out


def vegas_optimize(dims, bins, alpha, params, seed, ncalls, nrefine, atol, rtol, nitn, max_iter=256,
                   oracle=REF):
    """The reference's Vegas::Optimize on the camel with its own generator
    seeded by `seed` (the reference build only).  Returns a dict: iterations
    (StatsData tuples), bins, ncalls (after the last Refine), pooled
    StatsData, edges [dims, bins + 1]."""
    p = np.ascontiguousarray(params, dtype=np.float64)
    iters = (abi.Stats * max_iter)()
    b_out, n_out = C.c_int64(), C.c_int64()
    pooled = abi.Stats()
    cap = dims * (bins * 2 ** 12 + 1)
    edges = np.empty(cap)
    n_it = oracle().ref_vegas_optimize(dims, bins, alpha, _p(p), p.size, seed, ncalls, nrefine, atol, rtol, nitn,
                                       max_iter, iters, C.byref(b_out), C.byref(n_out), C.byref(pooled),
                                       _p(edges), cap)
    B = b_out.value
    return {"iterations": [iters[i].as_tuple() for i in range(min(n_it, max_iter))], "n_iterations": n_it,
            "bins": B, "ncalls": n_out.value, "pooled": pooled.as_tuple(),
            "edges": edges[:dims * (B + 1)].reshape(dims, B + 1).copy()}


def select(alpha, v, oracle=REF):
    a = np.ascontiguousarray(alpha, dtype=np.float64)
    v = np.ascontiguousarray(v, dtype=np.float64)
    out = np.empty(v.shape[0], dtype=np.int32)
    oracle().ref_select(_p(a), a.size, _p(v), v.shape[0], _p(out))
    return out


class MultiChannel:
    """Reference Integrand<FourVector> + MultiChannel over a ChannelSet."""

    def __init__(self, cs, bins, params, fkind=abi.CHILI_FUNC_PROPAGATOR, fparams=(),
                 pre=abi.CHILI_PRE_FINITE, oracle=REF):
        self.oracle = oracle
        self.cs = cs
        self.params = params
        self.bins = bins
        self.h = self.oracle().ref_mc_create(cs.descs, cs.nch, C.byref(cs.cuts), cs.sqrts, cs.n_ext, bins,
                                     C.byref(params))
        if not self.h:
            raise RuntimeError("reference rejected the channel set")
        self.ndims = self.oracle().ref_mc_ndims(self.h)
        self.nch = cs.nch
        self.n_ext = cs.n_ext
        fp = np.ascontiguousarray(fparams, dtype=np.float64)
        self._fp = fp
        self.oracle().ref_mc_set_integrand(self.h, fkind, _p(fp) if fp.size else None, fp.size, pre)

    def __del__(self):
        if getattr(self, "h", None):
            try:
                self.oracle().ref_mc_destroy(self.h)
            except Exception:
                pass
            self.h = None

    def set_cuts(self, sqrts, ptmin=30.0, etamax=99.0, delta_r=0.4):
        """PreProcess = CHILI_PRE_CUTS."""
        self.oracle().ref_mc_set_cuts(self.h, sqrts, ptmin, etamax, delta_r)

    def set_grids(self, edges):
        self.oracle().ref_mc_set_grids(self.h, _p(np.ascontiguousarray(edges, dtype=np.float64)))

    def get_grids(self):
        out = np.empty((self.nch, self.ndims, self.bins + 1))
        self.oracle().ref_mc_get_grids(self.h, _p(out))
        return out

    def set_alpha(self, a):
        self.oracle().ref_mc_set_alpha(self.h, _p(np.ascontiguousarray(a, dtype=np.float64)))

    def get_alpha(self):
        a, b, md = np.empty(self.nch), np.empty(self.nch), C.c_double()
        self.oracle().ref_mc_get_alpha(self.h, _p(a), _p(b), C.byref(md))
        return a, b, md.value

    def fsm_generate(self, ch, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        mom = np.empty((x.shape[0], self.n_ext, 4))
        self.oracle().ref_fsm_generate(self.h, ch, _p(x), x.shape[0], _p(mom))
        return mom

    def fsm_weight(self, ch, mom):
        mom = np.ascontiguousarray(mom, dtype=np.float64)
        x = np.empty((mom.shape[0], self.ndims))
        w = np.empty(mom.shape[0])
        self.oracle().ref_fsm_weight(self.h, ch, _p(mom), mom.shape[0], _p(x), _p(w))
        return w, x

    def weight(self, mom, ich):
        mom = np.ascontiguousarray(mom, dtype=np.float64)
        ich = np.ascontiguousarray(ich, dtype=np.int32)
        n = mom.shape[0]
        w, dens, x = np.empty(n), np.empty((n, self.nch)), np.empty((n, self.ndims))
        self.oracle().ref_mc_weight(self.h, _p(mom), _p(ich), n, _p(w), _p(dens), _p(x))
        return w, dens, x

    def iterate(self, u, guard=True):
        u = np.ascontiguousarray(u, dtype=np.float64)
        st, info = abi.Stats(), abi.MCIterInfo()
        rc = self.oracle().ref_mc_iterate(self.h, _p(u), u.shape[0], 1 if guard else 0, C.byref(st), C.byref(info))
        if rc != 0:
            raise RuntimeError(f"reference iteration ran out of uniforms (rc={rc})")
        return st, info

    def training(self):
        h = np.empty((self.nch, self.ndims, self.bins))
        a = np.empty(self.nch)
        self.oracle().ref_mc_get_training(self.h, _p(h), _p(a))
        return h, a

    def save(self, path):
        """MultiChannel::SaveAs (the reference build only)."""
        assert self.oracle().ref_mc_save(self.h, str(path).encode()) == 0

    def load(self, path):
        """MultiChannel::LoadFrom (the reference build only)."""
        assert self.oracle().ref_mc_load(self.h, str(path).encode()) == 0

    def set_defer(self, defer=True):
        """Collect the training data but leave Train to train()."""
        self.oracle().ref_mc_set_defer(self.h, 1 if defer else 0)

    def set_fixed_budget(self, on=True):
        """Every drawn point counts as a call, no retries: the semantics of
        the CUDA library's batched integrands with option batch_retry 0 (the C
        port only)."""
        self.oracle().ref_mc_set_fixed_budget(self.h, 1 if on else 0)

    def train(self, hist, atrain):
        """MultiChannel::Train on given training data (the MPI mode's step
        after the all-reduce)."""
        self.oracle().ref_mc_train(self.h, _p(np.ascontiguousarray(hist, dtype=np.float64)),
                                   _p(np.ascontiguousarray(atrain, dtype=np.float64)))

    def point_values(self, u):
        """Value f*w of each point, no retries (the C port only): (val, ich, mom)."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        n = u.shape[0]
        val, ich, mom = np.empty(n), np.empty(n, dtype=np.int32), np.empty((n, self.n_ext, 4))
        self.oracle().ref_mc_point_values(self.h, _p(u), n, _p(val), _p(ich), _p(mom))
        return val, ich, mom

    def run_native(self, seed, niter):
        st = abi.Stats()
        self.oracle().ref_mc_run_native(self.h, seed, niter, C.byref(st))
        return st

    def evaluate_batch(self, ch, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        out = np.empty(u.shape[0])
        self.oracle().ref_evaluate_batch(self.h, ch, _p(u), u.shape[0], _p(out))
        return out


def philox_uniforms(seed, ctr0, n, d, oracle=None):
    """The CUDA library's counter-based uniforms, regenerated on the CPU (port only)."""
    oracle = oracle or PORT
    out = np.empty((n, d))
    oracle().ref_philox_uniforms(seed, ctr0, n, d, _p(out))
    return out


def philox_stream_uniforms(seed, ctr0, n, d, stream, oracle=None):
    """Stream `stream` of the CUDA library's counter-based generator (port only)."""
    oracle = oracle or PORT
    out = np.empty((n, d))
    oracle().ref_philox_stream_uniforms(seed, ctr0, n, d, stream, _p(out))
    return out


def construct_channels(sqrts, flavs, rules, masses, widths, cuts=None, smax=2, oracle=REF):
    """The reference's ConstructChannels (the reference build only) with a
    Model whose Combinable is the table rules {(f1, f2): [flavours]}.
    Returns (channels, ptmin, etamax): channels = [(info, decays)] with info
    [(idx, pid, mass, width)] and decays [(parent, child1, child2)] from the
    mappers' serialized descriptions, in the reference's order; ptmin and
    etamax the completed cut tables (second overload only, else {})."""
    import struct
    rows = []
    for (f1, f2), out in rules.items():
        out = list(out)
        rows.append([f1, f2, len(out)] + out + [0] * (8 - len(out)))
    rt = np.ascontiguousarray(rows if rows else np.zeros((0, 11)), dtype=np.int32)
    fl = np.ascontiguousarray(flavs, dtype=np.int32)
    mt = (abi.IdxValue * max(1, len(masses)))(*[abi.IdxValue(abs(k), v) for k, v in masses.items()])
    wt = (abi.IdxValue * max(1, len(widths)))(*[abi.IdxValue(abs(k), v) for k, v in widths.items()])
    cin = abi.ChannelSet([], cuts, sqrts, len(flavs)) if cuts is not None else None
    cap = 1 << 24
    buf = C.create_string_buffer(cap)
    ln = C.c_int64()
    po, eo = (abi.IdxValue * 1024)(), (abi.IdxValue * 1024)()
    npo, neo = C.c_int(), C.c_int()
    n = oracle().ref_construct_channels(float(sqrts), _p(fl), len(flavs), _p(rt), len(rows), mt, len(masses), wt,
                                        len(widths), C.byref(cin.cuts) if cin else None, int(smax), buf, cap,
                                        C.byref(ln), po, C.byref(npo), eo, C.byref(neo), 1024)
    if n < 0:
        raise RuntimeError("the reference's ConstructChannels threw")
    data = buf.raw[:ln.value]
    pos = 0

    def take(fmt):
        nonlocal pos
        v = struct.unpack_from(fmt, data, pos)
        pos += struct.calcsize(fmt)
        return v

    def pinfo():
        return take("<Iidd")

    chans = []
    for _ in range(n):
        (nl,) = take("<Q")
        pos += nl  # mapper name
        (ni,) = take("<Q")
        info = [pinfo() for _ in range(ni)]
        (nd,) = take("<Q")
        dec = [(pinfo(), pinfo(), pinfo()) for _ in range(nd)]
        take("<ddQQ")
        (npt,) = take("<Q")
        take("<%dd" % npt)
        chans.append((info, dec))
    ptmin = {po[k].idx: po[k].value for k in range(npo.value)} if cuts is not None else {}
    etamax = {eo[k].idx: eo[k].value for k in range(neo.value)} if cuts is not None else {}
    return chans, ptmin, etamax

