"""Python binding of libchili_b200 (include/chili_gpu.h) over ctypes.

Arrays may be numpy arrays (host memory; staged by the library) or CUDA torch
tensors (device memory; used in place).  Every call checks the returned status
and raises ChiliError with the library's message.  There is no CPU fallback:
without the built library or a CUDA device the calls raise.
"""
import ctypes as C
import os

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libchili_b200.so")

_lib = None


class ChiliError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"chili_gpu error {code} ({abi.STATUS_NAMES.get(code, '?')}): {msg}")
        self.code = code


def _declare(lib):
    vp, i32, i64, u64, dbl = C.c_void_p, C.c_int, C.c_int64, C.c_uint64, C.c_double
    P = C.POINTER
    sigs = {
        "chili_gpu_create": ([i32, P(vp)], i32),
        "chili_gpu_destroy": ([vp], i32),
        "chili_gpu_last_error": ([vp], C.c_char_p),
        "chili_gpu_set_stream": ([vp, vp], i32),
        "chili_gpu_synchronize": ([vp], i32),
        "chili_gpu_launch_count": ([vp], u64),
        "chili_gpu_set_option": ([vp, C.c_char_p, i64], i32),
        "chili_gpu_kernel_time": ([vp, C.c_char_p, P(dbl), P(u64)], i32),
        "chili_gpu_set_grids": ([vp, vp, i32, i32, i32], i32),
        "chili_gpu_get_grids": ([vp, vp, i32, i32, i32], i32),
        "chili_gpu_grid_map": ([vp, i32, vp, vp, vp, i64], i32),
        "chili_gpu_grid_weight": ([vp, i32, vp, vp, vp, i64], i32),
        "chili_gpu_grid_adapt": ([vp, i32, dbl, vp], i32),
        "chili_gpu_grid_split": ([vp, i32], i32),
        "chili_gpu_set_integrand": ([vp, i32, vp, i32], i32),
        "chili_gpu_set_preprocess": ([vp, i32], i32),
        "chili_gpu_set_preprocess_cuts": ([vp, dbl, dbl, dbl, dbl], i32),
        "chili_gpu_vegas_iterate": ([vp, u64, u64, u64, vp, dbl, i32, vp, vp], i32),
        "chili_gpu_vegas_iterate_noalloc": ([vp, vp, i32, i32, vp, i32, u64, u64, u64, vp, vp], i32),
        "chili_gpu_vegas_generate": ([vp, u64, u64, u64, vp, vp], i32),
        "chili_gpu_fsmapper_weight_inout": ([vp, i32, vp, vp, vp, i64], i32),
        "chili_gpu_pack_training": ([vp, vp, i64], i32),
        "chili_gpu_set_channels": ([vp, P(abi.ChannelDesc), i32, P(abi.Cuts), dbl, i32], i32),
        "chili_gpu_ndims": ([vp], i32),
        "chili_gpu_check_channels": ([P(abi.ChannelDesc), i32, P(abi.Cuts), dbl, i32, C.c_char_p,
                                      C.c_size_t], i32),
        "chili_gpu_fsmapper_generate": ([vp, i32, vp, vp, i64], i32),
        "chili_gpu_fsmapper_weight": ([vp, i32, vp, vp, vp, i64], i32),
        "chili_gpu_set_alpha": ([vp, vp, i32], i32),
        "chili_gpu_get_alpha": ([vp, vp, vp, vp, i32], i32),
        "chili_gpu_select_channel": ([vp, vp, vp, i64], i32),
        "chili_gpu_multichannel_weight": ([vp, vp, vp, vp, vp, vp, i64], i32),
        "chili_gpu_multichannel_iterate": ([vp, P(abi.MultiChannelParams), u64, u64, vp, i64, i32,
                                            P(abi.Stats), P(abi.MCIterInfo)], i32),
        "chili_gpu_get_training": ([vp, vp, vp], i32),
        "chili_gpu_multichannel_train": ([vp, P(abi.MultiChannelParams), vp, vp], i32),
        "chili_gpu_save_checkpoint": ([vp, C.c_char_p, P(abi.MultiChannelParams), vp, i64], i32),
        "chili_gpu_load_checkpoint": ([vp, C.c_char_p, P(abi.MultiChannelParams), vp, i64, P(i64)], i32),
        "chili_gpu_generate": ([vp, i64, u64, u64, vp, vp, vp], i32),
        "chili_gpu_evaluate_batch": ([vp, i32, vp, vp, i64], i32),
        "chili_gpu_generate_unweighted": ([vp, i64, u64, u64, dbl, vp, vp, vp, i64, P(i64),
                                           P(abi.UnweightInfo)], i32),
        "chili_gpu_flow_init": ([vp, P(abi.FlowParams)], i32),
        "chili_gpu_flow_nparams": ([vp], i64),
        "chili_gpu_flow_get_params": ([vp, vp], i32),
        "chili_gpu_flow_set_params": ([vp, vp], i32),
        "chili_gpu_flow_get_beta": ([vp, vp], i32),
        "chili_gpu_flow_set_beta": ([vp, vp], i32),
        "chili_gpu_flow_density": ([vp, vp, vp, i64, vp, vp], i32),
        "chili_gpu_flow_sample_u": ([vp, vp, vp, i64, vp, vp], i32),
        "chili_gpu_flow_loss_grad": ([vp, vp, vp, vp, vp, vp, i64, P(dbl), vp], i32),
        "chili_gpu_flow_train": ([vp, i32, u64, u64, vp], i32),
        "chili_gpu_flow_iterate": ([vp, u64, u64, u64, i32, P(abi.Stats), P(abi.FlowIterInfo)], i32),
        "chili_gpu_tc_selftest": ([vp, i32, i32, i32, vp, vp, vp], i32),
        "chili_construct_channels": ([dbl, vp, i32, P(abi.Model), P(abi.Cuts), i32, P(vp), C.c_char_p,
                                      C.c_size_t], i32),
        "chili_channel_list_get": ([vp, P(P(abi.ChannelDesc)), P(i32), P(P(abi.Cuts))], i32),
        "chili_channel_list_free": ([vp], None),
        "chili_gpu_batch_set": ([vp, P(abi.Task), i32], i32),
        "chili_gpu_batch_iterate": ([vp, i32, u64, i32, vp, P(abi.BatchInfo)], i32),
        "chili_gpu_batch_get_grid": ([vp, i32, vp, vp], i32),
    }
    for name, (args, res) in sigs.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return sigs


EXPORTED = None


def load(path=LIB_PATH):
    """Load the CUDA library (raises if it is missing)."""
    global _lib, EXPORTED
    if _lib is None:
        if not os.path.exists(path):
            raise ChiliError(abi.CHILI_ERR_STATE,
                             f"{path} is not built; run `python -m chili_b200.build`")
        lib = C.CDLL(path)
        EXPORTED = sorted(_declare(lib))
        _lib = lib
    return _lib


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags.c_contiguous:
            raise ValueError("arrays must be C-contiguous")
        return C.c_void_p(a.ctypes.data)
    if hasattr(a, "data_ptr"):  # torch tensor
        if not a.is_contiguous():
            raise ValueError("tensors must be contiguous")
        return C.c_void_p(a.data_ptr())
    raise TypeError(f"unsupported buffer type {type(a)}")


def _f64(a):
    return None if a is None else (np.ascontiguousarray(a, dtype=np.float64) if isinstance(a, (np.ndarray, list, tuple)) else a)


class Context:
    """One chili_ctx: a device, a stream, grids, channels and an integrand."""

    def __init__(self, device=0):
        self.lib = load()
        h = C.c_void_p()
        self._check(self.lib.chili_gpu_create(device, C.byref(h)), None)
        self.h = h
        self._keep = []
        self.nch = 0
        self.dims = 0
        self.bins = 0
        self.n_ext = 0

    def _check(self, rc, h):
        if rc != abi.CHILI_OK:
            msg = self.lib.chili_gpu_last_error(h)
            raise ChiliError(rc, msg.decode() if msg else "")

    def call(self, name, *args):
        self._check(getattr(self.lib, name)(self.h, *args), self.h)

    def close(self):
        if getattr(self, "h", None):
            self.lib.chili_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------- basics
    def set_stream(self, stream_ptr):
        self.call("chili_gpu_set_stream", C.c_void_p(stream_ptr) if stream_ptr else None)

    def synchronize(self):
        self.call("chili_gpu_synchronize")

    def set_option(self, name, value):
        self.call("chili_gpu_set_option", name.encode(), int(value))

    def kernel_time(self, name):
        ms, n = C.c_double(), C.c_uint64()
        self.call("chili_gpu_kernel_time", name.encode(), C.byref(ms), C.byref(n))
        return ms.value, n.value

    @property
    def launches(self):
        return int(self.lib.chili_gpu_launch_count(self.h))

    # ----------------------------------------------------------------- grids
    def set_grids(self, edges):
        edges = _f64(edges)
        nch, dims, b1 = edges.shape
        self.call("chili_gpu_set_grids", _ptr(edges), nch, dims, b1 - 1)
        self.dims, self.bins = dims, b1 - 1

    def uniform_grids(self, nch, dims, bins):
        e = np.tile(np.arange(bins + 1, dtype=np.float64) / bins, (nch, dims, 1))
        self.set_grids(e)

    def get_grids(self):
        nch = self.nch if self.nch else 1
        out = np.empty((self._grid_count(), self.dims, self.bins + 1))
        self.call("chili_gpu_get_grids", _ptr(out), out.shape[0], self.dims, self.bins)
        return out

    def _grid_count(self):
        return getattr(self, "_g_nch", None) or (self.nch if self.nch else 1)

    def grid_map(self, ch, u):
        u = _f64(u)
        n = u.shape[0]
        x = np.empty_like(u)
        jac = np.empty(n)
        self.call("chili_gpu_grid_map", ch, _ptr(u), _ptr(x), _ptr(jac), n)
        return x, jac

    def grid_weight(self, ch, x):
        x = _f64(x)
        n = x.shape[0]
        w = np.empty(n)
        b = np.empty(x.shape, dtype=np.int32)
        self.call("chili_gpu_grid_weight", ch, _ptr(x), _ptr(w), _ptr(b), n)
        return w, b

    def grid_adapt(self, ch, alpha, train):
        self.call("chili_gpu_grid_adapt", ch, float(alpha), _ptr(_f64(train)))

    def grid_split(self, nsplit=2):
        self.call("chili_gpu_grid_split", nsplit)
        self.bins *= nsplit

    # ------------------------------------------------------------- integrand
    def set_integrand(self, kind, params=()):
        p = np.ascontiguousarray(params, dtype=np.float64)
        self._keep.append(p)
        self.call("chili_gpu_set_integrand", kind, _ptr(p) if p.size else None, int(p.size))

    def set_preprocess_cuts(self, sqrts, ptmin=30.0, etamax=99.0, delta_r=0.4):
        """PreProcess = CHILI_PRE_CUTS (physical region and cuts)."""
        self.call("chili_gpu_set_preprocess_cuts", float(sqrts), float(ptmin), float(etamax), float(delta_r))

    def set_preprocess(self, kind):
        self.call("chili_gpu_set_preprocess", kind)

    # --------------------------------------------------------- plain VEGAS
    def vegas_iterate(self, ncalls, seed=42, counter=0, u=None, alpha=1.5, adapt=True, train=False):
        st = abi.Stats()
        tr = np.empty(self.dims * self.bins) if train else None
        u = _f64(u)
        self.call("chili_gpu_vegas_iterate", int(ncalls), int(seed), int(counter), _ptr(u),
                  float(alpha), 1 if adapt else 0, C.byref(st), _ptr(tr))
        return (st, tr) if train else st

    def vegas_generate(self, n, seed=42, counter=0, out=None):
        """n materialised VEGAS points of grid 0 on the camel: (x[n, dims],
        w[n]).  out = (x, w) may be given (numpy or CUDA tensors)."""
        if out is None:
            out = (np.empty((n, self.dims)), np.empty(n))
        x, w = out
        self.call("chili_gpu_vegas_generate", int(n), int(seed), int(counter), _ptr(x), _ptr(w))
        return x, w

    # -------------------------------------------------------------- channels
    def set_channels(self, cs):
        self._keep.append(cs)
        self.call("chili_gpu_set_channels", cs.descs, cs.nch, C.byref(cs.cuts), cs.sqrts, cs.n_ext)
        self.nch, self.n_ext = cs.nch, cs.n_ext
        self.ndims = int(self.lib.chili_gpu_ndims(self.h))

    def fsmapper_generate(self, ch, x):
        x = _f64(x)
        n = x.shape[0]
        mom = np.empty((n, self.n_ext, 4))
        self.call("chili_gpu_fsmapper_generate", ch, _ptr(x), _ptr(mom), n)
        return mom

    def fsmapper_weight(self, ch, mom):
        mom = _f64(mom)
        n = mom.shape[0]
        x = np.empty((n, self.ndims))
        w = np.empty(n)
        self.call("chili_gpu_fsmapper_weight", ch, _ptr(mom), _ptr(x), _ptr(w), n)
        return w, x

    # ---------------------------------------------------------- multichannel
    def set_alpha(self, alpha):
        a = _f64(alpha)
        self.call("chili_gpu_set_alpha", _ptr(a), self.nch)

    def get_alpha(self):
        a, b, md = np.empty(self.nch), np.empty(self.nch), C.c_double()
        self.call("chili_gpu_get_alpha", _ptr(a), _ptr(b), C.byref(md), self.nch)
        return a, b, md.value

    def select_channel(self, v):
        v = _f64(v)
        out = np.empty(v.shape[0], dtype=np.int32)
        self.call("chili_gpu_select_channel", _ptr(v), _ptr(out), v.shape[0])
        return out

    def multichannel_weight(self, mom, ich):
        mom = _f64(mom)
        ich = np.ascontiguousarray(ich, dtype=np.int32)
        n = mom.shape[0]
        w, dens, x = np.empty(n), np.empty((n, self.nch)), np.empty((n, self.ndims))
        self.call("chili_gpu_multichannel_weight", _ptr(mom), _ptr(ich), _ptr(w), _ptr(dens), _ptr(x), n)
        return w, dens, x

    def multichannel_iterate(self, params, seed=7, counter=0, u=None, guard=True):
        st, info = abi.Stats(), abi.MCIterInfo()
        u = _f64(u)
        n_u = 0 if u is None else u.shape[0]
        self.call("chili_gpu_multichannel_iterate", C.byref(params), int(seed), int(counter), _ptr(u),
                  n_u, 1 if guard else 0, C.byref(st), C.byref(info))
        return st, info

    def get_training(self):
        h = np.empty((self.nch, self.ndims, self.bins))
        a = np.empty(self.nch)
        self.call("chili_gpu_get_training", _ptr(h), _ptr(a))
        return h, a

    def packed_training_len(self):
        return self.nch * self.ndims * self.bins + self.nch + 6

    def pack_training(self, buf):
        """[hist | alpha_train | n, sum, sum2, n_finite | max, -min] of the last
        iteration into buf (a CUDA tensor stays on the device)."""
        self.call("chili_gpu_pack_training", _ptr(buf), int(buf.shape[0]))
        return buf

    def multichannel_train(self, params, hist, alpha_train):
        """Train from given (e.g. all-reduced) training data."""
        self.call("chili_gpu_multichannel_train", C.byref(params), _ptr(_f64(hist)), _ptr(_f64(alpha_train)))

    def save_checkpoint(self, path, params, results=()):
        """The reference's results.chili (MultiChannel::SaveAs)."""
        res = (abi.Stats * max(len(results), 1))()
        for k, s in enumerate(results):
            res[k] = s if isinstance(s, abi.Stats) else abi.Stats(*s)
        self.call("chili_gpu_save_checkpoint", str(path).encode(), C.byref(params), C.cast(res, C.c_void_p),
                  len(results))

    def load_checkpoint(self, path, max_results=4096):
        """MultiChannel::LoadFrom; returns (params, [Stats])."""
        p = abi.MultiChannelParams.defaults()
        res = (abi.Stats * max_results)()
        n = C.c_int64()
        self.call("chili_gpu_load_checkpoint", str(path).encode(), C.byref(p), C.cast(res, C.c_void_p), max_results,
                  C.byref(n))
        return p, [res[k] for k in range(min(n.value, max_results))]

    def generate(self, n, seed=7, counter=0):
        mom = np.empty((n, self.n_ext, 4))
        w = np.empty(n)
        ch = np.empty(n, dtype=np.int32)
        self.call("chili_gpu_generate", int(n), int(seed), int(counter), _ptr(mom), _ptr(w), _ptr(ch))
        return mom, w, ch

    def generate_unweighted(self, n, w_max, seed=7, counter=0, max_events=None, out=None):
        """Unweighted events of n drawn points: (mom [k, n_ext, 4], wgt [k],
        ch [k], UnweightInfo), k = min(kept, max_events).  out: optional
        (mom, wgt, ch) buffers (numpy or device tensors) of max_events rows."""
        if max_events is None:
            max_events = n
        if out is None:
            out = (np.empty((max_events, self.n_ext, 4)), np.empty(max_events), np.empty(max_events, dtype=np.int32))
        mom, wgt, ch = out
        ne = C.c_int64()
        info = abi.UnweightInfo()
        self.call("chili_gpu_generate_unweighted", int(n), int(seed), int(counter), float(w_max), _ptr(mom),
                  _ptr(wgt), _ptr(ch), int(max_events), C.byref(ne), C.byref(info))
        k = min(ne.value, max_events)
        return tuple(None if a is None else a[:k] for a in (mom, wgt, ch)) + (info,)

    def evaluate_batch(self, ch, u):
        u = _f64(u)
        out = np.empty(u.shape[0])
        self.call("chili_gpu_evaluate_batch", ch, _ptr(u), _ptr(out), u.shape[0])
        return out

    # ------------------------------------------------------ learned proposal
    def flow_init(self, params=None, **kw):
        p = params or abi.FlowParams.defaults(**kw)
        self.call("chili_gpu_flow_init", C.byref(p))
        self.flow_np = int(self.lib.chili_gpu_flow_nparams(self.h))
        return self.flow_np

    def flow_get_params(self):
        out = np.empty(self.flow_np, dtype=np.float32)
        self.call("chili_gpu_flow_get_params", _ptr(out))
        return out

    def flow_set_params(self, prm):
        prm = np.ascontiguousarray(prm, dtype=np.float32)
        assert prm.size == self.flow_np
        self.call("chili_gpu_flow_set_params", _ptr(prm))

    def flow_get_beta(self):
        out = np.empty(self.nch)
        self.call("chili_gpu_flow_get_beta", _ptr(out))
        return out

    def flow_set_beta(self, beta):
        self.call("chili_gpu_flow_set_beta", _ptr(_f64(beta)))

    def _flow_map(self, name, x, ch):
        x = np.ascontiguousarray(x, dtype=np.float32)
        ch = np.ascontiguousarray(ch, dtype=np.int32)
        out = np.empty_like(x)
        lq = np.empty(x.shape[0], dtype=np.float32)
        self.call(name, _ptr(x), _ptr(ch), x.shape[0], _ptr(out), _ptr(lq))
        return out, lq

    def flow_density(self, u, ch):
        """u -> z and log q(u) of each point's channel flow."""
        return self._flow_map("chili_gpu_flow_density", u, ch)

    def flow_sample_u(self, z, ch):
        """z -> u and log q(u)."""
        return self._flow_map("chili_gpu_flow_sample_u", z, ch)

    def flow_loss_grad(self, u, ch, logf, feat, logprior):
        f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)
        u, feat, logprior, logf = f32(u), f32(feat), f32(logprior), f32(logf)
        ch = np.ascontiguousarray(ch, dtype=np.int32)
        loss = C.c_double()
        grad = np.empty(self.flow_np, dtype=np.float32)
        self.call("chili_gpu_flow_loss_grad", _ptr(u), _ptr(ch), _ptr(logf), _ptr(feat), _ptr(logprior),
                  u.shape[0], C.byref(loss), _ptr(grad))
        return loss.value, grad

    def flow_train(self, steps, seed=7, counter=0):
        loss = np.empty(max(steps, 1))
        self.call("chili_gpu_flow_train", int(steps), int(seed), int(counter), _ptr(loss))
        return loss[:steps]

    def flow_iterate(self, ncalls, seed=7, counter=0, adapt_beta=False):
        st, info = abi.Stats(), abi.FlowIterInfo()
        self.call("chili_gpu_flow_iterate", int(ncalls), int(seed), int(counter), 1 if adapt_beta else 0,
                  C.byref(st), C.byref(info))
        return st, info

    def tc_selftest(self, mode, A, B, N):
        A = np.ascontiguousarray(A, dtype=np.float32)
        B = np.ascontiguousarray(B, dtype=np.float32)
        K = A.shape[1] if mode != 1 else A.shape[0]
        out = np.empty((128, N), dtype=np.float32)
        self.call("chili_gpu_tc_selftest", mode, K, N, _ptr(A), _ptr(B), _ptr(out))
        return out


    # ------------------------------------------------ batched integrands
    def batch_set(self, tasks):
        """tasks: list of dicts, {"kind": "camel", "dims", "bins", "ncalls",
        "params", "grid_alpha"} or {"kind": "multichannel", "channels":
        ChannelSet, "bins", "ncalls", "fkind", "params", "pre", "pre_cuts",
        "grid_alpha", "beta", "min_alpha"}."""
        arr = (abi.Task * len(tasks))()
        keep = []
        shapes = []
        for k, t in enumerate(tasks):
            T = arr[k]
            T.bins = int(t.get("bins", 50))
            T.ncalls = int(t["ncalls"])
            T.grid_alpha = float(t.get("grid_alpha", 1.5))
            T.beta = float(t.get("beta", 0.25))
            T.min_alpha = float(t.get("min_alpha", 1e-5))
            prm = np.ascontiguousarray(t.get("params", []), dtype=np.float64)
            keep.append(prm)
            T.nparams = prm.size
            T.params = prm.ctypes.data_as(C.POINTER(C.c_double)) if prm.size else None
            if t["kind"] == "camel":
                T.kind = abi.CHILI_TASK_CAMEL
                T.dims = int(t["dims"])
                shapes.append((1, T.dims, T.bins))
            else:
                cs = t["channels"]
                keep.append(cs)
                T.kind = abi.CHILI_TASK_MULTICHANNEL
                T.fkind = int(t.get("fkind", abi.CHILI_FUNC_PROPAGATOR))
                T.pre = int(t.get("pre", abi.CHILI_PRE_FINITE))
                for i, v in enumerate(t.get("pre_cuts", (0.0, 0.0, 0.0, 0.0))):
                    T.pre_cuts[i] = float(v)
                T.nch = cs.nch
                T.descs = C.cast(cs.descs, C.POINTER(abi.ChannelDesc))
                T.cuts = C.pointer(cs.cuts)
                T.sqrts = cs.sqrts
                T.n_ext = cs.n_ext
                shapes.append((cs.nch, cs.ndims, T.bins))
        self._batch_shapes = []
        self.call("chili_gpu_batch_set", arr, len(tasks))
        self._batch_shapes = shapes
        return shapes

    def batch_iterate(self, iterations=1, seed=42, adapt=True):
        """-> (stats [iterations, ntasks, 6] as n, min, max, sum, sum2,
        n_finite; BatchInfo)."""
        nt = len(getattr(self, "_batch_shapes", []))
        st = np.empty((iterations, max(nt, 1), 6), dtype=np.float64)
        info = abi.BatchInfo()
        self.call("chili_gpu_batch_iterate", int(iterations), int(seed), 1 if adapt else 0, _ptr(st),
                  C.byref(info))
        return st, info

    def batch_get_grid(self, task):
        nch, dims, bins = self._batch_shapes[task]
        edges = np.empty((nch, dims, bins + 1), dtype=np.float64)
        alpha = np.empty(nch, dtype=np.float64)
        self.call("chili_gpu_batch_get_grid", int(task), _ptr(edges), _ptr(alpha))
        return edges, alpha


def flow_layout(dims, nch, n_ext, layers=6, hidden=128, depth=2):
    """Offsets of the flat parameter vector of the learned proposal (the
    layout that include/chili_gpu.h documents): a list of (name, offset,
    shape) with the oracle's parameter names."""
    from . import flowspec
    return flowspec.layout(dims, nch, n_ext, layers, hidden, depth)


def construct_channels(flavs, combinable, masses, widths, sqrts, cuts=None, smax=2):
    """ConstructChannels (src/Channel/ChannelNode.cc:74-291) in the library:
    flavs = incoming then outgoing flavours; combinable = callable (f1, f2) ->
    flavours, or a dict {(f1, f2): [flavours]}; masses / widths = {pid:
    value} (keyed by |pid|); cuts = None (the reference's default cuts) or a
    cut dict (channels.default_cuts layout).  Returns an abi.ChannelSet for
    Context.set_channels."""
    lib = load()
    fn = (lambda a, b: combinable.get((a, b), [])) if isinstance(combinable, dict) else combinable

    def cb(f1, f2, out, max_out, user):
        try:
            r = [int(v) for v in fn(int(f1), int(f2))]
        except Exception:
            return -1
        if len(r) > max_out:
            return -1
        for i, v in enumerate(r):
            out[i] = v
        return len(r)

    cfn = abi.COMBINABLE_FN(cb)
    mt = (abi.IdxValue * max(1, len(masses)))(*[abi.IdxValue(abs(int(k)), float(v)) for k, v in masses.items()])
    wt = (abi.IdxValue * max(1, len(widths)))(*[abi.IdxValue(abs(int(k)), float(v)) for k, v in widths.items()])
    model = abi.Model(cfn, None, len(masses), mt, len(widths), wt)
    fl = (C.c_int32 * len(flavs))(*[int(f) for f in flavs])
    cin = abi.ChannelSet([], cuts, sqrts, len(flavs)) if cuts is not None else None
    h = C.c_void_p()
    err = C.create_string_buffer(512)
    rc = lib.chili_construct_channels(float(sqrts), fl, len(flavs), C.byref(model),
                                      C.byref(cin.cuts) if cin else None, int(smax), C.byref(h), err, 512)
    if rc != 0:
        raise ChiliError(rc, err.value.decode())
    try:
        dp, n, cp = C.POINTER(abi.ChannelDesc)(), C.c_int32(), C.POINTER(abi.Cuts)()
        lib.chili_channel_list_get(h, C.byref(dp), C.byref(n), C.byref(cp))
        chans = []
        for i in range(n.value):
            d = dp[i]
            info = [abi.ParticleInfo(d.info[k].idx, d.info[k].pid, d.info[k].mass, d.info[k].width)
                    for k in range(d.n_info)]
            dec = [abi.Decay(*[abi.ParticleInfo(q.idx, q.pid, q.mass, q.width)
                               for q in (d.decays[k].parent, d.decays[k].child1, d.decays[k].child2)])
                   for k in range(d.n_decays)]
            chans.append((info, dec))
        c = cp.contents
        out_cuts = {"sexternal": [c.sexternal[k] for k in range(c.n_sexternal)],
                    "deltaR": {(c.deltaR[k].pid1, c.deltaR[k].pid2): c.deltaR[k].value for k in range(c.n_deltaR)},
                    "smin": {c.smin[k].idx: c.smin[k].value for k in range(c.n_smin)},
                    "ptmin": {c.ptmin[k].idx: c.ptmin[k].value for k in range(c.n_ptmin)},
                    "etamax": {c.etamax[k].idx: c.etamax[k].value for k in range(c.n_etamax)}}
    finally:
        lib.chili_channel_list_free(h)
    return abi.ChannelSet(chans, out_cuts, sqrts, len(flavs))


def check_channels(cs):
    """Host-only validation of a ChannelSet; returns '' or the reason."""
    lib = load()
    buf = C.create_string_buffer(512)
    lib.chili_gpu_check_channels(cs.descs, cs.nch, C.byref(cs.cuts), cs.sqrts, cs.n_ext, buf, 512)
    return buf.value.decode()


def stats_mean_error(st):
    """StatsData::Mean and ::Error (Statistics.hh:90-126)."""
    n, s, s2 = st[0], st[3], st[4]
    mean = s / n
    var = (s2 / n - mean * mean) / (n - 1)
    return mean, float(np.sqrt(var)) if var > 0 else 0.0


def optimize(ctx, params, seed=7, counter=0, log=None):
    """MultiChannel::Optimize (MultiChannel.hh:253-270) on a context with
    channels, grids and integrand set: iterations until the pooled relative
    error reaches params.rtol or params.niterations iterations ran.  With
    `log` (a text file object) one JSON line per iteration: iteration,
    estimate and error of the iteration and pooled, points tried, calls,
    nonzero values, largest weight, unweighting efficiency (sum / w_max / n),
    seconds.  Returns (pooled mean, pooled error, the per-iteration
    records)."""
    import json
    import time
    pooled = np.zeros(6)
    records = []
    it = 0
    while it < params.niterations:
        t0 = time.perf_counter()
        st, info = ctx.multichannel_iterate(params, seed=seed, counter=counter)
        dt = time.perf_counter() - t0
        counter += info.points_tried
        t = st.as_tuple()
        pooled += np.array(t) * np.array([1, 0, 0, 1, 1, 1])
        m_it, e_it = stats_mean_error(t)
        mean, err = stats_mean_error(pooled)
        rec = {"iteration": it, "estimate": m_it, "error": e_it, "pooled": mean, "pooled_error": err,
               "points_tried": int(info.points_tried), "n": t[0], "n_nonzero": t[5], "w_max": info.weight_max,
               "unweighting_efficiency": (t[3] / info.weight_max / t[0]) if info.weight_max > 0 else 0.0,
               "seconds": dt}
        records.append(rec)
        if log is not None:
            log.write(json.dumps(rec) + "\n")
        it += 1
        if mean != 0 and err / abs(mean) <= params.rtol:
            break
    mean, err = stats_mean_error(pooled)
    return mean, err, records
