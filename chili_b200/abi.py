"""ctypes mirror of include/chili_gpu.h (structs, enums, limits).

The same structs describe channels and cuts to the CUDA library
(libchili_b200.so) and to the CPU oracles used by the tests, so the layout here
must match the header field for field.
"""
import ctypes as C

CHILI_OK = 0
CHILI_ERR_INVALID_ARG = 1
CHILI_ERR_CUDA = 2
CHILI_ERR_TIMEOUT = 3
CHILI_ERR_NAN_GRID = 4
CHILI_ERR_STATE = 5
CHILI_ERR_LIMIT = 6

STATUS_NAMES = {
    CHILI_OK: "ok",
    CHILI_ERR_INVALID_ARG: "invalid argument",
    CHILI_ERR_CUDA: "CUDA error",
    CHILI_ERR_TIMEOUT: "timeout",
    CHILI_ERR_NAN_GRID: "non-finite grid",
    CHILI_ERR_STATE: "bad state",
    CHILI_ERR_LIMIT: "limit exceeded",
}

CHILI_MAX_EXT = 10
CHILI_MAX_DIMS = 32
CHILI_MAX_CHANNELS = 200
CHILI_MAX_BINS = 4096
CHILI_MAX_INTEGRAND_PARAMS = 128

CHILI_FUNC_UNIT = 0
CHILI_FUNC_CAMEL = 1
CHILI_FUNC_PROPAGATOR = 2
CHILI_FUNC_PROPAGATOR_TOP2 = 3

CHILI_PRE_ACCEPT_ALL = 0
CHILI_PRE_FINITE = 1
CHILI_PRE_CUTS = 2


class ParticleInfo(C.Structure):
    """chili_particle_info == ParticleInfo (ChannelNode.hh:26-32)."""
    _fields_ = [("idx", C.c_uint32), ("pid", C.c_int32),
                ("mass", C.c_double), ("width", C.c_double)]

    def key(self):
        """Ordering key of ParticleInfo::operator< (ChannelNode.cc:293-301)."""
        return (self.idx, self.mass, self.width)

    def __repr__(self):
        return f"P({self.idx},{self.pid},{self.mass},{self.width})"


class Decay(C.Structure):
    _fields_ = [("parent", ParticleInfo), ("child1", ParticleInfo),
                ("child2", ParticleInfo)]


class ChannelDesc(C.Structure):
    _fields_ = [("n_info", C.c_int32), ("info", C.POINTER(ParticleInfo)),
                ("n_decays", C.c_int32), ("decays", C.POINTER(Decay))]


class IdxValue(C.Structure):
    _fields_ = [("idx", C.c_uint32), ("value", C.c_double)]


class PidPairValue(C.Structure):
    _fields_ = [("pid1", C.c_int32), ("pid2", C.c_int32), ("value", C.c_double)]


class Cuts(C.Structure):
    _fields_ = [("n_sexternal", C.c_int32), ("sexternal", C.POINTER(C.c_double)),
                ("n_deltaR", C.c_int32), ("deltaR", C.POINTER(PidPairValue)),
                ("n_smin", C.c_int32), ("smin", C.POINTER(IdxValue)),
                ("n_ptmin", C.c_int32), ("ptmin", C.POINTER(IdxValue)),
                ("n_etamax", C.c_int32), ("etamax", C.POINTER(IdxValue))]


class Stats(C.Structure):
    """chili_stats == StatsData (Statistics.hh:62-142) field order."""
    _fields_ = [("n", C.c_double), ("min", C.c_double), ("max", C.c_double),
                ("sum", C.c_double), ("sum2", C.c_double), ("n_finite", C.c_double)]

    def as_tuple(self):
        return (self.n, self.min, self.max, self.sum, self.sum2, self.n_finite)


class MultiChannelParams(C.Structure):
    _fields_ = [("ncalls", C.c_uint64), ("niterations", C.c_uint64),
                ("rtol", C.c_double), ("nrefine", C.c_uint64),
                ("beta", C.c_double), ("min_alpha", C.c_double),
                ("refine_size", C.c_double), ("max_bins", C.c_uint64),
                ("iteration", C.c_uint64), ("should_optimize", C.c_int32),
                ("grid_alpha", C.c_double)]

    @classmethod
    def defaults(cls, **kw):
        """MultiChannelParams defaults (MultiChannel.hh:38-45), grid alpha of
        VegasParams (Vegas.hh:36)."""
        p = cls(ncalls=10000, niterations=10, rtol=1e-5, nrefine=1, beta=0.25,
                min_alpha=1e-5, refine_size=1.5, max_bins=200, iteration=0,
                should_optimize=1, grid_alpha=1.0)
        for k, v in kw.items():
            setattr(p, k, v)
        return p


class MCIterInfo(C.Structure):
    _fields_ = [("points_tried", C.c_uint64), ("points_accepted", C.c_uint64),
                ("rejected_pre", C.c_uint64), ("rejected_nan", C.c_uint64),
                ("weight_max", C.c_double), ("nonfinite_alpha_terms", C.c_double),
                ("points_weighted", C.c_uint64), ("points_drawn", C.c_uint64), ("chunks", C.c_uint64)]


class FlowParams(C.Structure):
    """chili_flow_params (learned proposal)."""
    _fields_ = [("layers", C.c_int32), ("batch", C.c_int32), ("lr", C.c_double), ("init_seed", C.c_uint64),
                ("hidden", C.c_int32), ("depth", C.c_int32)]

    @classmethod
    def defaults(cls, **kw):
        p = cls(layers=6, batch=65536, lr=1e-3, init_seed=1, hidden=128, depth=2)
        for k, v in kw.items():
            setattr(p, k, v)
        return p


class FlowIterInfo(C.Structure):
    _fields_ = [("points", C.c_uint64), ("nonzero", C.c_uint64), ("nonfinite", C.c_uint64),
                ("weight_max", C.c_double), ("unweighting_efficiency", C.c_double)]


COMBINABLE_FN = C.CFUNCTYPE(C.c_int, C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.c_int32, C.c_void_p)


class Model(C.Structure):
    """chili_model: Combinable callback and |pid|-keyed masses and widths."""
    _fields_ = [("combinable", COMBINABLE_FN), ("user", C.c_void_p),
                ("n_masses", C.c_int32), ("masses", C.POINTER(IdxValue)),
                ("n_widths", C.c_int32), ("widths", C.POINTER(IdxValue))]


class UnweightInfo(C.Structure):
    """chili_unweight_info."""
    _fields_ = [("points", C.c_uint64), ("rejected_pre", C.c_uint64), ("kept", C.c_uint64),
                ("overweight", C.c_uint64), ("sum", C.c_double), ("max", C.c_double)]


CHILI_TASK_CAMEL = 0
CHILI_TASK_MULTICHANNEL = 1


class Task(C.Structure):
    """chili_task (batched integrands)."""
    _fields_ = [("kind", C.c_int32), ("dims", C.c_int32), ("bins", C.c_int32), ("ncalls", C.c_uint64),
                ("grid_alpha", C.c_double), ("beta", C.c_double), ("min_alpha", C.c_double),
                ("fkind", C.c_int32), ("nparams", C.c_int32), ("params", C.POINTER(C.c_double)),
                ("pre", C.c_int32), ("nch", C.c_int32), ("descs", C.POINTER(ChannelDesc)),
                ("cuts", C.POINTER(Cuts)), ("sqrts", C.c_double), ("n_ext", C.c_int32),
                ("pre_cuts", C.c_double * 4)]


class BatchInfo(C.Structure):
    _fields_ = [("block", C.c_uint32), ("points_per_thread", C.c_uint32), ("ms_per_iteration", C.c_double),
                ("units", C.c_uint64), ("points", C.c_uint64), ("retry_rounds", C.c_uint64)]


class ChannelSet:
    """Owns ctypes arrays for a list of channel descriptions and one Cuts
    table, keeping them alive while a library call reads them."""

    def __init__(self, channels, cuts, sqrts, n_ext):
        self.sqrts = float(sqrts)
        self.n_ext = int(n_ext)
        self._keep = []
        self.descs = (ChannelDesc * len(channels))()
        for i, (info, decays) in enumerate(channels):
            ia = (ParticleInfo * max(1, len(info)))(*info)
            da = (Decay * max(1, len(decays)))(*decays)
            self._keep += [ia, da]
            self.descs[i] = ChannelDesc(len(info), ia, len(decays), da)
        self.nch = len(channels)
        self.channels = channels
        self.cuts = self._make_cuts(cuts)

    def _make_cuts(self, cuts):
        sext = (C.c_double * max(1, len(cuts["sexternal"])))(*cuts["sexternal"])
        dr = [PidPairValue(a, b, v) for (a, b), v in cuts["deltaR"].items()]
        dra = (PidPairValue * max(1, len(dr)))(*dr)
        tabs = {}
        for name in ("smin", "ptmin", "etamax"):
            items = [IdxValue(k, v) for k, v in cuts[name].items()]
            tabs[name] = (IdxValue * max(1, len(items)))(*items)
            tabs["n_" + name] = len(items)
        self._keep += [sext, dra] + [tabs[k] for k in ("smin", "ptmin", "etamax")]
        return Cuts(len(cuts["sexternal"]), sext, len(dr), dra,
                    tabs["n_smin"], tabs["smin"], tabs["n_ptmin"], tabs["ptmin"],
                    tabs["n_etamax"], tabs["etamax"])

    @property
    def ndims(self):
        return 3 * (self.n_ext - 2) - 2
