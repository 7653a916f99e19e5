"""The reference's MPI mode on host processes (TEST INFRASTRUCTURE ONLY:
tests/ and bench.py's CPU legs).

MultiChannel::operator() under ENABLE_MPI (MultiChannel.hh:207-212) runs
ncalls / size points on every rank, all-reduces the alpha-training sums and
every channel's histogram before MultiChannel::Train (MultiChannel.hh:184-190)
and the StatsData in UpdateResults (MultiChannel.cc:69-77), so every rank
adapts alike.  MPI is not installed here; this module runs one process per
rank, each holding the reference's own Integrand + MultiChannel
(oracle/_ref through oracle.binding), and does the all-reduce in the parent:
rank k iterates on its own uniform stream (numpy, seed (seed, k)) with the
training deferred, the parent sums the training data and StatsData, and
every rank runs the reference's own Train on the sums.

Processes are started with the spawn method, so a parent that already uses
CUDA may create them.
"""
import multiprocessing as mp
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(conn, rank, spec):
    sys.path.insert(0, ROOT)
    from chili_b200 import abi, channels, workloads
    from oracle import binding
    cs = workloads.channel_set(spec["n_out"], spec.get("sqrts", 1000.0))
    params = workloads.mc_params(spec["ncalls_rank"], iterations=spec.get("iterations", 20))
    oracle = binding.REF if spec.get("oracle", "ref") == "ref" else binding.PORT
    R = binding.MultiChannel(cs, spec["bins"], params, getattr(abi, "CHILI_FUNC_" + spec["fkind"]),
                             channels.propagator_params(), pre=abi.CHILI_PRE_FINITE, oracle=oracle)
    if spec.get("cuts", True):
        R.set_cuts(cs.sqrts)
    R.set_defer(True)
    rng = np.random.default_rng((spec["seed"], rank))
    factor = 12.0
    conn.send(("ready", R.ndims))
    while True:
        msg = conn.recv()
        if msg[0] == "stop":
            break
        if msg[0] == "iterate":
            while True:
                rows = int(spec["ncalls_rank"] * factor) + 256
                u = workloads.uniforms53(rng, (rows, R.ndims + 1))
                t0 = time.perf_counter()
                try:
                    st, info = R.iterate(u, guard=True)
                except RuntimeError:
                    factor *= 2
                    continue
                dt = time.perf_counter() - t0
                break
            # rows for the next iteration: this one's rate with a margin
            factor = max(1.5, 1.3 * info.points_tried / spec["ncalls_rank"])
            hist, atrain = R.training()
            conn.send(("done", st.as_tuple(), hist, atrain, info.weight_max, info.points_tried, dt))
        elif msg[0] == "train":
            t0 = time.perf_counter()
            R.train(msg[1], msg[2])
            conn.send(("trained", time.perf_counter() - t0))
        elif msg[0] == "state":
            a, b, md = R.get_alpha()
            conn.send(("state", a, b, md, R.get_grids()))


class RefMPI:
    """`nranks` processes running the reference's MultiChannel in its MPI
    mode on one workload.  spec: n_out, bins, ncalls (per iteration, all
    ranks together), fkind, seed, cuts (the physical-region PreProcess)."""

    def __init__(self, nranks, n_out=4, bins=100, ncalls=1_000_000, fkind="PROPAGATOR", seed=7, cuts=True,
                 oracle="ref"):
        self.nranks = nranks
        self.ncalls_rank = ncalls // nranks  # MultiChannel.hh:209
        spec = dict(n_out=n_out, bins=bins, ncalls_rank=self.ncalls_rank, fkind=fkind, seed=seed, cuts=cuts,
                    oracle=oracle)
        ctx = mp.get_context("spawn")
        self.conns, self.procs = [], []
        for k in range(nranks):
            a, b = ctx.Pipe()
            p = ctx.Process(target=_rank_main, args=(b, k, spec), daemon=True)
            p.start()
            self.conns.append(a)
            self.procs.append(p)
        self.ndims = [c.recv() for c in self.conns][0][1]

    def iterate(self):
        """One MultiChannel::operator() of every rank, then the all-reduce
        and Train on every rank.  Returns (stats: the summed StatsData
        fields (n, min, max, sum, sum2, n_finite), weight_max over ranks,
        points tried, seconds: the slowest rank's iteration plus its Train,
        as an MPI job would take)."""
        for c in self.conns:
            c.send(("iterate",))
        res = [c.recv() for c in self.conns]
        st = np.array([r[1] for r in res])
        hist = sum(r[2] for r in res)
        atrain = sum(r[3] for r in res)
        for c in self.conns:
            c.send(("train", hist, atrain))
        tt = [c.recv()[1] for c in self.conns]
        stats = (st[:, 0].sum(), st[:, 1].min(), st[:, 2].max(), st[:, 3].sum(), st[:, 4].sum(), st[:, 5].sum())
        seconds = max(r[6] + t for r, t in zip(res, tt))
        return stats, max(r[4] for r in res), sum(r[5] for r in res), seconds

    def state(self, rank=0):
        self.conns[rank].send(("state",))
        _, a, b, md, grids = self.conns[rank].recv()
        return a, b, md, grids

    def close(self):
        for c in self.conns:
            try:
                c.send(("stop",))
            except (BrokenPipeError, OSError):
                pass
        for p in self.procs:
            p.join(timeout=10)
            if p.is_alive():
                p.terminate()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def _vegas_rank_main(conn, rank, spec):
    sys.path.insert(0, ROOT)
    from chili_b200 import workloads
    from oracle import binding
    dims, bins = spec["dims"], spec["bins"]
    params = np.asarray(workloads.camel_params(dims), dtype=np.float64)
    rng = np.random.default_rng((spec["seed"], rank))
    n = spec["ncalls_rank"]
    conn.send(("ready",))
    while True:
        msg = conn.recv()
        if msg[0] == "stop":
            break
        if msg[0] == "iterate":
            edges = msg[1]
            u = workloads.uniforms53(rng, (n, dims))
            t0 = time.perf_counter()
            st, train, _ = binding.vegas_iterate(edges, spec["alpha"], params, u, adapt=False)
            conn.send(("done", st.as_tuple(), train, time.perf_counter() - t0))


class RefVegasMPI:
    """The reference's Vegas::operator() (Vegas.cc:18-52) in its MPI mode on
    `nranks` host processes: every rank runs ncalls / size points (Vegas.cc:
    24-28) of the camel on its own uniform stream, the training histogram and
    StatsData are summed (Vegas.cc:44-47), and the reference's own
    AdaptiveMap::Adapt runs on the sum (Vegas.cc:49)."""

    def __init__(self, nranks, dims=4, bins=50, alpha=1.5, ncalls=100_000, seed=42):
        from oracle import binding
        self.binding = binding
        self.nranks, self.dims, self.bins, self.alpha = nranks, dims, bins, alpha
        self.ncalls_rank = ncalls // nranks
        self.edges = np.tile(np.arange(bins + 1, dtype=np.float64) / bins, (dims, 1))
        spec = dict(dims=dims, bins=bins, alpha=alpha, ncalls_rank=self.ncalls_rank, seed=seed)
        ctx = mp.get_context("spawn")
        self.conns, self.procs = [], []
        for k in range(nranks):
            a, b = ctx.Pipe()
            p = ctx.Process(target=_vegas_rank_main, args=(b, k, spec), daemon=True)
            p.start()
            self.conns.append(a)
            self.procs.append(p)
        for c in self.conns:
            c.recv()

    def iterate(self):
        """One iteration: (summed StatsData fields, seconds = the slowest
        rank's points plus the adaptation)."""
        for c in self.conns:
            c.send(("iterate", self.edges))
        res = [c.recv() for c in self.conns]
        st = np.array([r[1] for r in res])
        train = sum(r[2] for r in res)
        t0 = time.perf_counter()
        self.edges = self.binding.am_adapt(self.edges, self.alpha, train)
        t_adapt = time.perf_counter() - t0
        stats = (st[:, 0].sum(), st[:, 1].min(), st[:, 2].max(), st[:, 3].sum(), st[:, 4].sum(), st[:, 5].sum())
        return stats, max(r[3] for r in res) + t_adapt

    close = RefMPI.close
    __enter__ = RefMPI.__enter__
    __exit__ = RefMPI.__exit__
