"""The reference's MPI mode as synchronized ranks (chili_b200/parallel.py),
on CPU with the gloo backend and world_size 2, the C oracle as each rank's
integrator: after every iteration all ranks hold identical grids and channel
weights, and they equal a single process that integrated both ranks' points
(the concatenated uniform streams)."""
import os
import socket

import numpy as np
import pytest

from chili_b200 import channels, workloads
from chili_b200 import abi

NCALLS = 3000
ITERS = 2
BINS = 50


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _PortRank:
    def __init__(self, rank):
        from oracle import port
        cs = channels.multichannel_2_to_4()
        self.params = workloads.mc_params(NCALLS)
        self.O = port.MultiChannel(cs, BINS, self.params, abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
        self.O.set_defer(True)
        self.rng = np.random.default_rng(100 + rank)
        self.used = []

    def run(self, params):
        u = workloads.uniforms53(self.rng, (NCALLS * 4, self.O.ndims + 1))
        st, info = self.O.iterate(u)
        self.used.append(u[:info.points_tried])
        return st.as_tuple(), info

    def training(self):
        return self.O.training()

    def train(self, params, hist, atrain):
        self.O.train(hist, atrain)


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    from chili_b200 import parallel
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r = _PortRank(rank)
        merged = []
        for _ in range(ITERS):
            st, info = parallel.synced_iteration(r, r.params)
            merged.append(st)
        a, b, md = r.O.get_alpha()
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), alpha=a, grids=r.O.get_grids(),
                 merged=np.array(merged), **{f"u{k}": u for k, u in enumerate(r.used)})
    finally:
        dist.destroy_process_group()


def test_two_ranks_match_one_process(tmp_path):
    import torch.multiprocessing as mp
    from oracle import port
    if not port.available():
        pytest.skip("C oracle not built")
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    r0, r1 = (np.load(tmp_path / f"rank{k}.npz") for k in range(2))
    # identical state on both ranks
    assert np.array_equal(r0["alpha"], r1["alpha"]) and np.array_equal(r0["grids"], r1["grids"])
    assert np.array_equal(r0["merged"], r1["merged"])
    # one process over both ranks' points, with its own training step
    cs = channels.multichannel_2_to_4()
    one = port.MultiChannel(cs, BINS, workloads.mc_params(2 * NCALLS), abi.CHILI_FUNC_PROPAGATOR,
                            channels.propagator_params())
    for k in range(ITERS):
        st, info = one.iterate(np.concatenate([r0[f"u{k}"], r1[f"u{k}"]]))
        m = r0["merged"][k]
        # iteration 0 starts from identical state; later ones from grids that
        # differ in the last bits (the summation order of the training data)
        tol = 1e-12 if k == 0 else 1e-9
        assert st.n == m[0] and st.n_finite == m[5]
        assert abs(st.sum - m[3]) <= tol * abs(st.sum) and abs(st.sum2 - m[4]) <= tol * abs(st.sum2)
        assert abs(st.max - m[2]) <= tol * abs(st.max) and abs(st.min - m[1]) <= tol * abs(st.min) + 1e-300
    a1, _, _ = one.get_alpha()
    assert np.allclose(a1, r0["alpha"], rtol=1e-10, atol=0)
    assert np.allclose(one.get_grids(), r0["grids"], rtol=1e-10, atol=1e-14)


def _worker_dies(rank, world, port, out_dir):
    """Rank 1 leaves after its first synchronized iteration, before the
    second one's collective (between steps, with nothing in flight); rank 0
    must learn of it from the process group (an error from its next
    all-reduce within the group's timeout), not hang."""
    import datetime
    import time
    import torch.distributed as dist
    from chili_b200 import parallel
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    r = _PortRank(rank)
    parallel.synced_iteration(r, r.params)
    if rank == 1:
        os._exit(0)  # leaves without destroying the group
    t0 = time.monotonic()
    outcome = "completed"
    try:
        parallel.synced_iteration(r, r.params)
    except Exception as e:  # gloo reports the lost peer or the timeout
        outcome = type(e).__name__
    with open(os.path.join(out_dir, "rank0.txt"), "w") as f:
        f.write(f"{outcome} {time.monotonic() - t0:.1f}")
    os._exit(0)


def test_a_rank_that_leaves_is_detected(tmp_path):
    import torch.multiprocessing as mp
    from oracle import port
    if not port.available():
        pytest.skip("C oracle not built")
    ctx = mp.start_processes(_worker_dies, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=False,
                             start_method="spawn")
    for p in ctx.processes:
        p.join(120)
    assert all(not p.is_alive() for p in ctx.processes)
    outcome, secs = (tmp_path / "rank0.txt").read_text().split()
    assert outcome != "completed" and float(secs) < 60
