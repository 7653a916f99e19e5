"""The reference's MPI mode on the library path (chili_b200/parallel.py):
two ranks, each a chili_b200 context on the same GPU with its own counter
range, exchange the packed training buffer in device memory
(chili_gpu_pack_training -> all-reduce of CUDA tensors -> the library
trains from device pointers into the summed buffer; MultiChannel.hh:184-212).
The group is gloo (one GPU here; NCCL needs one GPU per rank), so the
exchange itself stages through host memory inside the collective, not in
the library.  No kernel of one rank waits on the other: the ranks meet only
in the host-side collective between iterations.

After every iteration both ranks hold identical grids and channel weights,
and they equal one process that ran both counter ranges on one context
(training deferred), summed the two packed buffers and trained once: counts
exactly, sums, grids and channel weights to the rounding of the partial-sum
folds (each context chunks its points after its own acceptance history)."""
import os
import socket

import numpy as np
import pytest

from chili_b200 import abi, channels, workloads

pytestmark = pytest.mark.gpu

NCALLS = 50_000
ITERS = 3
BINS = 100
COUNTER0 = [0, 1 << 40]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _context():
    from chili_b200 import gpu
    cs = workloads.channel_set(4)
    ctx = gpu.Context(0)
    ctx.set_channels(cs)
    ctx.uniform_grids(cs.nch, ctx.ndims, BINS)
    ctx.set_integrand(abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    ctx.set_preprocess_cuts(cs.sqrts)
    return ctx


def _worker(rank, world, port, out_dir):
    import datetime

    import torch
    import torch.distributed as dist

    from chili_b200 import parallel
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        torch.cuda.set_device(0)
        ctx = _context()
        r = parallel.GpuRank(ctx, seed=7, counter=COUNTER0[rank])
        params = workloads.mc_params(NCALLS)
        merged = []
        for _ in range(ITERS):
            st, info = parallel.synced_iteration(r, params, device=torch.device("cuda", 0))
            merged.append(st)
        a, b, md = ctx.get_alpha()
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), alpha=a, best=b, grids=ctx.get_grids(),
                 merged=np.array(merged))
        ctx.close()
    finally:
        dist.destroy_process_group()


def test_two_library_ranks_equal_one_process(tmp_path):
    import torch
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    r0, r1 = (np.load(tmp_path / f"rank{k}.npz") for k in range(2))
    assert np.array_equal(r0["alpha"], r1["alpha"]) and np.array_equal(r0["grids"], r1["grids"])
    assert np.array_equal(r0["merged"], r1["merged"])

    # one process, one context, both counter ranges
    ctx = _context()
    ctx.set_option("defer_train", 1)
    params = workloads.mc_params(NCALLS)
    counters = list(COUNTER0)
    n = ctx.packed_training_len()
    for k in range(ITERS):
        bufs = []
        for q in range(2):
            st, info = ctx.multichannel_iterate(params, seed=7, counter=counters[q])
            counters[q] += info.points_tried
            buf = torch.empty(n, dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            bufs.append(ctx.pack_training(buf))
            ctx.synchronize()
        tot = bufs[0] + bufs[1]
        nh = n - 6 - ctx.nch
        h, a = tot[:nh].contiguous(), tot[nh:nh + ctx.nch].contiguous()
        torch.cuda.synchronize()
        ctx.multichannel_train(params, h, a)
        ctx.synchronize()
        s = tot.cpu().numpy()
        m = r0["merged"][k]
        # counts exact; the sums agree to the order of the partial-sum folds
        # (the chunking follows each context's own acceptance history)
        assert m[0] == s[nh + ctx.nch]
        assert abs(m[3] - s[nh + ctx.nch + 1]) <= 1e-12 * abs(m[3])
        assert abs(m[4] - s[nh + ctx.nch + 2]) <= 1e-12 * abs(m[4])
    a, b, md = ctx.get_alpha()
    assert np.allclose(a, r0["alpha"], rtol=1e-10, atol=0) and np.allclose(b, r0["best"], rtol=1e-10, atol=0)
    assert np.allclose(ctx.get_grids(), r0["grids"], rtol=1e-10, atol=1e-14)
    ctx.close()
