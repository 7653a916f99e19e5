"""chili_gpu_vegas_iterate_noalloc, the entry point for callers that cannot
call cudaMalloc (their device memory belongs to another framework's allocator,
or their memory budget is fixed in advance): called through the C ABI on
caller-owned device buffers, its StatsData and training histogram match those
of chili_gpu_vegas_iterate on the same grid, integrand and uniforms, on two
calls in a row (the second call finds the first call's leftovers in the shared
scratch array).  Collected last, so that a run stopping at the first failure
has already run every other test."""
import ctypes as C

import numpy as np
import pytest

from chili_b200 import abi, gpu, workloads

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def test_noalloc_vegas_matches_the_context_entry_point():
    import torch

    lib = gpu.load()
    dims, bins, n, seed = 4, 50, 200_000, 5
    rng = np.random.default_rng(77)
    inner = np.sort(rng.random((dims, bins - 1)), axis=1)
    edges = np.concatenate([np.zeros((dims, 1)), inner, np.ones((dims, 1))], axis=1)
    params = np.array(workloads.camel_params(dims), dtype=np.float64)

    ctx = gpu.Context(0)
    ctx.set_grids(edges[None])
    ctx.set_integrand(abi.CHILI_FUNC_CAMEL, params)

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    edges_d = torch.tensor(edges, dtype=torch.float64, device=dev).contiguous()
    stats_d = torch.empty(6, dtype=torch.float64, device=dev)
    train_d = torch.empty(dims * bins, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        counter = call * n
        st, tr = ctx.vegas_iterate(n, seed=seed, counter=counter, alpha=1.5, adapt=False, train=True)
        rc = lib.chili_gpu_vegas_iterate_noalloc(C.c_void_p(stream), C.c_void_p(edges_d.data_ptr()), dims, bins,
                                                 params.ctypes.data_as(C.c_void_p), params.size, n, seed, counter,
                                                 C.c_void_p(stats_d.data_ptr()), C.c_void_p(train_d.data_ptr()))
        assert rc == abi.CHILI_OK, lib.chili_gpu_last_error(None)
        torch.cuda.synchronize(dev)
        got = stats_d.cpu().numpy()
        want = np.array(st.as_tuple())
        assert got[0] == want[0] and got[5] == want[5]          # n, n_finite
        assert np.allclose(got[1:5], want[1:5], rtol=RTOL, atol=0)  # min, max, sum, sum2
        assert np.allclose(train_d.cpu().numpy(), tr, rtol=RTOL, atol=0)
    ctx.close()


def test_noalloc_rejects_sizes_beyond_its_limits():
    import torch

    lib = gpu.load()
    dev = torch.device("cuda", 0)
    buf = torch.zeros(64, dtype=torch.float64, device=dev)
    params = np.zeros(2 + 2 * 40)
    p = C.c_void_p(buf.data_ptr())
    rc = lib.chili_gpu_vegas_iterate_noalloc(None, p, 40, 50, params.ctypes.data_as(C.c_void_p), params.size,
                                             1000, 1, 0, p, p)
    assert rc == abi.CHILI_ERR_LIMIT
    host = np.zeros(64)
    rc = lib.chili_gpu_vegas_iterate_noalloc(None, host.ctypes.data_as(C.c_void_p), 4, 2,
                                             params.ctypes.data_as(C.c_void_p), 10, 1000, 1, 0, p, p)
    assert rc == abi.CHILI_ERR_INVALID_ARG
