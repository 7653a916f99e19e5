"""Workload presets: the integrands and settings the benchmarks run.

camel_params      the D-dim camel with unit integral (VEGAS workload)
MC_2TO4           2->4 propagator integrand, 15 channels, 100 bins, 1e6/iter
MC_2TO6           2->6, 45 channels, 200 bins, 1e7/iter
batched_tasks     512 uneven integrands for one batched launch
uniforms53        53-bit uniforms k*2^-53 (exactly representable in the
                  reference's generate_canonical, so both sides see them)
"""
import math

import numpy as np

from . import abi, channels


def camel_norm(dims, sigma, a, b):
    """N such that N * [exp(-|x-a|^2/s^2) + exp(-|x-b|^2/s^2)] integrates to 1
    over [0,1]^D: each Gaussian factorises into (sqrt(pi) s / 2)
    [erf((1-c)/s) + erf(c/s)] per dimension."""
    def g(c):
        return math.sqrt(math.pi) * sigma / 2 * (math.erf((1 - c) / sigma) + math.erf(c / sigma))
    ia = math.prod(g(c) for c in a)
    ib = math.prod(g(c) for c in b)
    return 1.0 / (ia + ib)


def camel_params(dims=4, sigma=0.1, a=None, b=None):
    a = [1 / 3] * dims if a is None else list(a)
    b = [2 / 3] * dims if b is None else list(b)
    return [sigma, camel_norm(dims, sigma, a, b)] + a + b


# The plain-VEGAS workload: 4-d camel, 50 bins, alpha 1.5, 10 x 1e5, seed 42.
VEGAS_CAMEL = dict(dims=4, bins=50, alpha=1.5, ncalls=100_000, iterations=10, seed=42)

# The multichannel workload: 2->4 at sqrt(S) = 1 TeV, 15 channels, 100 bins,
# 20 x 1e6 points, seed 7, alpha adapted every iteration, no grid refinement.
MC_2TO4 = dict(n_out=4, sqrts=1000.0, bins=100, ncalls=1_000_000, iterations=20, seed=7)
MC_2TO6 = dict(n_out=6, sqrts=1000.0, bins=200, ncalls=10_000_000, iterations=10, seed=7)


def mc_params(ncalls, iterations=20, **kw):
    """MultiChannelParams that run exactly `iterations` x `ncalls` without
    refinement (nrefine beyond the iteration count, rtol 0)."""
    return abi.MultiChannelParams.defaults(ncalls=ncalls, niterations=iterations, rtol=0.0,
                                           nrefine=iterations + 1, **kw)


def channel_set(n_out, sqrts=1000.0):
    if n_out == 4:
        return channels.multichannel_2_to_4(sqrts)
    if n_out == 6:
        return channels.multichannel_2_to_6(sqrts)
    return channels.multichannel_2_to_n(n_out, sqrts)


def uniforms53(rng, shape):
    """Uniforms k * 2^-53 in [0, 1)."""
    k = rng.integers(0, 2 ** 53, size=shape, dtype=np.uint64)
    return k.astype(np.float64) * 2.0 ** -53


def batched_tasks(seed=2024, n_camel=256, n_mc=256, camel_bins=50, mc_bins=50, scale=1.0):
    """The batched workload: n_camel camel functions of dimension 2..12
    (sigma uniform in [0.05, 0.2], centres uniform in [0.2, 0.8], grid alpha
    1.5) and n_mc 2->n propagator integrands (n = 2..5, sqrt(S) uniform in
    [200, 2000] GeV, M and Gamma of the Z, channel weights adapted), each with
    a point count log-uniform in [1e4, 1e6] (times `scale`, at least 100);
    task dicts for gpu.Context.batch_set."""
    rng = np.random.default_rng(seed)
    tasks = []
    sets = {}
    for _ in range(n_camel):
        dims = int(rng.integers(2, 13))
        sigma = float(rng.uniform(0.05, 0.2))
        a, b = rng.uniform(0.2, 0.8, dims), rng.uniform(0.2, 0.8, dims)
        tasks.append({"kind": "camel", "dims": dims, "bins": camel_bins, "grid_alpha": 1.5,
                      "ncalls": max(100, int(round(10 ** rng.uniform(4, 6) * scale))),
                      "params": camel_params(dims, sigma, a, b)})
    mp = abi.MultiChannelParams.defaults()
    for _ in range(n_mc):
        n_out = int(rng.integers(2, 6))
        sqrts = float(rng.uniform(200.0, 2000.0))
        key = (n_out, sqrts)
        if key not in sets:
            sets[key] = channel_set(n_out, sqrts)
        tasks.append({"kind": "multichannel", "channels": sets[key], "bins": mc_bins,
                      "ncalls": max(100, int(round(10 ** rng.uniform(4, 6) * scale))), "grid_alpha": mp.grid_alpha,
                      "beta": mp.beta, "min_alpha": mp.min_alpha, "fkind": abi.CHILI_FUNC_PROPAGATOR,
                      "params": channels.propagator_params(), "pre": abi.CHILI_PRE_FINITE})
    return tasks

