"""End-to-end checks of the benchmark workloads on the GPU, seeded and with the
on-device generator: the GPU iteration run on the counter-based uniforms
reproduces the C oracle run on the same uniforms regenerated on the host, and
the 2->6 workload matches the oracle as well."""
import numpy as np
import pytest

from chili_b200 import abi, channels, workloads
from oracle import port

pytestmark = pytest.mark.gpu


def _close(a, b, tol):
    return abs(a - b) <= tol * max(abs(b), 1e-300)


# (6, 200): the large workload's grids, whose per-channel bin-search tables
# (75 KB) take the 512-thread variant of the channel kernel
@pytest.mark.parametrize("n_out,nch_bins,ncalls", [(4, 100, 30_000), (6, 50, 10_000), (6, 200, 10_000)])
def test_philox_iteration_matches_oracle(ctx_factory, n_out, nch_bins, ncalls):
    cs = workloads.channel_set(n_out)
    ctx = ctx_factory()
    ctx.set_channels(cs)
    ctx.uniform_grids(cs.nch, ctx.ndims, nch_bins)
    kind = abi.CHILI_FUNC_PROPAGATOR if n_out == 4 else abi.CHILI_FUNC_PROPAGATOR_TOP2
    ctx.set_integrand(kind, channels.propagator_params())
    ctx.set_preprocess(abi.CHILI_PRE_FINITE)
    params = workloads.mc_params(ncalls)
    O = port.MultiChannel(cs, nch_bins, params, kind, channels.propagator_params())
    seed, counter = 11, 0
    for it in range(3):
        st, info = ctx.multichannel_iterate(params, seed=seed, counter=counter)
        u = port.philox_uniforms(seed, counter, info.points_tried, ctx.ndims + 1)
        st_o, info_o = O.iterate(u)
        assert info_o.points_tried == info.points_tried, it
        assert st.n == st_o.n and st.n_finite == st_o.n_finite
        assert _close(st.sum, st_o.sum, 1e-11) and _close(st.sum2, st_o.sum2, 1e-11)
        a = ctx.get_alpha()[0]
        a_o = O.get_alpha()[0]
        assert np.max(np.abs(a - a_o) / a_o) < 1e-11
        # continue from the oracle's state so that rounding cannot accumulate
        ctx.set_grids(O.get_grids())
        ctx.set_alpha(a_o)
        counter += info.points_tried


def test_launch_count_and_determinism(ctx_factory):
    cs = workloads.channel_set(4)
    res = []
    for _ in range(2):
        ctx = ctx_factory()
        ctx.set_channels(cs)
        ctx.uniform_grids(cs.nch, ctx.ndims, 100)
        ctx.set_integrand(abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
        ctx.set_preprocess(abi.CHILI_PRE_FINITE)
        l0 = ctx.launches
        st, info = ctx.multichannel_iterate(workloads.mc_params(50_000), seed=3)
        assert ctx.launches - l0 >= 10
        res.append((st.as_tuple(), info.points_tried, ctx.get_alpha()[0].tolist()))
    assert res[0][1] == res[1][1]
    assert res[0][0][0] == res[1][0][0]
    assert _close(res[0][0][3], res[1][0][3], 1e-13)


def test_cut_preprocess_iteration_matches_oracle(ctx_factory):
    """CHILI_PRE_CUTS on the GPU: the same rejections, StatsData and alpha as
    the C oracle on the same counter-based uniforms."""
    cs = workloads.channel_set(4)
    ctx = ctx_factory()
    ctx.set_channels(cs)
    ctx.uniform_grids(cs.nch, ctx.ndims, 100)
    ctx.set_integrand(abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    ctx.set_preprocess_cuts(1000.0)
    params = workloads.mc_params(20_000)
    O = port.MultiChannel(cs, 100, params, abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    O.set_cuts(1000.0)
    seed, counter = 13, 0
    for it in range(2):
        st, info = ctx.multichannel_iterate(params, seed=seed, counter=counter)
        u = port.philox_uniforms(seed, counter, info.points_tried, ctx.ndims + 1)
        st_o, info_o = O.iterate(u)
        assert info_o.points_tried == info.points_tried and info_o.rejected_pre == info.rejected_pre, it
        assert st.n == st_o.n and st.n_finite == st_o.n_finite
        assert _close(st.sum, st_o.sum, 1e-11) and _close(st.sum2, st_o.sum2, 1e-11)
        ctx.set_grids(O.get_grids())
        ctx.set_alpha(O.get_alpha()[0])
        counter += info.points_tried


def test_deferred_train_equals_the_iteration_training(ctx_factory):
    """defer_train + get_training + multichannel_train (the per-rank steps of
    the MPI mode, here with one rank) leave the same grids and channel weights
    as an iteration that trains itself."""
    cs = workloads.channel_set(4)
    res = []
    for defer in (False, True):
        ctx = ctx_factory()
        ctx.set_channels(cs)
        ctx.uniform_grids(cs.nch, ctx.ndims, 100)
        ctx.set_integrand(abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
        ctx.set_preprocess(abi.CHILI_PRE_FINITE)
        params = workloads.mc_params(50_000)
        if defer:
            ctx.set_option("defer_train", 1)
        counter = 0
        for it in range(2):
            st, info = ctx.multichannel_iterate(params, seed=17, counter=counter)
            counter += info.points_tried
            if defer:
                h, a = ctx.get_training()
                ctx.multichannel_train(params, h, a)
        res.append((ctx.get_grids(), ctx.get_alpha()[0], st.as_tuple()))
    # the histograms are summed with atomics (order varies in the last bits
    # between runs), so the adapted grids of the first iteration, and with
    # them the points of the second, agree to rounding only
    assert np.allclose(res[0][0], res[1][0], rtol=1e-12, atol=1e-15)
    assert np.allclose(res[0][1], res[1][1], rtol=1e-10, atol=0)
    st0, st1 = res[0][2], res[1][2]
    assert st0[0] == st1[0] and st0[5] == st1[5]
    assert _close(st0[3], st1[3], 1e-10) and _close(st0[4], st1[4], 1e-10)


def test_optimize_writes_one_json_line_per_iteration(ctx_factory):
    """gpu.optimize: MultiChannel::Optimize's loop with a JSON-lines log of
    every iteration; stops at niterations (rtol 0) and pools the iterations."""
    import io
    import json
    from chili_b200 import gpu
    cs = workloads.channel_set(4)
    ctx = ctx_factory()
    ctx.set_channels(cs)
    ctx.uniform_grids(cs.nch, ctx.ndims, 50)
    ctx.set_integrand(abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    ctx.set_preprocess_cuts(cs.sqrts)
    buf = io.StringIO()
    mean, err, recs = gpu.optimize(ctx, workloads.mc_params(20_000, iterations=3), seed=5, log=buf)
    lines = [json.loads(x) for x in buf.getvalue().splitlines()]
    assert [r["iteration"] for r in lines] == [0, 1, 2] and len(recs) == 3
    assert all(r["n"] >= 20_000 and r["w_max"] > 0 and 0 < r["unweighting_efficiency"] < 1 for r in lines)
    assert lines[-1]["pooled"] == mean and mean > 0 and 0 < err < mean


# (1, 500_000): chunks of more slices
@pytest.mark.parametrize("pipeline,ncalls", [(1, 200_000), (0, 200_000), (1, 500_000)])
def test_host_uniforms_in_slices_match_device_uniforms(ctx_factory, pipeline, ncalls):
    """Host uniforms (pinned) are uploaded in slices (2^16, 2^17, 2^18, then
    2^19 rows) and each slice is mapped and weighted as its own queued round; the same uniforms in
    device memory are read in place in one round.  Both take the same points
    (counts exact) and agree to the rounding of the partial-sum folds, over
    two adapting iterations with the physical-region cuts (the first one on
    uniform grids outgrows its predicted upload and needs a second one).
    The first iteration's largest weight agrees bit for bit.  Both weight
    passes: the phased one and the fused per-point one (pipeline 0)."""
    import torch
    cs = workloads.channel_set(4)
    ctxs = []
    for _ in range(2):
        ctx = ctx_factory()
        ctx.set_channels(cs)
        ctx.uniform_grids(cs.nch, ctx.ndims, 100)
        ctx.set_integrand(abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
        ctx.set_preprocess_cuts(1000.0)
        ctx.set_option("pipeline", pipeline)
        ctxs.append(ctx)
    params = workloads.mc_params(ncalls)
    if ncalls > 200_000:
        # adapted grids first (uniform grids accept too few points under the
        # cuts for the uniforms below), the same on both contexts
        ctxs[0].multichannel_iterate(params, seed=3)
        ctxs[1].set_grids(ctxs[0].get_grids())
        ctxs[1].set_alpha(ctxs[0].get_alpha()[0])
    rng = np.random.default_rng(29)
    for it in range(2):
        n_u = 2_500_000 if ncalls <= 200_000 else 4_000_000
        host = torch.empty((n_u, ctxs[0].ndims + 1), dtype=torch.float64, pin_memory=True)
        host.numpy()[:] = workloads.uniforms53(rng, tuple(host.shape))
        dev = host.to("cuda")
        st_h, info_h = ctxs[0].multichannel_iterate(params, u=host.numpy(), guard=True)
        st_d, info_d = ctxs[1].multichannel_iterate(params, u=dev, guard=True)
        assert info_h.points_tried == info_d.points_tried > (1 << 18), it
        assert info_h.rejected_pre == info_d.rejected_pre
        assert st_h.n == st_d.n and st_h.n_finite == st_d.n_finite
        assert _close(st_h.sum, st_d.sum, 1e-12) and _close(st_h.sum2, st_d.sum2, 1e-12)
        # the first iteration runs on identical grids (largest weight bit for
        # bit); the second on grids adapted from atomically summed histograms
        tol = 0 if it == 0 else 1e-12
        assert _close(st_h.min, st_d.min, tol) and _close(st_h.max, st_d.max, tol), it
        assert np.allclose(ctxs[0].get_alpha()[0], ctxs[1].get_alpha()[0], rtol=1e-10, atol=0)
        assert np.allclose(ctxs[0].get_grids(), ctxs[1].get_grids(), rtol=1e-10, atol=1e-15)
