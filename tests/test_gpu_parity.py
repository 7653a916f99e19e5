"""Parity of the CUDA path (called through the C ABI) with the reference's own
CPU code (oracle/_ref, the unmodified Chili sources) on identical inputs.

Bars: grid map, Jacobian, FindBin and channel selection bit-exact; FP64
momenta, weights and accumulated sums within 1e-12 relative at the 99th
percentile (the reference's libm and CUDA's differ by an ulp; see the tail
checks below).
"""
import numpy as np
import pytest

from chili_b200 import abi, channels, workloads
from chili_b200.workloads import uniforms53
from oracle import port, ref

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def rel(a, b):
    a, b = np.atleast_1d(np.asarray(a, dtype=np.float64)), np.atleast_1d(np.asarray(b, dtype=np.float64))
    d = np.abs(a - b)
    s = np.maximum(np.abs(b), 1e-300)
    out = d / s
    out[(a == b) | (np.isnan(a) & np.isnan(b))] = 0.0
    return out


def random_grid(rng, dims, bins):
    """A non-uniform monotone grid with edges 0 and 1."""
    e = np.sort(rng.random((dims, bins - 1)), axis=1)
    return np.concatenate([np.zeros((dims, 1)), e, np.ones((dims, 1))], axis=1)


@pytest.fixture(scope="module")
def rng():
    return np.random.default_rng(20261203)


def test_grid_map_and_weight_bit_exact(ctx_factory, rng):
    ctx = ctx_factory()
    dims, bins = 4, 50
    edges = random_grid(rng, dims, bins)
    ctx.set_grids(edges[None])
    u = uniforms53(rng, (200_000, dims))
    u[:5] = 0.0  # x == 0 exactly: FindBin returns SIZE_MAX in the reference
    x, jac = ctx.grid_map(0, u)
    xr, jr = ref.am_map(edges, u)
    assert np.array_equal(x, xr)
    assert np.array_equal(jac, jr)
    # points on edges and between them
    on_edges = edges[:, 1:bins].T.copy()  # every interior edge, exactly
    xe = np.concatenate([x, on_edges, np.zeros((1, dims)), np.ones((1, dims))])
    w, b = ctx.grid_weight(0, xe)
    wr, br = ref.am_weight(edges, xe)
    assert np.array_equal(b, br)
    ok = ~np.isnan(wr)  # the reference reads outside its table there
    assert np.array_equal(w[ok], wr[ok])
    # tables the hinted search must not shortcut: not monotone, with a NaN, all
    # zero; and a peaked one (many edges per hint cell)
    bad = edges.copy()
    bad[0, 10:20] = bad[0, 10:20][::-1].copy()
    bad[1, 25] = np.nan
    bad[2, :] = 0.0
    bad[3, 1:bins] = np.sort(0.5 + 1e-4 * rng.random(bins - 1))
    ctx.set_grids(bad[None])
    xs = np.concatenate([uniforms53(rng, (100_000, dims)), bad[:, 1:bins].T, np.zeros((1, dims))])
    w, b = ctx.grid_weight(0, xs)
    wr, br = ref.am_weight(bad, xs)
    assert np.array_equal(b, br)
    ok = ~np.isnan(wr)
    assert np.array_equal(w[ok], wr[ok], equal_nan=True)


def test_grid_adapt_and_split(ctx_factory, rng):
    ctx = ctx_factory()
    dims, bins = 6, 100
    edges = random_grid(rng, dims, bins)
    train = rng.random(dims * bins) ** 4
    train[bins:2 * bins] = 0.0  # an all-zero dimension: the reference zeroes its edges
    train[2 * bins + 7] = 0.0
    ctx.set_grids(edges[None])
    ctx.grid_adapt(0, 1.5, train)
    got = ctx.get_grids()[0]
    want = ref.am_adapt(edges, 1.5, train)
    assert np.max(rel(got, want)) < RTOL
    assert np.all(got[1] == 0.0)
    for nsplit in (2, 3, 4):
        ctx.set_grids(edges[None])
        ctx.grid_split(nsplit)
        assert np.array_equal(ctx.get_grids()[0], ref.am_split(edges, nsplit))


def test_vegas_iteration_matches_reference(ctx_factory, rng):
    ctx = ctx_factory()
    p = workloads.camel_params()
    dims, bins = 4, 50
    edges = random_grid(rng, dims, bins)
    ctx.set_grids(edges[None])
    ctx.set_integrand(abi.CHILI_FUNC_CAMEL, p)
    u = uniforms53(rng, (100_000, dims))
    st, tr = ctx.vegas_iterate(len(u), u=u, alpha=1.5, adapt=True, train=True)
    st_r, tr_r, e_r = ref.vegas_iterate(edges, 1.5, p, u, adapt=True)
    assert st.n == st_r.n and st.n_finite == st_r.n_finite
    assert rel(st.min, st_r.min) < RTOL and rel(st.max, st_r.max) < RTOL
    assert rel(st.sum, st_r.sum) < 1e-12 and rel(st.sum2, st_r.sum2) < 1e-12
    assert np.max(rel(tr, tr_r)) < 1e-12
    assert np.max(rel(ctx.get_grids()[0], e_r)) < 1e-11


@pytest.mark.parametrize("ppt", [1, 2, 4])
@pytest.mark.parametrize("dims,bins,n", [(4, 50, 200_003), (7, 100, 4_097), (1, 2, 5), (9, 30, 1_537)])
def test_vegas_generate_matches_reference(ctx_factory, rng, dims, bins, n, ppt):
    """Materialised VEGAS points: the device generator's uniforms (counter
    stream regenerated by the C port) through the reference's own
    AdaptiveMap::operator() give x bit for bit; the weight f(x) J within
    1e-12 (CUDA's exp against numpy's).  Sizes that are not a multiple of
    the tile (256 points per thread slot), odd row lengths, a one-bin-pair
    grid, a dimension without a compile-time kernel (9), and 1, 2 or 4
    points per thread."""
    from oracle import port
    ctx = ctx_factory()
    ctx.set_option("vegas_gen_ppt", ppt)
    p = workloads.camel_params(dims)
    edges = random_grid(rng, dims, bins)
    ctx.set_grids(edges[None])
    ctx.set_integrand(abi.CHILI_FUNC_CAMEL, p)
    seed, ctr = 42, 12345
    x, w = ctx.vegas_generate(n, seed=seed, counter=ctr)
    u = port.philox_uniforms(seed, ctr, n, dims)
    x_r, jac_r = ref.am_map(edges, u)
    assert np.array_equal(x, x_r)
    a, b = np.asarray(p[2:2 + dims]), np.asarray(p[2 + dims:2 + 2 * dims])
    s2 = p[0] * p[0]
    f = p[1] * (np.exp(-np.sum((x_r - a) ** 2, axis=1) / s2) + np.exp(-np.sum((x_r - b) ** 2, axis=1) / s2))
    assert np.max(rel(w, f * jac_r)) < 1e-12


def test_vegas_camel_converges(ctx_factory):
    ctx = ctx_factory()
    cfg = workloads.VEGAS_CAMEL
    ctx.uniform_grids(1, cfg["dims"], cfg["bins"])
    ctx.set_integrand(abi.CHILI_FUNC_CAMEL, workloads.camel_params(cfg["dims"]))
    tot = np.zeros(6)
    for it in range(cfg["iterations"]):
        st = ctx.vegas_iterate(cfg["ncalls"], seed=cfg["seed"], counter=it * cfg["ncalls"], alpha=cfg["alpha"])
        tot[0] += st.n
        tot[3] += st.sum
        tot[4] += st.sum2
    from chili_b200.gpu import stats_mean_error
    mean, err = stats_mean_error(tot)
    assert abs(mean - 1.0) < 4 * err, (mean, err)
    assert err / mean < 0.01


@pytest.fixture(scope="module")
def mc2():
    cs = channels.multichannel_2_to_4()
    return cs


def test_fsmapper_forward_and_inverse(ctx_factory, rng, mc2):
    ctx = ctx_factory()
    ctx.set_channels(mc2)
    ctx.set_integrand(abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    R = ref.MultiChannel(mc2, 100, workloads.mc_params(1000))
    n = 20_000
    worst = []
    for ch in range(mc2.nch):
        x = uniforms53(rng, (n, ctx.ndims))
        mom = ctx.fsmapper_generate(ch, x)
        mom_r = R.fsm_generate(ch, x)
        nan_g = np.isnan(mom).any(axis=(1, 2))
        nan_r = np.isnan(mom_r).any(axis=(1, 2))
        assert np.mean(nan_g != nan_r) < 1e-3
        ok = ~(nan_g | nan_r)
        scale = np.abs(mom_r[ok][:, :, :1])
        d = np.abs(mom[ok] - mom_r[ok]) / np.maximum(scale, 1e-300)
        worst.append(np.percentile(d.max(axis=(1, 2)), 99))
        assert np.percentile(d.max(axis=(1, 2)), 99) < RTOL, (ch, np.percentile(d, 99))
        # inverse on the reference's momenta
        w, xi = ctx.fsmapper_weight(ch, mom_r[ok])
        w_r, xi_r = R.fsm_weight(ch, mom_r[ok])
        fin = np.isfinite(w_r) & (w_r != 0)
        assert np.percentile(rel(w[fin], w_r[fin]), 99) < RTOL, ch
        assert np.mean((w == 0) != (w_r == 0)) < 1e-3
        # round trip of the channel's own points
        back = xi_r[fin]
        assert np.percentile(np.abs(back - x[ok][fin]), 99) < 1e-6


def test_channel_selection_bit_exact(ctx_factory, rng, mc2):
    ctx = ctx_factory()
    ctx.set_channels(mc2)
    alpha = rng.random(mc2.nch) ** 3
    alpha[3] = 0.0
    ctx.set_alpha(alpha)
    v = uniforms53(rng, 300_000)
    assert np.array_equal(ctx.select_channel(v), ref.select(alpha, v))


def _mc_pair(ctx_factory, cs, bins, ncalls, rng):
    ctx = ctx_factory()
    ctx.set_channels(cs)
    params = workloads.mc_params(ncalls)
    R = ref.MultiChannel(cs, bins, params, abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    ctx.set_integrand(abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    ctx.set_preprocess(abi.CHILI_PRE_FINITE)
    edges = np.stack([random_grid(rng, R.ndims, bins) for _ in range(cs.nch)])
    ctx.set_grids(edges)
    R.set_grids(edges)
    return ctx, R, params


@pytest.mark.parametrize("point_program", [1, 0])
def test_combined_weight(ctx_factory, rng, mc2, point_program):
    ctx, R, _ = _mc_pair(ctx_factory, mc2, 100, 1000, rng)
    ctx.set_option("point_program", point_program)
    alpha = rng.random(mc2.nch) + 0.1
    alpha /= alpha.sum()
    ctx.set_alpha(alpha)
    R.set_alpha(alpha)
    n = 20_000
    ich = rng.integers(0, mc2.nch, n).astype(np.int32)
    x = uniforms53(rng, (n, R.ndims))
    mom = np.concatenate([R.fsm_generate(c, x[ich == c]) for c in range(mc2.nch)])
    ich = np.concatenate([ich[ich == c] for c in range(mc2.nch)])
    ok = ~np.isnan(mom).any(axis=(1, 2))
    mom, ich = mom[ok], ich[ok]
    w, dens, xs = ctx.multichannel_weight(mom, ich)
    w_r, dens_r, xs_r = R.weight(mom, ich)
    fin = np.isfinite(w_r) & np.isfinite(w)
    assert np.mean(np.isfinite(w_r) != np.isfinite(w)) < 2e-4
    assert np.percentile(rel(w[fin], w_r[fin]), 99) < RTOL
    df = np.isfinite(dens_r) & (dens_r != 0)
    assert np.percentile(rel(dens[df], dens_r[df]), 99) < RTOL


WEIGHT_PATHS = {"pipeline": dict(point_program=1, pipeline=1),
                "pipeline_fused_combine": dict(point_program=1, pipeline=1, pipeline_fuse=1),
                "pipeline_global_tables": dict(point_program=1, pipeline=1, channel_tables=0),
                "fused_point_program": dict(point_program=1, pipeline=0),
                "per_channel": dict(point_program=0, pipeline=0)}


@pytest.mark.parametrize("path", list(WEIGHT_PATHS))
def test_multichannel_iteration_matches_reference(ctx_factory, rng, mc2, path):
    ncalls = 20_000
    ctx, R, params = _mc_pair(ctx_factory, mc2, 100, ncalls, rng)
    for k, v in WEIGHT_PATHS[path].items():
        ctx.set_option(k, v)
    for it in range(3):
        u = uniforms53(rng, (3 * ncalls, R.ndims + 1))
        st, info = ctx.multichannel_iterate(params, u=u, guard=True)
        st_r, info_r = R.iterate(u, guard=True)
        assert info.points_tried == info_r.points_tried, (it, info.points_tried, info_r.points_tried)
        assert info.rejected_pre == info_r.rejected_pre
        assert info.rejected_nan == info_r.rejected_nan
        assert st.n == st_r.n and st.n_finite == st_r.n_finite
        assert rel(st.sum, st_r.sum) < 1e-11 and rel(st.sum2, st_r.sum2) < 1e-11
        assert rel(st.max, st_r.max) < RTOL
        a, b, md = ctx.get_alpha()
        a_r, b_r, md_r = R.get_alpha()
        assert np.max(rel(a, a_r)) < 1e-11
        # MaxDifference (MultiChannel.cc:138-154): the largest pairwise gap of
        # the alpha-training sums, and the adapted weights saved whenever it
        # is the smallest so far
        assert np.isfinite(md) and md_r < 1.7e308, (md, md_r)
        assert rel(md, md_r)[0] < 1e-10, (md, md_r)
        assert np.max(rel(b, b_r)) < 1e-11, (b, b_r)
        g, g_r = ctx.get_grids(), R.get_grids()
        assert np.max(np.abs(g - g_r)) < 1e-10
        # continue both from identical state so later iterations stay comparable
        ctx.set_grids(g_r)
        ctx.set_alpha(a_r)


def test_evaluate_batch(ctx_factory, rng, mc2):
    ctx, R, _ = _mc_pair(ctx_factory, mc2, 100, 1000, rng)
    for ch in (0, 7, 12):
        u = uniforms53(rng, (20_000, R.ndims))
        out = ctx.evaluate_batch(ch, u)
        out_r = R.evaluate_batch(ch, u)
        fin = np.isfinite(out_r)
        assert np.mean((out == 0) != (out_r == 0)) < 1e-3
        nz = fin & (out_r != 0) & (out != 0)
        assert np.percentile(rel(out[nz], out_r[nz]), 99) < RTOL


def test_generate_events(ctx_factory, mc2):
    ctx = ctx_factory()
    ctx.set_channels(mc2)
    ctx.uniform_grids(mc2.nch, ctx.ndims, 100)
    ctx.set_integrand(abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    mom, w, ch = ctx.generate(100_000, seed=3)
    assert np.all(np.isfinite(w))
    counts = np.bincount(ch, minlength=mc2.nch) / len(ch)
    assert np.allclose(counts, 1 / mc2.nch, atol=0.01)
    ok = ~np.isnan(mom).any(axis=(1, 2))
    tot = mom[ok].sum(axis=1)
    assert np.max(np.abs(tot)) < 1e-9 * 1000  # momentum conservation (all-outgoing)


def test_multichannel_iteration_degenerate_grids(ctx_factory, rng, mc2):
    """Edge tables that are not monotone or hold a NaN (the hinted bin search
    must fall back to the plain lower_bound) give the reference's results.
    (An all-zero table, which the reference's Adapt leaves for a dimension
    without data, makes every point's combined weight a sum of signed
    infinities whose NaN-or-not outcome hinges on the signs of zero densities,
    i.e. on last-ulp differences between the two libms; it is checked at the
    level of the bin search in test_grid_map_and_weight_bit_exact instead.)"""
    ncalls = 10_000
    ctx, R, params = _mc_pair(ctx_factory, mc2, 100, ncalls, rng)
    edges = R.get_grids()
    edges[3, 2, 10:20] = edges[3, 2, 10:20][::-1].copy()  # non-monotone
    edges[8, 0, 50] = np.nan                                # NaN edge
    ctx.set_grids(edges)
    R.set_grids(edges)
    u = uniforms53(rng, (12 * ncalls, R.ndims + 1))
    st, info = ctx.multichannel_iterate(params, u=u, guard=True)
    st_r, info_r = R.iterate(u, guard=True)
    assert info.points_tried == info_r.points_tried
    assert st.n == st_r.n and st.n_finite == st_r.n_finite
    assert rel(st.sum, st_r.sum) < 1e-11


def test_constructed_channels_iterate_like_the_reference(ctx_factory, rng):
    """A channel set from the library's ConstructChannels (gluon 2->4, smax 2:
    14 channels with massless s-channel decays) on the GPU against the
    reference's MultiChannel built from the same descriptions: combined
    weights per point within 1e-12 at p99, and an iteration on the same
    uniforms with the same counts, the sum within 5e-9 and the sum of
    squares within 2e-8: the largest weights dominate them, and near the
    nested decays' thresholds they amplify the last-ulp differences between
    CUDA's and glibc's pow / atan / log.  (Without the product-by-product
    rounding of the phase-space arithmetic the weights drifted by ~1e-9.)"""
    from chili_b200 import gpu
    flavs = [21] * 6
    cs = gpu.construct_channels(flavs, {(21, 21): [21]}, {21: 0.0}, {21: 0.0}, 1000.0, smax=2)
    assert cs.nch == 14
    ncalls = 20_000
    ctx, R, params = _mc_pair(ctx_factory, cs, 50, ncalls, rng)
    n = 20_000
    ich = rng.integers(0, cs.nch, n).astype(np.int32)
    x = uniforms53(rng, (n, R.ndims))
    mom = np.concatenate([R.fsm_generate(c, x[ich == c]) for c in range(cs.nch)])
    ich = np.concatenate([ich[ich == c] for c in range(cs.nch)])
    ok = ~np.isnan(mom).any(axis=(1, 2))
    w, _, _ = ctx.multichannel_weight(mom[ok], ich[ok])
    w_r, _, _ = R.weight(mom[ok], ich[ok])
    fin = np.isfinite(w_r) & np.isfinite(w)
    assert np.mean(np.isfinite(w_r) != np.isfinite(w)) < 2e-4
    assert np.percentile(rel(w[fin], w_r[fin]), 99) < RTOL
    u = uniforms53(rng, (4 * ncalls, R.ndims + 1))
    st, info = ctx.multichannel_iterate(params, u=u, guard=True)
    st_r, info_r = R.iterate(u, guard=True)
    assert info.points_tried == info_r.points_tried and info.rejected_pre == info_r.rejected_pre
    assert st.n == st_r.n and st.n_finite == st_r.n_finite
    # the sum of 2e4 values is dominated by its largest weights, and near the
    # nested decays' thresholds those amplify last-ulp libm differences to
    # ~1e-7 per point (seen on B200 over random grids: 5e-11 .. 1e-9)
    assert rel(st.sum, st_r.sum) < 5e-9 and rel(st.sum2, st_r.sum2) < 2e-8
    assert np.max(rel(ctx.get_alpha()[0], R.get_alpha()[0])) < 1e-8


def test_channel_tables_in_shared_memory_are_bit_identical(ctx_factory, rng):
    """The phased weight pass with each channel's bin-search tables staged in
    shared memory gives the same bits as with the tables read from global
    memory: the first iteration's StatsData of the 2->4 workload on the
    device's own uniforms. Later iterations start from grids adapted on
    histograms summed with FP64 atomics, whose order varies from run to run,
    so they agree to rounding."""
    cs = workloads.channel_set(4)
    out = []
    for tables in (1, 0):
        ctx = ctx_factory()
        ctx.set_option("channel_tables", tables)
        ctx.set_channels(cs)
        ctx.uniform_grids(cs.nch, ctx.ndims, 100)
        ctx.set_integrand(abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
        ctx.set_preprocess_cuts(cs.sqrts)
        params = workloads.mc_params(100_000)
        c, sts = 0, []
        for _ in range(4):
            st, info = ctx.multichannel_iterate(params, seed=3, counter=c, guard=True)
            c += info.points_tried
            sts.append(st.as_tuple())
        out.append((sts, ctx.get_alpha()[0], ctx.get_grids()))
    assert out[0][0][0] == out[1][0][0]
    for a, b in zip(out[0][0][1:], out[1][0][1:]):
        assert a[0] == b[0] and a[5] == b[5]
        assert all(rel(x, y) < 1e-11 for x, y in zip(a[2:5], b[2:5]))
    assert np.allclose(out[0][1], out[1][1], rtol=1e-10, atol=0)
    assert np.allclose(out[0][2], out[1][2], rtol=1e-10, atol=0)
