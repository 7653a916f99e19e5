"""Bad inputs made on the host, none of which may fault the GPU: NaN and
out-of-range uniforms, all-zero training histograms, a massive propagator of
zero width, NaN channel weights.  Each runs through the C ABI and is checked
against the reference (oracle/_ref) where the reference defines the outcome,
against the C oracle where the reference's own behaviour is undefined (it
indexes its grid out of bounds on such inputs), and otherwise for a clean
status."""
import numpy as np
import pytest

from chili_b200 import abi, channels, workloads
from chili_b200.abi import ChannelSet, Decay, ParticleInfo
from chili_b200.workloads import uniforms53
from oracle import port, ref

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    d = np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
    return np.where(a == b, 0.0, d)


def _ctx(ctx_factory, cs, bins):
    ctx = ctx_factory()
    ctx.set_channels(cs)
    ctx.uniform_grids(cs.nch, ctx.ndims, bins)
    ctx.set_integrand(abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    ctx.set_preprocess(abi.CHILI_PRE_FINITE)
    return ctx


def test_nan_uniforms_in_a_multichannel_iteration(ctx_factory):
    """NaN uniforms (and u = 1.0 exactly) give NaN momenta, which the finite
    PreProcess rejects and the retry loop replaces: the same counts and sums
    as the C oracle."""
    cs = workloads.channel_set(4)
    params = workloads.mc_params(5000)
    ctx = _ctx(ctx_factory, cs, 50)
    O = port.MultiChannel(cs, 50, params, abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    rng = np.random.default_rng(7)
    u = uniforms53(rng, (8 * 5000, O.ndims + 1))
    bad = rng.random(u.shape[0]) < 0.02
    u[bad, rng.integers(0, O.ndims, bad.sum())] = np.nan
    u[rng.random(u.shape[0]) < 0.01, 0] = 1.0
    st, info = ctx.multichannel_iterate(params, u=u, guard=True)
    st_o, info_o = O.iterate(u, guard=True)
    assert info.points_tried == info_o.points_tried and info.rejected_pre == info_o.rejected_pre
    assert st.n == st_o.n and st.n_finite == st_o.n_finite
    assert rel(st.sum, st_o.sum) < 1e-11
    assert np.isfinite(st.sum) and np.all(np.isfinite(ctx.get_grids()))


def test_nan_uniforms_in_plain_vegas(ctx_factory):
    """NaN uniforms in plain VEGAS: the point's value is NaN and is counted,
    its square lands in the bins of its finite coordinates (those bins become
    NaN, as Vegas.cc:33-40 would make them), the NaN coordinate's add is
    skipped; the status is clean and the result is the C oracle's."""
    ctx = ctx_factory()
    p = workloads.camel_params()
    ctx.uniform_grids(1, 4, 50)
    ctx.set_integrand(abi.CHILI_FUNC_CAMEL, p)
    rng = np.random.default_rng(3)
    u = uniforms53(rng, (20000, 4))
    u[::97, 2] = np.nan
    st, tr = ctx.vegas_iterate(len(u), u=u, alpha=1.5, adapt=False, train=True)
    edges = np.tile(np.linspace(0.0, 1.0, 51), (4, 1))
    st_o, tr_o, _ = port.vegas_iterate(edges, 1.5, p, u, adapt=False)
    assert st.n == st_o.n == len(u) and st.n_finite == st_o.n_finite
    assert np.isnan(st.sum) and np.isnan(st_o.sum)
    assert np.array_equal(np.isnan(tr), np.isnan(tr_o))
    fin = np.isfinite(tr_o)
    assert fin.any() and np.max(rel(tr[fin], tr_o[fin])) < 1e-12


def test_all_zero_histogram_adaptation(ctx_factory):
    """AdaptiveMap::Adapt on all-zero histogram rows (AdaptiveMap.cc:93, norm
    == 0): the reference leaves those dimensions' edges all zero (bit for bit
    here too); the dimension with data agrees within 1e-12 (CUDA's and
    glibc's pow and log differ in the last ulp)."""
    ctx = ctx_factory()
    rng = np.random.default_rng(1)
    e = np.sort(rng.random((3, 19)), axis=1)
    edges = np.concatenate([np.zeros((3, 1)), e, np.ones((3, 1))], axis=1)
    ctx.set_grids(edges[None])
    train = np.zeros(3 * 20)
    train[20:40] = rng.random(20)  # dimension 1 has data, 0 and 2 none
    ctx.grid_adapt(0, 1.5, train)
    want = ref.am_adapt(edges, 1.5, train)
    got = ctx.get_grids()[0]
    assert np.array_equal(got[[0, 2]], want[[0, 2]]) and not want[[0, 2]].any()
    assert np.max(rel(got[1], want[1])) < 1e-12


def test_zero_width_massive_propagator(ctx_factory):
    """A decay whose parent has a mass but zero width takes the massless
    propagator branch, as in the reference (Channel.cc:73-79): the same
    combined weights."""
    flavs = [1, -1, 11, -11, 13, -13]
    cuts = channels.default_cuts(flavs)
    legs = [ParticleInfo(1 << i, flavs[i], 0.0, 0.0) for i in range(6)]
    z = ParticleInfo(4 | 8, 23, channels.MZ, 0.0)
    chans = [([legs[5], legs[4], z], [Decay(z, legs[2], legs[3])]),
             ([legs[5], legs[4], legs[3], legs[2]], [])]
    cuts["ptmin"][12] = 0.0
    cuts["etamax"][12] = 99.0
    cs = ChannelSet(chans, cuts, 1000.0, 6)
    ctx = _ctx(ctx_factory, cs, 20)
    R = ref.MultiChannel(cs, 20, workloads.mc_params(1000), abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    rng = np.random.default_rng(2)
    x = uniforms53(rng, (4000, R.ndims))
    ich = rng.integers(0, 2, 4000).astype(np.int32)
    mom = np.concatenate([R.fsm_generate(c, x[ich == c]) for c in range(2)])
    ich = np.concatenate([ich[ich == c] for c in range(2)])
    ok = ~np.isnan(mom).any(axis=(1, 2))
    w, _, _ = ctx.multichannel_weight(mom[ok], ich[ok])
    w_r, _, _ = R.weight(mom[ok], ich[ok])
    fin = np.isfinite(w) & np.isfinite(w_r)
    assert fin.mean() > 0.5
    assert np.percentile(rel(w[fin], w_r[fin]), 99) < 1e-12


def test_nan_channel_weights_do_not_fault(ctx_factory):
    """NaN channel weights (what the reference's unguarded alpha training
    produces): every combined weight is NaN, every point a NaN retry, and the
    iteration gives up after its bounded number of rounds (option
    max_rounds, here 20) with CHILI_ERR_TIMEOUT instead of looping forever as
    the reference does; the context stays usable."""
    from chili_b200.gpu import ChiliError
    cs = workloads.channel_set(4)
    ctx = _ctx(ctx_factory, cs, 50)
    ctx.set_option("max_rounds", 20)
    ctx.set_alpha(np.full(cs.nch, np.nan))
    with pytest.raises(ChiliError) as e:
        ctx.multichannel_iterate(workloads.mc_params(2000, should_optimize=0), seed=1)
    assert e.value.code == abi.CHILI_ERR_TIMEOUT
    ctx.set_alpha(np.full(cs.nch, 1.0 / cs.nch))
    st, info = ctx.multichannel_iterate(workloads.mc_params(2000), seed=1)
    assert st.n >= 2000 and np.isfinite(st.sum)
