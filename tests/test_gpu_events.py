"""Unweighted event output (chili_gpu_generate_unweighted) against the C
oracle on the same counter-based uniforms: the oracle's value of every drawn
point (MultiChannel.hh:214-233 without retries) and hit-or-miss with the
accept-stream uniforms give the kept events; the CUDA library must keep the
same events in the same order, with the same channels, momenta within
1e-10 relative (p99; the values within 1e-11), weights sign(v) max(|v|,
w_max)."""
import numpy as np
import pytest

from chili_b200 import abi, channels, workloads
from oracle import port

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    d = np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
    return np.where(a == b, 0.0, d)


@pytest.fixture(scope="module")
def adapted(ctx_factory):
    """A 2->4 context after one adapting iteration (non-uniform grids and
    channel weights) and the oracle in the same state."""
    cs = workloads.channel_set(4)
    ctx = ctx_factory()
    ctx.set_channels(cs)
    ctx.uniform_grids(cs.nch, ctx.ndims, 50)
    ctx.set_integrand(abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    ctx.set_preprocess_cuts(cs.sqrts)
    params = workloads.mc_params(100_000)
    st, info = ctx.multichannel_iterate(params, seed=3)
    O = port.MultiChannel(cs, 50, params, abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    O.set_cuts(cs.sqrts)
    O.set_grids(ctx.get_grids())
    O.set_alpha(ctx.get_alpha()[0])
    return ctx, O, info.weight_max


def oracle_events(O, seed, counter, n, w_max):
    u = port.philox_uniforms(seed, counter, n, O.ndims + 1)
    val, ich, mom = O.point_values(u)
    r = port.philox_stream_uniforms(seed, counter, n, 2, 1)[:, 0]
    keep = r * w_max < np.abs(val)
    margin = np.abs(r * w_max - np.abs(val)) <= 1e-9 * np.maximum(np.abs(val), 1e-300)
    return val, ich, mom, keep, margin


def test_unweighted_events_match_the_oracle(adapted):
    ctx, O, wmax_iter = adapted
    n, seed, counter = 200_000, 11, 1 << 33
    w_max = wmax_iter / 20  # some events overweight
    mom, wgt, ch, info = ctx.generate_unweighted(n, w_max, seed=seed, counter=counter)
    val, ich, mom_o, keep, margin = oracle_events(O, seed, counter, n, w_max)
    assert info.points == n
    assert margin.sum() == 0, "a hit-or-miss decision within rounding of its threshold"
    assert info.kept == keep.sum() and info.kept > 500
    idx = np.nonzero(keep)[0]
    assert len(idx) == len(wgt)
    assert np.array_equal(ch, ich[idx])
    assert np.percentile(rel(mom, mom_o[idx]).max(axis=(1, 2)), 99) < 1e-10
    want_w = np.copysign(np.maximum(np.abs(val[idx]), w_max), val[idx])
    assert np.percentile(rel(wgt, want_w), 99) < 1e-11
    assert info.overweight == np.sum(np.abs(val[idx]) > w_max)
    assert rel(info.sum, val.sum()) < 1e-11
    assert rel(info.max, val.max()) < 1e-11
    # sum(wgt) / n is an unbiased estimate of the mean value
    mean = val.mean()
    p = np.minimum(np.abs(val) / w_max, 1.0)
    sigma = np.sqrt(np.sum(np.where(p < 1, w_max * np.abs(val) - val ** 2, 0.0))) / n
    assert abs(wgt.sum() / n - mean) < 5 * sigma + 1e-12 * abs(mean)


def test_unweighted_events_truncation_and_errors(adapted):
    from chili_b200.gpu import ChiliError
    ctx, O, wmax_iter = adapted
    n, seed = 50_000, 5
    mom, wgt, ch, info = ctx.generate_unweighted(n, wmax_iter, seed=seed, counter=0)
    m2, w2, c2, i2 = ctx.generate_unweighted(n, wmax_iter, seed=seed, counter=0, max_events=7)
    assert i2.kept == info.kept and len(w2) == min(7, info.kept)
    assert np.array_equal(w2, wgt[:len(w2)]) and np.array_equal(m2, mom[:len(w2)])
    # deterministic: the same counters give the same events
    _, w3, _, i3 = ctx.generate_unweighted(n, wmax_iter, seed=seed, counter=0)
    assert np.array_equal(w3, wgt)
    with pytest.raises(ChiliError):
        ctx.generate_unweighted(n, 0.0)
    with pytest.raises(ChiliError):
        ctx.generate_unweighted(n, float("nan"))
