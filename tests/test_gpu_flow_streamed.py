"""The streamed-weight coupling kernels, which every conditioner wider or
deeper than 2 x 128 runs on (3 x 256 is the large workload's): on a 2 x 128
flow against the kernels that keep the weights in shared memory (the same
function), and at 3 x 256 against the FP64 oracle (oracle/flow.py, with the
bf16 rounding of the tensor-core operands emulated) in both directions and
for the loss gradients; then a few training steps."""
import numpy as np
import pytest

from chili_b200 import abi, channels, flowspec, workloads
from oracle import flow as F

pytestmark = pytest.mark.gpu


def _setup(ctx_factory, hidden, depth, streamed=False, layers=6, batch=4096):
    cs = workloads.channel_set(4)
    ctx = ctx_factory()
    ctx.set_channels(cs)
    ctx.uniform_grids(cs.nch, ctx.ndims, 100)
    ctx.set_integrand(abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    ctx.set_preprocess(abi.CHILI_PRE_FINITE)
    ctx.set_alpha(np.full(cs.nch, 1.0 / cs.nch))
    if streamed:
        ctx.set_option("flow_streamed", 1)
    ctx.flow_init(abi.FlowParams.defaults(batch=batch, layers=layers, hidden=hidden, depth=depth))
    return ctx, cs


def _perturbed(ctx, cs, rng, layers, hidden, depth, scale=0.05):
    # theta = W3 h sums over `hidden` units: the perturbation shrinks with
    # sqrt(hidden) so that the splines are as steep as in the 2 x 128 tests
    scale *= np.sqrt(128 / hidden)
    lay = flowspec.layout(ctx.ndims, cs.nch, cs.n_ext, layers, hidden, depth)
    assert lay[-1][1] + int(np.prod(lay[-1][2])) == ctx.flow_np
    p = flowspec.unflatten(ctx.flow_get_params(), lay)
    for k in p:
        if k.startswith("W3") or k.startswith("E") or k in ("A3", "c3", "c1", "c2"):
            p[k] = p[k] + rng.normal(0, scale, p[k].shape)
    return flowspec.flatten(p, lay), lay


def _batch(rng, cs, dims, n, beta):
    nfeat = flowspec.n_features(cs.n_ext)
    b = dict(u=rng.random((n, dims)).astype(np.float32).astype(np.float64),
             ch=rng.integers(0, cs.nch, n),
             logf=rng.normal(0, 0.7, n).astype(np.float32).astype(np.float64),
             logbeta=np.log(beta).astype(np.float32).astype(np.float64),
             feat=rng.uniform(-1, 1, (n, nfeat)).astype(np.float32).astype(np.float64),
             logprior=(np.log(1 / cs.nch) + rng.normal(0, 1, (n, cs.nch))).astype(np.float32).astype(np.float64))
    b["logf"][::17] = -np.inf
    return b


def test_streamed_kernels_match_resident_kernels(ctx_factory):
    """2 x 128: the same products in the same K order on both kernel
    families, so densities, inverses and gradients agree to f32 rounding."""
    rng = np.random.default_rng(11)
    res, cs = _setup(ctx_factory, 128, 2)
    stm, _ = _setup(ctx_factory, 128, 2, streamed=True)
    flat, lay = _perturbed(res, cs, rng, 6, 128, 2)
    res.flow_set_params(flat)
    stm.flow_set_params(flat)
    n = 3000  # a partial last tile
    u = rng.random((n, res.ndims)).astype(np.float32)
    ch = rng.integers(0, cs.nch, n)
    z_r, lq_r = res.flow_density(u, ch)
    z_s, lq_s = stm.flow_density(u, ch)
    assert np.abs(z_s - z_r).max() < 1e-6, np.abs(z_s - z_r).max()
    assert np.abs(lq_s - lq_r).max() < 1e-4, np.abs(lq_s - lq_r).max()
    u_r, _ = res.flow_sample_u(z_r, ch)
    u_s, _ = stm.flow_sample_u(z_r, ch)
    assert np.abs(u_s - u_r).max() < 1e-6
    beta = rng.dirichlet(np.ones(cs.nch) * 5)
    res.flow_set_beta(beta)
    stm.flow_set_beta(beta)
    b = _batch(rng, cs, res.ndims, 1000, beta)
    L_r, g_r = res.flow_loss_grad(b["u"], b["ch"], b["logf"], b["feat"], b["logprior"])
    L_s, g_s = stm.flow_loss_grad(b["u"], b["ch"], b["logf"], b["feat"], b["logprior"])
    assert abs(L_s - L_r) <= 1e-5 * abs(L_r)
    gr, gs = flowspec.unflatten(g_r, lay), flowspec.unflatten(g_s, lay)
    for k in gr:
        nrm = np.linalg.norm(gr[k])
        assert np.linalg.norm(gs[k] - gr[k]) <= 1e-4 * max(nrm, 1e-12), k


@pytest.mark.parametrize("hidden,depth", [(256, 3), (128, 4)])
def test_wide_flow_matches_oracle_both_directions(ctx_factory, hidden, depth):
    ctx, cs = _setup(ctx_factory, hidden, depth)
    rng = np.random.default_rng(12)
    flat, lay = _perturbed(ctx, cs, rng, 6, hidden, depth)
    ctx.flow_set_params(flat)
    p = flowspec.unflatten(flat, lay)
    spec = F.Spec(ctx.ndims, cs.nch, flowspec.n_features(cs.n_ext), hidden=hidden, depth=depth)
    n = 2000
    u = rng.random((n, ctx.ndims)).astype(np.float32)
    ch = rng.integers(0, cs.nch, n)
    z, lq = ctx.flow_density(u, ch)
    zo, lqo, _ = F.flow_forward(spec, p, u.astype(np.float64), ch, use_bf16=True)
    # a point that ends in a very steep part of a spline turns the
    # f32-accumulation differences into large coordinate and log-derivative
    # differences, so the tails are bounded by quantiles (a wrong tile, column
    # or layer would move far more than 0.1% / 0.5% of the values, and by
    # O(1)); measured on B200 at 3 x 256: z median 6e-8, max 2.7e-3; log q
    # median 1.0e-5, 99.5% quantile 2.5e-2, max 0.14
    dz = np.abs(z - zo)
    assert np.median(dz) < 1e-6 and np.quantile(dz, 0.999) < 2e-3 and dz.max() < 2e-2, \
        (np.median(dz), np.quantile(dz, 0.999), dz.max())
    dl = np.abs(lq - lqo)
    assert np.median(dl) < 1e-4 and np.quantile(dl, 0.995) < 5e-2 and dl.max() < 1.0, \
        (np.median(dl), np.quantile(dl, 0.995), dl.max(), int(np.argmax(dl)))
    u2, lq2 = ctx.flow_sample_u(z, ch)
    assert np.abs(u2 - u).max() < 1e-3
    assert np.median(np.abs(lq2 - lq)) < 1e-4
    uo, _ = F.flow_inverse(spec, p, z.astype(np.float64), ch, use_bf16=True)
    assert np.median(np.abs(u2 - uo)) < 1e-6


def test_wide_loss_gradients_match_oracle(ctx_factory):
    hidden, depth = 256, 3
    ctx, cs = _setup(ctx_factory, hidden, depth)
    rng = np.random.default_rng(13)
    flat, lay = _perturbed(ctx, cs, rng, 6, hidden, depth)
    ctx.flow_set_params(flat)
    p = flowspec.unflatten(flat, lay)
    beta = rng.dirichlet(np.ones(cs.nch) * 5)
    ctx.flow_set_beta(beta)
    spec = F.Spec(ctx.ndims, cs.nch, flowspec.n_features(cs.n_ext), hidden=hidden, depth=depth)
    b = _batch(rng, cs, ctx.ndims, 1000, beta)
    loss, grad = ctx.flow_loss_grad(b["u"], b["ch"], b["logf"], b["feat"], b["logprior"])
    Lo, go, _ = F.loss_and_grads(spec, p, b, use_bf16=True)
    # the same bars as the 2 x 128 kernels' test: bf16 operands emulated,
    # f32 accumulation order and f32 spline arithmetic left
    assert abs(loss - Lo) <= 2e-4 * Lo, (loss, Lo)
    g = flowspec.unflatten(grad, lay)
    worst = {}
    for k in go:
        nrm = np.linalg.norm(go[k])
        if nrm == 0:
            assert np.abs(g[k]).max() < 1e-6, k
            continue
        worst[k] = np.linalg.norm(g[k] - go[k]) / nrm
    bad = {k: v for k, v in worst.items() if v > 1e-2}
    assert not bad, bad
    # measured on B200 at 3 x 256: the coupling layers' blocks median 2.4e-3;
    # the channel-weight network's blocks 0.5-1.5e-3 (their bf16 operands are
    # emulated too; what is left comes from the flow's log q through the loss)
    assert np.median(list(worst.values())) < 4e-3, worst


def test_wide_flow_trains(ctx_factory):
    """Ten coupling layers of 3 x 256 (the large workload's network) on the
    2->4 channels: training steps run, the loss stays finite and falls, and
    an integration pass through the trained flow gives finite statistics."""
    ctx, cs = _setup(ctx_factory, 256, 3, layers=10, batch=16384)
    loss = ctx.flow_train(60, seed=31, counter=0)
    assert np.all(np.isfinite(loss))
    assert loss[-15:].mean() < loss[:15].mean(), (loss[:15].mean(), loss[-15:].mean())
    st, info = ctx.flow_iterate(200_000, seed=32, counter=0)
    assert info.points == 200_000 and info.nonfinite == 0
    assert np.isfinite(st.sum) and st.sum > 0
