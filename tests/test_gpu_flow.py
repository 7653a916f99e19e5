"""The learned proposal on the GPU, through the C ABI: the tcgen05 products
against numpy on bf16-rounded inputs, the coupling flow (both directions)
and the loss gradients against the FP64 oracle (oracle/flow.py, emulating the
bf16 rounding of the tensor-core operands), and what training gains: the
trained flow path has a lower variance per point than the untrained one and
its integral agrees with the plain multichannel path."""
import numpy as np
import pytest

from chili_b200 import abi, channels, flowspec, workloads
from oracle import flow as F

pytestmark = pytest.mark.gpu


def bf16(a):
    return F.bf16(a)


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("K,N", [(16, 128), (128, 128), (256, 256), (128, 16), (64, 80)])
def test_tensor_core_products(ctx_factory, mode, K, N):
    ctx = ctx_factory()
    rng = np.random.default_rng(K * 1000 + N + mode)
    if mode == 0:
        A, B = rng.normal(size=(128, K)), rng.normal(size=(N, K))
        ref = bf16(A) @ bf16(B).T
    elif mode == 1:
        A, B = rng.normal(size=(K, 128)), rng.normal(size=(K, N))
        ref = bf16(A).T @ bf16(B)
    else:
        A, B = rng.normal(size=(128, K)), rng.normal(size=(K, N))
        ref = bf16(A) @ bf16(B)
    C = ctx.tc_selftest(mode, A, B, N)
    assert np.abs(C - ref).max() <= 1e-4 * max(1.0, np.abs(ref).max())


def test_bounded_wait_gives_up_and_the_context_survives(ctx_factory):
    """Failure detection without a fault: a tensor-core wait on an mbarrier
    that nothing arrives on gives up after its bounded number of polls, the
    kernel releases its tensor memory and the call reports CHILI_ERR_TIMEOUT;
    the same context then runs a product normally."""
    from chili_b200.gpu import ChiliError
    ctx = ctx_factory()
    rng = np.random.default_rng(4)
    A, B = rng.normal(size=(128, 64)), rng.normal(size=(64, 64))
    with pytest.raises(ChiliError) as e:
        ctx.tc_selftest(3, A, B, 64)
    assert e.value.code == abi.CHILI_ERR_TIMEOUT
    C = ctx.tc_selftest(0, A, B, 64)
    assert np.abs(C - bf16(A) @ bf16(B).T).max() <= 1e-4 * max(1.0, np.abs(bf16(A) @ bf16(B).T).max())


def _setup(ctx_factory, batch=4096, plain_iters=0, cuts=False):
    cs = workloads.channel_set(4)
    ctx = ctx_factory()
    ctx.set_channels(cs)
    ctx.uniform_grids(cs.nch, ctx.ndims, 100)
    ctx.set_integrand(abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    if cuts:
        ctx.set_preprocess_cuts(1000.0)
    else:
        ctx.set_preprocess(abi.CHILI_PRE_FINITE)
    ctx.set_alpha(np.full(cs.nch, 1.0 / cs.nch))
    for it in range(plain_iters):
        ctx.multichannel_iterate(workloads.mc_params(200_000), seed=5, counter=it * 10_000_000)
    ctx.flow_init(abi.FlowParams.defaults(batch=batch))
    return ctx, cs


def _random_params(ctx, cs, rng, scale=0.05):
    lay = flowspec.layout(ctx.ndims, cs.nch, cs.n_ext)
    p = flowspec.unflatten(ctx.flow_get_params(), lay)
    for k in p:
        if k.startswith("W3") or k.startswith("E") or k in ("A3", "c3", "c1", "c2"):
            p[k] = p[k] + rng.normal(0, scale, p[k].shape)
    flat = flowspec.flatten(p, lay)
    ctx.flow_set_params(flat)
    return flowspec.unflatten(flat, lay), lay


def test_initial_flow_is_identity_on_gpu(ctx_factory):
    ctx, cs = _setup(ctx_factory)
    rng = np.random.default_rng(1)
    u = rng.random((1000, ctx.ndims)).astype(np.float32)
    ch = rng.integers(0, cs.nch, 1000)
    z, lq = ctx.flow_density(u, ch)
    # the identity up to the bf16 rounding of the slope bias
    # (softplus^-1(1 - 1e-3)), exactly as the oracle rounds it
    assert np.abs(z - u).max() < 1e-4
    assert np.abs(lq).max() < 2e-2
    lay = flowspec.layout(ctx.ndims, cs.nch, cs.n_ext)
    p = flowspec.unflatten(ctx.flow_get_params(), lay)
    spec = F.Spec(ctx.ndims, cs.nch, flowspec.n_features(cs.n_ext))
    zo, lqo, _ = F.flow_forward(spec, p, u.astype(np.float64), ch, use_bf16=True)
    assert np.abs(z - zo).max() < 1e-6
    assert np.abs(lq - lqo).max() < 1e-4


def test_flow_matches_oracle_both_directions(ctx_factory):
    ctx, cs = _setup(ctx_factory)
    rng = np.random.default_rng(2)
    p, lay = _random_params(ctx, cs, rng)
    spec = F.Spec(ctx.ndims, cs.nch, flowspec.n_features(cs.n_ext))
    n = 2000  # not a multiple of 128: partial last tile
    u = rng.random((n, ctx.ndims)).astype(np.float32)
    ch = rng.integers(0, cs.nch, n)
    z, lq = ctx.flow_density(u, ch)
    zo, lqo, _ = F.flow_forward(spec, p, u.astype(np.float64), ch, use_bf16=True)
    dz = np.abs(z - zo)
    assert np.median(dz) < 1e-6 and dz.max() < 2e-3, (np.median(dz), dz.max())
    dl = np.abs(lq - lqo)
    assert np.median(dl) < 1e-4 and dl.max() < 2e-2, (np.median(dl), dl.max())
    # sampling direction: inverse of the density direction
    u2, lq2 = ctx.flow_sample_u(z, ch)
    assert np.abs(u2 - u).max() < 1e-3
    assert np.median(np.abs(lq2 - lq)) < 1e-4
    uo, lqo2 = F.flow_inverse(spec, p, z.astype(np.float64), ch, use_bf16=True)
    assert np.median(np.abs(u2 - uo)) < 1e-6


def test_loss_gradients_match_oracle(ctx_factory):
    ctx, cs = _setup(ctx_factory)
    rng = np.random.default_rng(3)
    p, lay = _random_params(ctx, cs, rng)
    beta = rng.dirichlet(np.ones(cs.nch) * 5)
    ctx.flow_set_beta(beta)
    nfeat = flowspec.n_features(cs.n_ext)
    spec = F.Spec(ctx.ndims, cs.nch, nfeat)
    n = 1000
    batch = dict(u=rng.random((n, ctx.ndims)).astype(np.float32).astype(np.float64),
                 ch=rng.integers(0, cs.nch, n),
                 logf=rng.normal(0, 0.7, n).astype(np.float32).astype(np.float64),
                 logbeta=np.log(beta).astype(np.float32).astype(np.float64),
                 feat=rng.uniform(-1, 1, (n, nfeat)).astype(np.float32).astype(np.float64),
                 logprior=(np.log(1 / cs.nch) + rng.normal(0, 1, (n, cs.nch))).astype(np.float32).astype(np.float64))
    batch["logf"][::17] = -np.inf
    loss, grad = ctx.flow_loss_grad(batch["u"], batch["ch"], batch["logf"], batch["feat"], batch["logprior"])
    Lo, go, _ = F.loss_and_grads(spec, p, batch, use_bf16=True)
    # the oracle rounds the tensor-core operands to bf16 as the GPU does; the
    # rest is f32 accumulation order and the spline's f32 arithmetic (seen on
    # B200: loss within 6e-5, each parameter block within 4e-3, median 7e-4)
    assert abs(loss - Lo) <= 2e-4 * Lo, (loss, Lo)
    g = flowspec.unflatten(grad, lay)
    worst = {}
    for k in go:
        ref = go[k]
        nrm = np.linalg.norm(ref)
        if nrm == 0:
            assert np.abs(g[k]).max() < 1e-6, k
            continue
        worst[k] = np.linalg.norm(g[k] - ref) / nrm
    bad = {k: v for k, v in worst.items() if v > 1e-2}
    assert not bad, bad
    assert np.median(list(worst.values())) < 2e-3, worst


def _rel_var(st):
    m = st.sum / st.n
    return (st.sum2 / st.n - m * m) / (m * m), m, np.sqrt(max(st.sum2 / st.n - m * m, 0) / (st.n - 1))


def test_training_gain_and_integral_agreement(ctx_factory):
    """On the physical region with cuts (where every channel covers the same
    phase space): the untrained flow path is the plain multichannel estimator
    (identity flow, channel weights = the multichannel prior), training lowers
    its variance per point, and the plain path judges the integral."""
    ctx, cs = _setup(ctx_factory, batch=16384, plain_iters=4, cuts=True)
    n = 1_000_000
    plain = [ctx.multichannel_iterate(workloads.mc_params(n, should_optimize=0), seed=9, counter=(50 + k) * 10 ** 8)[0]
             for k in range(2)]
    s = sum(p.sum for p in plain)
    s2 = sum(p.sum2 for p in plain)
    nn = sum(p.n for p in plain)
    mp = s / nn
    ep = np.sqrt((s2 / nn - mp * mp) / (nn - 1))
    rvp = (s2 / nn - mp * mp) / (mp * mp)
    st0, _ = ctx.flow_iterate(4 * n, seed=21, counter=0)
    rv0, m0, e0 = _rel_var(st0)
    assert abs(m0 - mp) < 4 * np.hypot(e0, ep), (m0, mp, e0, ep)
    assert 0.7 < rv0 / rvp < 1.4, (rv0, rvp)  # the same estimator as the plain path
    loss = ctx.flow_train(200, seed=22, counter=0)
    assert np.all(np.isfinite(loss))
    assert loss[-40:].mean() < loss[:40].mean()
    ctx.flow_iterate(n, seed=23, counter=0, adapt_beta=True)
    st1, info = ctx.flow_iterate(4 * n, seed=24, counter=0)
    rv1, m1, e1 = _rel_var(st1)
    assert rv1 < rv0, (rv1, rv0)
    assert abs(m1 - mp) < 4 * np.hypot(e1, ep), (m1, mp, e1, ep)
    assert info.points == 4 * n and 0 < info.unweighting_efficiency <= 1 and info.nonfinite == 0
