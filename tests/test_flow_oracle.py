"""The learned proposal's CPU oracle (oracle/flow.py): hand-derived
gradients against central finite differences in FP64, the spline round trip,
the identity initialisation, and the host mirror of the library's parameter
layout (chili_b200/flowspec.py). No GPU."""
import numpy as np
import pytest

from chili_b200 import flowspec
from oracle import flow as F


def _perturbed(spec, rng, scale=0.05):
    p = spec.init(rng)
    for k in p:
        if k.startswith("W3") or k.startswith("E") or k in ("A3", "c3", "c1"):
            p[k] = p[k] + rng.normal(0, scale, p[k].shape)
    return p


def _batch(rng, n, dims, nch, nfeat):
    b = dict(u=rng.random((n, dims)), ch=rng.integers(0, nch, n), logf=rng.normal(0, 0.5, n),
             logbeta=np.log(rng.dirichlet(np.ones(nch))), feat=rng.normal(0, 1, (n, nfeat)),
             logprior=rng.normal(0, 1, (n, nch)))
    b["logf"][3] = -np.inf
    return b


@pytest.mark.parametrize("depth", [2, 3])
def test_gradients_match_central_differences(depth):
    rng = np.random.default_rng(0)
    spec = F.Spec(10, 3, 10, layers=6 if depth == 2 else 3, hidden=16, depth=depth)
    p = _perturbed(spec, rng)
    batch = _batch(rng, 40, 10, 3, 10)
    L, g, _ = F.loss_and_grads(spec, p, batch)
    assert np.isfinite(L) and L > 0
    worst = 0.0
    for k in p:
        flat = p[k].reshape(-1)
        gk = g[k].reshape(-1)
        idx = list(rng.choice(flat.size, min(6, flat.size), replace=False)) + [int(np.argmax(np.abs(gk)))]
        for i in idx:
            old = flat[i]
            h = 1e-7
            flat[i] = old + h
            lp = F.loss_and_grads(spec, p, batch)[0]
            flat[i] = old - h
            lm = F.loss_and_grads(spec, p, batch)[0]
            flat[i] = old
            fd = (lp - lm) / (2 * h)
            err = abs(fd - gk[i]) / max(1e-3 * np.abs(gk).max(), abs(fd), 1e-12)
            worst = max(worst, err)
    assert worst < 1e-4, worst


def test_spline_round_trip_and_log_det():
    rng = np.random.default_rng(1)
    spec = F.Spec(10, 4, 10, layers=6, hidden=32)
    # moderate weights: log q up to ~20 (much steeper maps amplify rounding)
    p = _perturbed(spec, rng, 0.1)
    u = rng.random((500, 10))
    ch = rng.integers(0, 4, 500)
    z, lq, _ = F.flow_forward(spec, p, u, ch)
    u2, lq2 = F.flow_inverse(spec, p, z, ch)
    assert np.abs(u2 - u).max() < 1e-12
    assert np.abs(lq - lq2).max() < 1e-11
    # log q is the log Jacobian: finite-difference check of one dimension of one layer
    th = rng.normal(0, 1, (200, 49))
    x = rng.random(200)
    y, lj = F.spline_forward(th, x)
    h = 1e-7
    yp, _ = F.spline_forward(th, x + h)
    ym, _ = F.spline_forward(th, x - h)
    assert np.abs(np.log((yp - ym) / (2 * h)) - lj).max() < 1e-5


def test_initial_flow_is_the_identity():
    rng = np.random.default_rng(2)
    spec = F.Spec(10, 15, 10)
    p = spec.init(rng)
    u = rng.random((300, 10))
    z, lq, _ = F.flow_forward(spec, p, u, rng.integers(0, 15, 300))
    assert np.abs(z - u).max() < 1e-12
    assert np.abs(lq).max() < 1e-12


@pytest.mark.parametrize("dims,layers,hidden,depth", [(4, 6, 128, 2), (7, 6, 128, 2), (10, 6, 128, 2),
                                                      (16, 10, 128, 2), (10, 10, 256, 3), (7, 4, 128, 4)])
def test_host_layout_mirror_matches_the_oracle(dims, layers, hidden, depth):
    for a, b in zip(flowspec.masks(dims, layers), F.masks(dims, layers)):
        assert (a == b).all()
    spec = F.Spec(dims, 15, flowspec.n_features(6), layers=layers, hidden=hidden, depth=depth)
    p = spec.init(np.random.default_rng(3))
    lay = flowspec.layout(dims, 15, 6, layers, hidden, depth)
    assert [n for n, _, _ in lay] == list(p.keys())
    for name, _, shape in lay:
        assert tuple(shape) == p[name].shape, name
    flat = flowspec.flatten(p, lay)
    back = flowspec.unflatten(flat, lay)
    for k in p:
        assert np.allclose(back[k], p[k].astype(np.float32))
    assert all(int((~m).sum()) <= 5 for m in flowspec.masks(dims, layers))


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 0.0, np.float32(3.14159)])
    r = F.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == -2.5 and r[4] == 0.0
    assert abs(r[5] - 3.140625) < 1e-12


def test_deeper_conditioner_at_identity_init():
    """A 3 x 256 conditioner starts as the identity flow like the 2 x 128 one:
    the last layer is zero apart from the slope bias on the constant unit."""
    rng = np.random.default_rng(5)
    spec = F.Spec(10, 15, 10, layers=10, hidden=256, depth=3)
    p = spec.init(rng)
    u = rng.random((200, 10))
    z, lq, _ = F.flow_forward(spec, p, u, rng.integers(0, 15, 200))
    assert np.abs(z - u).max() < 1e-12
    assert np.abs(lq).max() < 1e-12
