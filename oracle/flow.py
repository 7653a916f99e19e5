"""FP64 CPU oracle of the learned proposal: a channel-conditioned
rational-quadratic spline coupling flow on the VEGAS uniforms, a softmax
channel-weight network, the variance loss, hand-derived gradients and Adam.

TEST INFRASTRUCTURE ONLY: the tests and the benchmark's checks use it to
verify the CUDA kernels; no product path imports it.

Chili itself has no learned proposal, so there is no reference code to pin
this to. It restates published methods, each written out below:

* rational-quadratic spline on [0, 1] (Durkan, Bekasov, Murray, Papamakarios,
  "Neural Spline Flows", NeurIPS 2019, eqs. 4-8 and the inverse of their
  appendix A), K bins, all K+1 knot derivatives learned (no linear tails: the
  domain is the VEGAS unit hypercube);
* affine coupling structure (Dinh et al., "Density estimation using Real
  NVP", 2017) with fixed binary masks;
* multi-channel weights from a network with an analytic prior
  (Heimel et al., "MadNIS - Neural multi-channel importance sampling",
  SciPost Phys. 15 (2023) 141): per point, the estimator
  alpha_c(p) f(p) D_c(p) / (beta_c q_c(u)) for the channel c that generated
  the point, which is unbiased for any alpha(p) summing to one;
* Adam (Kingma & Ba, 2015).

The gradients are derived by hand (no autograd) and checked against central
finite differences in the tests. `bf16=True` rounds exactly the tensors that
the CUDA kernels feed to the tensor cores (GEMM operands) to bfloat16, so that
the GPU can be compared with a tight tolerance.
"""
import math

import numpy as np

K_BINS = 16
MIN_W = 1e-3
MIN_H = 1e-3
MIN_D = 1e-3
SLOPE = 0.01          # leaky-ReLU slope
# softplus^-1(1 - MIN_D): the derivative bias that makes the spline the identity
D_ID = math.log(math.expm1(1.0 - MIN_D))


def bf16(a):
    """Round float64/float32 values to bfloat16 (round to nearest even) and
    return them as float64."""
    f = np.asarray(a, dtype=np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    rnd = ((b >> 16) & 1) + 0x7FFF
    b = ((b + rnd) >> 16) << 16
    out = b.astype(np.uint32).view(np.float32).astype(np.float64)
    return np.where(np.isnan(f), np.nan, out)


def masks(dims, layers):
    """Conditioning masks: True = identity (conditioning) dimension; every
    layer transforms at most 5 dimensions (5 * 49 spline parameters fit one
    256-column tensor-core tile). Up to 10 dimensions the pattern cycles
    through alternating, half/half and shifted-pair splits and their
    complements; above 10, layer l transforms dimensions 5l .. 5l+4 (mod D)."""
    idx = np.arange(dims)
    out = []
    if dims <= 10:
        pats = [idx % 2 == 0, idx % 2 == 1, idx < dims // 2, idx >= dims // 2,
                ((idx + 1) // 2) % 2 == 0, ((idx + 1) // 2) % 2 == 1]
        for l in range(layers):
            m = pats[l % 6]
            if m.all() or not m.any():
                m = idx % 2 == (l % 2)
            out.append(m)
    else:
        for l in range(layers):
            t = (5 * l + np.arange(5)) % dims
            m = np.ones(dims, dtype=bool)
            m[t] = False
            out.append(m)
    return out


class Spec:
    """Sizes of the flow and the channel-weight network."""

    def __init__(self, dims, nch, nfeat, layers=6, hidden=128, bins=K_BINS, alpha_hidden=64, depth=2):
        self.dims, self.nch, self.nfeat = dims, nch, nfeat
        self.layers, self.hidden, self.bins, self.alpha_hidden = layers, hidden, bins, alpha_hidden
        self.depth = depth  # hidden layers of a conditioner (W1, then depth - 1 square matrices)
        self.masks = masks(dims, layers)
        self.cond = [np.where(m)[0] for m in self.masks]
        self.trans = [np.where(~m)[0] for m in self.masks]
        self.per_dim = 3 * bins + 1
        self.nparams = [len(t) * self.per_dim for t in self.trans]

    def init(self, rng):
        """Initial parameters: the flow is the identity (last conditioner
        layer zero apart from the derivative bias) and the channel-weight
        network returns the prior (last layer zero)."""
        H, P = self.hidden, None
        p = {}
        for l in range(self.layers):
            da, P = len(self.cond[l]), self.nparams[l]
            p[f"W1_{l}"] = rng.uniform(-1, 1, (H, da)) * math.sqrt(6.0 / da)
            p[f"E_{l}"] = np.zeros((self.nch, H))
            for k in range(self.depth - 1):
                p[w2_name(l, k)] = rng.uniform(-1, 1, (H, H)) * math.sqrt(6.0 / H)
            w3 = np.zeros((P, H))
            for j in range(len(self.trans[l])):
                o = j * self.per_dim + 2 * self.bins
                w3[o:o + self.bins + 1, H - 1] = D_ID
            p[f"W3_{l}"] = w3
        A, F = self.alpha_hidden, self.nfeat
        p["A1"] = rng.uniform(-1, 1, (A, F)) * math.sqrt(6.0 / F)
        p["c1"] = np.zeros(A)
        p["A2"] = rng.uniform(-1, 1, (A, A)) * math.sqrt(6.0 / A)
        p["c2"] = np.zeros(A)
        p["A3"] = np.zeros((self.nch, A))
        p["c3"] = np.zeros(self.nch)
        return p


def w2_name(l, k):
    """Name of the k-th square hidden matrix of coupling layer l (W2_l for
    the first, W2_l_k for the further ones of deeper conditioners)."""
    return f"W2_{l}" if k == 0 else f"W2_{l}_{k}"


def lrelu(x):
    return np.where(x > 0, x, SLOPE * x)


def dlrelu(h):
    return np.where(h > 0, 1.0, SLOPE)


# ---------------------------------------------------------------- the spline
def _softmax(t):
    t = t - t.max(axis=-1, keepdims=True)
    e = np.exp(t)
    return e / e.sum(axis=-1, keepdims=True)


def _softplus(t):
    return np.where(t > 20, t, np.log1p(np.exp(np.minimum(t, 20))))


def _sigmoid(t):
    return 1.0 / (1.0 + np.exp(-t))


def spline_knots(theta, bins=K_BINS):
    """theta [..., 3K+1] -> widths, heights (K), derivatives (K+1), knot
    positions xk, yk (K+1; cumulative sums in bin order, last forced to 1)."""
    tw, th, td = theta[..., :bins], theta[..., bins:2 * bins], theta[..., 2 * bins:]
    w = MIN_W + (1 - bins * MIN_W) * _softmax(tw)
    h = MIN_H + (1 - bins * MIN_H) * _softmax(th)
    d = MIN_D + _softplus(td)
    xk = np.concatenate([np.zeros(w.shape[:-1] + (1,)), np.cumsum(w, axis=-1)], axis=-1)
    yk = np.concatenate([np.zeros(h.shape[:-1] + (1,)), np.cumsum(h, axis=-1)], axis=-1)
    xk[..., -1] = 1.0
    yk[..., -1] = 1.0
    return w, h, d, xk, yk


def _bin(knots, v, bins):
    """Bin index: the number of interior knots not above v."""
    return np.sum(knots[..., 1:bins] <= v[..., None], axis=-1)


def _take(a, k):
    return np.take_along_axis(a, k[..., None], axis=-1)[..., 0]


def spline_forward(theta, x, bins=K_BINS):
    """y = RQS(x), log dy/dx."""
    w, h, d, xk, yk = spline_knots(theta, bins)
    k = _bin(xk, x, bins)
    wk, hk, x0, y0 = _take(w, k), _take(h, k), _take(xk, k), _take(yk, k)
    d0, d1 = _take(d, k), _take(d, k + 1)
    xi = (x - x0) / wk
    s = hk / wk
    om = xi * (1 - xi)
    A = s * xi * xi + d0 * om
    B = s + (d0 + d1 - 2 * s) * om
    C = d1 * xi * xi + 2 * s * om + d0 * (1 - xi) ** 2
    y = y0 + hk * A / B
    logj = 2 * np.log(s) + np.log(C) - 2 * np.log(B)
    return y, logj


def spline_inverse(theta, y, bins=K_BINS):
    """x = RQS^-1(y) (root of the quadratic in the bin), log dy/dx at x."""
    w, h, d, xk, yk = spline_knots(theta, bins)
    k = _bin(yk, y, bins)
    wk, hk, x0, y0 = _take(w, k), _take(h, k), _take(xk, k), _take(yk, k)
    d0, d1 = _take(d, k), _take(d, k + 1)
    s = hk / wk
    dl = d0 + d1 - 2 * s
    dy = y - y0
    a = hk * (s - d0) + dy * dl
    b = hk * d0 - dy * dl
    c = -s * dy
    disc = np.maximum(b * b - 4 * a * c, 0.0)
    xi = 2 * c / (-b - np.sqrt(disc))
    x = x0 + xi * wk
    om = xi * (1 - xi)
    B = s + dl * om
    C = d1 * xi * xi + 2 * s * om + d0 * (1 - xi) ** 2
    logj = 2 * np.log(s) + np.log(C) - 2 * np.log(B)
    return x, logj


def spline_backward(theta, x, gy, gj, bins=K_BINS):
    """Gradients of gy*y + gj*log(dy/dx) with respect to theta [..., 3K+1]
    and to x. Local partials of y and log J in (xi, s, d_k, d_k+1, h_k, y_k),
    then through xi = (x - x_k)/w_k, s = h_k/w_k, the cumulative knot sums and
    the softmax/softplus parametrisation."""
    w, h, d, xk, yk = spline_knots(theta, bins)
    k = _bin(xk, x, bins)
    wk, hk, x0 = _take(w, k), _take(h, k), _take(xk, k)
    d0, d1 = _take(d, k), _take(d, k + 1)
    xi = (x - x0) / wk
    s = hk / wk
    om = xi * (1 - xi)
    dl = d0 + d1 - 2 * s
    A = s * xi * xi + d0 * om
    B = s + dl * om
    C = d1 * xi * xi + 2 * s * om + d0 * (1 - xi) ** 2
    # partials of A, B, C
    A_xi, A_s, A_d0 = 2 * s * xi + d0 * (1 - 2 * xi), xi * xi, om
    B_xi, B_s, B_d0, B_d1 = dl * (1 - 2 * xi), 1 - 2 * om, om, om
    C_xi = 2 * d1 * xi + 2 * s * (1 - 2 * xi) - 2 * d0 * (1 - xi)
    C_s, C_d0, C_d1 = 2 * om, (1 - xi) ** 2, xi * xi
    hB2 = hk / (B * B)
    g_xi = gy * hB2 * (A_xi * B - A * B_xi) + gj * (C_xi / C - 2 * B_xi / B)
    g_s = gy * hB2 * (A_s * B - A * B_s) + gj * (2 / s + C_s / C - 2 * B_s / B)
    g_d0 = gy * hB2 * (A_d0 * B - A * B_d0) + gj * (C_d0 / C - 2 * B_d0 / B)
    g_d1 = gy * hB2 * (-A * B_d1) + gj * (C_d1 / C - 2 * B_d1 / B)
    g_hk = gy * A / B + g_s / wk
    g_x = g_xi / wk
    g_x0 = -g_xi / wk
    g_wk = -(g_xi * xi + g_s * s) / wk
    g_y0 = gy
    # scatter to widths / heights / derivatives
    ar = np.arange(bins)
    below = ar < k[..., None]
    gw = np.where(below, g_x0[..., None], 0.0) + np.where(ar == k[..., None], g_wk[..., None], 0.0)
    gh = np.where(below, g_y0[..., None], 0.0) + np.where(ar == k[..., None], g_hk[..., None], 0.0)
    ar1 = np.arange(bins + 1)
    gd = np.where(ar1 == k[..., None], g_d0[..., None], 0.0) + np.where(ar1 == (k + 1)[..., None], g_d1[..., None], 0.0)
    # the last knot is forced to 1: it carries no gradient (x_k, y_k < K only)
    sw = _softmax(theta[..., :bins])
    sh = _softmax(theta[..., bins:2 * bins])
    gsw = (1 - bins * MIN_W) * gw
    gsh = (1 - bins * MIN_H) * gh
    gtw = sw * (gsw - np.sum(gsw * sw, axis=-1, keepdims=True))
    gth = sh * (gsh - np.sum(gsh * sh, axis=-1, keepdims=True))
    gtd = gd * _sigmoid(theta[..., 2 * bins:])
    return np.concatenate([gtw, gth, gtd], axis=-1), g_x


# ---------------------------------------------------------------- the flow
def _mm(a, b, use_bf16):
    if use_bf16:
        return bf16(a) @ bf16(b)
    return a @ b


def conditioner(spec, p, l, xa, ch, use_bf16=False):
    """theta [N, P] from the conditioning coordinates xa [N, Da] and channels."""
    H = spec.hidden
    a0 = 2 * xa - 1
    # the GPU adds E[c] inside the first tensor-core product (a one-hot column),
    # so in bf16 mode E is rounded like the other operands
    E = bf16(p[f"E_{l}"]) if use_bf16 else p[f"E_{l}"]
    h = lrelu(_mm(a0, p[f"W1_{l}"].T, use_bf16) + E[ch])
    h[:, H - 1] = 1.0
    hs = [h]
    for k in range(spec.depth - 1):
        h = lrelu(_mm(h, p[w2_name(l, k)].T, use_bf16))
        h[:, H - 1] = 1.0
        hs.append(h)
    theta = _mm(h, p[f"W3_{l}"].T, use_bf16)
    return theta, (a0, *hs)


def flow_forward(spec, p, u, ch, use_bf16=False):
    """Density direction u -> z; returns z, log q(u) and the cache for the
    backward pass."""
    x = np.array(u, dtype=np.float64)
    logq = np.zeros(x.shape[0])
    cache = []
    for l in range(spec.layers):
        ci, ti = spec.cond[l], spec.trans[l]
        x = np.clip(x, 0.0, 1.0)
        theta, acts = conditioner(spec, p, l, x[:, ci], ch, use_bf16)
        th = theta.reshape(x.shape[0], len(ti), spec.per_dim)
        y, lj = spline_forward(th, x[:, ti], spec.bins)
        cache.append((x.copy(), th, acts))
        x[:, ti] = y
        logq += lj.sum(axis=1)
    return x, logq, cache


def flow_inverse(spec, p, z, ch, use_bf16=False):
    """Sampling direction z -> u; returns u and log q(u)."""
    x = np.array(z, dtype=np.float64)
    logq = np.zeros(x.shape[0])
    for l in reversed(range(spec.layers)):
        ci, ti = spec.cond[l], spec.trans[l]
        x = np.clip(x, 0.0, 1.0)
        theta, _ = conditioner(spec, p, l, x[:, ci], ch, use_bf16)
        th = theta.reshape(x.shape[0], len(ti), spec.per_dim)
        xin, lj = spline_inverse(th, x[:, ti], spec.bins)
        x[:, ti] = xin
        logq += lj.sum(axis=1)
    return x, logq


def flow_backward(spec, p, cache, ch, g_logq, use_bf16=False):
    """Gradients of sum_i g_logq[i] * log q(u_i) with respect to every flow
    parameter (z does not enter the loss: the base density is uniform)."""
    n = g_logq.shape[0]
    H = spec.hidden
    grads = {}
    gx = np.zeros((n, spec.dims))
    for l in reversed(range(spec.layers)):
        ci, ti = spec.cond[l], spec.trans[l]
        x_in, th, (a0, *hs) = cache[l]
        q = bf16 if use_bf16 else (lambda v: v)
        gy = gx[:, ti]
        gj = np.repeat(g_logq[:, None], len(ti), axis=1)
        gth, gxt = spline_backward(th, x_in[:, ti], gy, gj, spec.bins)
        gtheta = gth.reshape(n, -1)
        grads[f"W3_{l}"] = q(gtheta).T @ q(hs[-1])
        g = _mm(gtheta, p[f"W3_{l}"], use_bf16)  # gradient of the last hidden layer
        for k in reversed(range(spec.depth)):
            g[:, H - 1] = 0.0
            gp = g * dlrelu(hs[k])  # gradient of layer k's pre-activation
            if k > 0:
                grads[w2_name(l, k - 1)] = q(gp).T @ q(hs[k - 1])
                g = _mm(gp, p[w2_name(l, k - 1)], use_bf16)
        gp1q = q(gp)
        grads[f"W1_{l}"] = gp1q.T @ q(a0)
        gE = np.zeros((spec.nch, H))
        np.add.at(gE, ch, gp1q)
        grads[f"E_{l}"] = gE
        ga0 = _mm(gp, p[f"W1_{l}"], use_bf16)
        gnew = gx.copy()
        gnew[:, ti] = gxt
        gnew[:, ci] += 2 * ga0
        gx = gnew
    return grads


# ------------------------------------------------- the channel-weight network
def alpha_forward(spec, p, feat, logprior, use_bf16=False):
    """log alpha [N, nch] = log softmax(MLP(features) + log prior). With
    use_bf16 the three products take bf16 operands (the GPU runs them on the
    tensor cores); biases, log prior and the softmax stay unrounded."""
    a1 = lrelu(_mm(feat, p["A1"].T, use_bf16) + p["c1"])
    a2 = lrelu(_mm(a1, p["A2"].T, use_bf16) + p["c2"])
    logits = _mm(a2, p["A3"].T, use_bf16) + p["c3"] + logprior
    m = logits.max(axis=1, keepdims=True)
    lse = m[:, 0] + np.log(np.exp(logits - m).sum(axis=1))
    return logits - lse[:, None], (feat, a1, a2)


def alpha_backward(spec, p, cache, logalpha, g_logalpha_sel, ch, use_bf16=False):
    """Gradients of sum_i g[i] * log alpha_{c_i}(p_i). With use_bf16 every
    product's operands are rounded to bf16, the bias gradients included (the
    GPU sums the bf16 gradient rows against a constant-1 operand column)."""
    feat, a1, a2 = cache
    n = feat.shape[0]
    q = bf16 if use_bf16 else (lambda v: v)
    al = np.exp(logalpha)
    g_logits = -al * g_logalpha_sel[:, None]
    g_logits[np.arange(n), ch] += g_logalpha_sel
    g = {"A3": _mm(g_logits.T, a2, use_bf16), "c3": q(g_logits).sum(0)}
    g2 = _mm(g_logits, p["A3"], use_bf16) * dlrelu(a2)
    g["A2"], g["c2"] = _mm(g2.T, a1, use_bf16), q(g2).sum(0)
    g1 = _mm(g2, p["A2"], use_bf16) * dlrelu(a1)
    g["A1"], g["c1"] = _mm(g1.T, feat, use_bf16), q(g1).sum(0)
    return g


# ---------------------------------------------------------------- the loss
def loss_terms(logalpha_sel, logf, logbeta_sel, logq):
    """Per-point variance-loss terms l_i = alpha^2 F^2 / (beta^2 q), i.e. the
    second moment of the channel estimator alpha_c F / (beta_c q_c) under the
    flow, estimated with points drawn uniformly in u (the plain channel
    proposal). F <= 0 or non-finite (logf = -inf or NaN) gives 0."""
    t = 2 * logalpha_sel + 2 * logf - 2 * logbeta_sel - logq
    ok = np.isfinite(t)
    return np.where(ok, np.exp(np.where(ok, t, 0.0)), 0.0)


def loss_and_grads(spec, p, batch, use_bf16=False):
    """Mean variance-loss term over the batch and the gradient of every
    parameter. batch: u [N, D], ch [N], logf [N], logbeta [nch],
    feat [N, F], logprior [N, nch]."""
    u, ch, logf = batch["u"], batch["ch"], batch["logf"]
    n = u.shape[0]
    _, logq, fcache = flow_forward(spec, p, u, ch, use_bf16)
    logalpha, acache = alpha_forward(spec, p, batch["feat"], batch["logprior"], use_bf16)
    las = logalpha[np.arange(n), ch]
    ell = loss_terms(las, logf, batch["logbeta"][ch], logq)
    L = ell.mean()
    grads = flow_backward(spec, p, fcache, ch, -ell / n, use_bf16)
    grads.update(alpha_backward(spec, p, acache, logalpha, 2 * ell / n, ch, use_bf16))
    return L, grads, {"logq": logq, "logalpha": logalpha, "ell": ell}


class Adam:
    """Adam with bias correction (Kingma & Ba 2015, algorithm 1)."""

    def __init__(self, params, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.lr, self.b1, self.b2, self.eps = lr, b1, b2, eps
        self.m = {k: np.zeros_like(v) for k, v in params.items()}
        self.v = {k: np.zeros_like(v) for k, v in params.items()}
        self.t = 0

    def step(self, params, grads):
        self.t += 1
        c1 = 1 - self.b1 ** self.t
        c2 = 1 - self.b2 ** self.t
        for k, g in grads.items():
            self.m[k] = self.b1 * self.m[k] + (1 - self.b1) * g
            self.v[k] = self.b2 * self.v[k] + (1 - self.b2) * g * g
            params[k] = params[k] - self.lr * (self.m[k] / c1) / (np.sqrt(self.v[k] / c2) + self.eps)
