// flow.cu -- the learned proposal's entry points (include/chili_gpu.h,
// "learned proposal"): parameter layout and initialisation, the training
// step (sample batch -> flow forward -> channel-weight network and loss ->
// flow backward and weight gradients per layer -> Adam -> bf16 tiles), the
// flow-path integration pass, and the parity entry points.
#include <cuda_runtime.h>
#include <math_constants.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "context.h"
#include "flow_phys.cuh"
#include "flow_launch.h"

using namespace chili_flow;

struct FlowState {
    int D = 0, nch = 0, L = 0, F = 0, n_ext = 0, sms = 148;
    long long batch = 65536;
    float lr = 1e-3f;
    std::vector<FlowLayer> layers;
    std::vector<int> da, db;
    std::vector<std::vector<int>> cond, trans;
    std::vector<long long> off_w1, off_e, off_w2, off_w3;
    // conditioner: H hidden units, NH hidden layers; streamed: the
    // streamed-weight kernels (flow_wide.cuh) instead of the resident ones
    int H = kH, NH = 2;
    bool streamed = false;
    std::vector<std::vector<long long>> off_w2x;  // per layer: the NH - 1 square matrices
    std::vector<WideLayer> wlayers;
    DevBuf hsw, gpsw, gthsw;  // streamed kernels: saved activations, g_p tiles, g_theta tiles
    long long np_flow = 0, np = 0, off_alpha = 0;
    AlphaLayout AL{};
    DevBuf prm, m, v, grad, wtiles, atiles, part_f, part_a, loss_part, loss_dev;
    DevBuf beta, logbeta, cp;  // f32 beta, f32 log beta, f64 selection table
    std::vector<double> beta_host;
    // training
    long long nb = 0;
    DevBuf X, chb, logf, fval, feat, logprior, logq, glogq, g0, g1, thetas, h1s, h2s, gths, gp2s, gp1s, scal;
    double log_fscale = 0;
    bool have_scale = false;
    int adam_t = 0;
    // sampling; the channel-weight network's rows of a sampling chunk
    DevBuf sx0, sx1, sz, su, sch, slq, spart, sfold, fv;
    DevBuf slogf, sfeat, slogprior, sfval;
    // points of the flow path: momenta [leg][4][m], list, count
    DevBuf fmom, flist, fcount;
    DevBuf err;
};

namespace {

constexpr int kNsplit = 48;
constexpr int kAlphaSplit = 148;
constexpr long long kSampleChunk = 1ll << 20;

// Coupling masks: the rule of include/chili_gpu.h ("learned proposal").
void flow_masks(int D, int L, std::vector<std::vector<int>> &cond, std::vector<std::vector<int>> &trans) {
    cond.assign(L, {});
    trans.assign(L, {});
    for (int l = 0; l < L; ++l) {
        std::vector<bool> m(D);
        if (D <= 10) {
            for (int i = 0; i < D; ++i) {
                bool v;
                switch (l % 6) {
                case 0: v = i % 2 == 0; break;
                case 1: v = i % 2 == 1; break;
                case 2: v = i < D / 2; break;
                case 3: v = i >= D / 2; break;
                case 4: v = ((i + 1) / 2) % 2 == 0; break;
                default: v = ((i + 1) / 2) % 2 == 1; break;
                }
                m[i] = v;
            }
            bool all = true, none = true;
            for (int i = 0; i < D; ++i) {
                all = all && m[i];
                none = none && !m[i];
            }
            if (all || none)
                for (int i = 0; i < D; ++i) m[i] = (i % 2) == (l % 2);
        } else {
            for (int i = 0; i < D; ++i) m[i] = true;
            for (int k = 0; k < 5; ++k) m[(5 * l + k) % D] = false;
        }
        for (int i = 0; i < D; ++i) (m[i] ? cond[l] : trans[l]).push_back(i);
    }
}

uint64_t splitmix(uint64_t &s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
double unif_pm1(uint64_t &s) { return (static_cast<double>(splitmix(s) >> 11) * 0x1.0p-53) * 2.0 - 1.0; }

int need_flow(chili_ctx *ctx) {
    if (!ctx->flow) return fail(ctx, CHILI_ERR_STATE, "learned proposal not initialised (chili_gpu_flow_init)");
    return CHILI_OK;
}

template <class K>
int smem_attr(chili_ctx *ctx, K kernel, size_t bytes) {
    CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
    return CHILI_OK;
}

int upload_beta(chili_ctx *ctx) {
    FlowState &S = *ctx->flow;
    std::vector<float> b(S.nch), lb(S.nch);
    std::vector<double> cp(S.nch);
    double tot = 0;
    for (int c = 0; c < S.nch; ++c) tot += S.beta_host[c];
    double acc = 0;
    for (int c = 0; c < S.nch; ++c) {
        const double bc = S.beta_host[c] / tot;
        b[c] = static_cast<float>(bc);
        lb[c] = bc > 0 ? static_cast<float>(std::log(bc)) : -INFINITY;
        acc += bc;
        cp[c] = acc;
    }
    cp[S.nch - 1] = 1.0;
    CK(cudaMemcpyAsync(S.beta.p, b.data(), sizeof(float) * S.nch, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(S.logbeta.p, lb.data(), sizeof(float) * S.nch, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(S.cp.p, cp.data(), sizeof(double) * S.nch, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return CHILI_OK;
}

int pack_tiles(chili_ctx *ctx) {
    FlowState &S = *ctx->flow;
    const float *p = S.prm.as<float>();
    if (int rc = flow_launch_alpha_pack(ctx, p + S.off_alpha, S.AL, S.atiles.as<uint8_t>())) return rc;
    if (S.streamed) {
        for (int l = 0; l < S.L; ++l) {
            WidePackArgs a{};
            a.prm = p;
            a.off_w1 = S.off_w1[l];
            a.off_e = S.off_e[l];
            a.off_w3 = S.off_w3[l];
            for (int k = 0; k < S.NH - 1; ++k) a.off_w2[k] = S.off_w2x[l][k];
            a.H = S.H;
            a.nh = S.NH;
            a.da = S.da[l];
            a.nch = S.nch;
            a.db = S.db[l];
            a.w = S.wtiles.as<uint8_t>() + static_cast<size_t>(l) * wide_layer_bytes(S.H, S.NH);
            if (int rc = flow_launch_pack_wide(ctx, a)) return rc;
        }
        return CHILI_OK;
    }
    for (int l = 0; l < S.L; ++l) {
        uint8_t *wt = S.wtiles.as<uint8_t>() + static_cast<size_t>(l) * kWLayerBytes;
        k_flow_pack<<<(kPF * 128 + 255) / 256, 256, 0, ctx->stream>>>(
            p + S.off_w1[l], p + S.off_e[l], p + S.off_w2[l], p + S.off_w3[l], S.da[l], S.nch, S.db[l] * kPerDim, wt,
            wt + kWBytes);
        LAUNCHED();
    }
    return CHILI_OK;
}

int check_err(chili_ctx *ctx) {
    int e = 0;
    CK(cudaMemcpyAsync(&e, ctx->flow->err.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (e) {
        CK(cudaMemsetAsync(ctx->flow->err.p, 0, sizeof(int), ctx->stream));
        return fail(ctx, CHILI_ERR_TIMEOUT, "tensor-core wait gave up in flow kernel (code " + std::to_string(e) + ")");
    }
    return CHILI_OK;
}

// ------------------------------------------------------------ launches
int launch_wgrad(chili_ctx *ctx, const WgradArgs &a) {
    static bool attr = false;
    if (!attr) {
        if (int rc = smem_attr(ctx, k_flow_wgrad, kWgSmem)) return rc;
        attr = true;
    }
    KTimer kt_(ctx, KT_FLOW_WGRAD);
    k_flow_wgrad<<<dim3(kNsplit, 3), 128, kWgSmem, ctx->stream>>>(a);
    LAUNCHED();
    return CHILI_OK;
}

// ------------------------------------------------------ training buffers
int ensure_train(chili_ctx *ctx, long long n) {
    FlowState &S = *ctx->flow;
    if (S.nb >= n) return CHILI_OK;
    const long long tiles = (n + 127) / 128;
    const size_t fN = sizeof(float) * n;
    CK(S.X.ensure(fN * S.D * (S.L + 1)));
    CK(S.chb.ensure(sizeof(int32_t) * n));
    CK(S.logf.ensure(fN));
    CK(S.fval.ensure(sizeof(double) * n));
    CK(S.feat.ensure(fN * std::max(S.F, 1)));
    CK(S.logprior.ensure(fN * S.nch));
    CK(S.logq.ensure(fN));
    CK(S.glogq.ensure(fN));
    CK(S.g0.ensure(fN * S.D));
    CK(S.g1.ensure(fN * S.D));
    CK(S.thetas.ensure(fN * static_cast<size_t>(kMaxDB * kPerDim) * S.L));
    if (S.streamed) {
        const size_t act = static_cast<size_t>(wide_act_bytes(S.H)) * tiles;
        CK(S.hsw.ensure(act * S.NH * S.L));
        CK(S.gpsw.ensure(act * S.NH));
        CK(S.gthsw.ensure(static_cast<size_t>(tiles) * kGTileW));
        S.nb = n;
        return CHILI_OK;
    }
    CK(S.h1s.ensure(static_cast<size_t>(tiles) * kHTile * S.L));
    CK(S.h2s.ensure(static_cast<size_t>(tiles) * kHTile * S.L));
    CK(S.gths.ensure(static_cast<size_t>(tiles) * kGTile));
    CK(S.gp2s.ensure(static_cast<size_t>(tiles) * kHTile));
    CK(S.gp1s.ensure(static_cast<size_t>(tiles) * kHTile));
    S.nb = n;
    return CHILI_OK;
}

FlowLayer layer_dev(FlowState &S, int l) {
    FlowLayer L = S.layers[l];
    L.wt = S.wtiles.as<uint8_t>() + static_cast<size_t>(l) * kWLayerBytes;
    L.wtf = L.wt + kWBytes;
    L.E = S.prm.as<float>() + S.off_e[l];
    return L;
}

// One coupling layer forward on the kernels of the configured kind (theta
// and the activations saved for the backward pass when save).
int layer_forward(chili_ctx *ctx, int l, int mode, bool save, long long n, const float *xin, float *xout,
                  const int32_t *ch, float *logq, float *theta) {
    FlowState &S = *ctx->flow;
    const long long tiles = (n + 127) / 128;
    if (S.streamed) {
        WideFwdArgs a{};
        a.L = S.wlayers[l];
        a.n = n;
        a.xin = xin;
        a.xout = xout;
        a.ch = ch;
        a.logq = logq;
        if (save) a.hs = S.hsw.as<uint8_t>() + static_cast<size_t>(l) * S.NH * tiles * wide_act_bytes(S.H);
        a.theta = theta;
        a.err = S.err.as<int>();
        return flow_launch_layer_wide(ctx, mode, save, a, S.sms);
    }
    LayerArgs a{};
    a.L = layer_dev(S, l);
    a.n = n;
    a.xin = xin;
    a.xout = xout;
    a.ch = ch;
    a.logq = logq;
    if (save) {
        a.h1s = S.h1s.as<uint8_t>() + static_cast<size_t>(l) * tiles * kHTile;
        a.h2s = S.h2s.as<uint8_t>() + static_cast<size_t>(l) * tiles * kHTile;
    }
    a.theta = theta;
    a.err = S.err.as<int>();
    return flow_launch_layer(ctx, mode, save, a, S.sms);
}

// Backward and weight gradients of coupling layer l on the streamed-weight
// kernels.
int layer_backward_streamed(chili_ctx *ctx, int l, long long n, const float *xin, const float *theta,
                            const float *gout, float *gin) {
    FlowState &S = *ctx->flow;
    const long long tiles = (n + 127) / 128;
    const uint8_t *hs = S.hsw.as<uint8_t>() + static_cast<size_t>(l) * S.NH * tiles * wide_act_bytes(S.H);
    WideBwdArgs b{};
    b.L = S.wlayers[l];
    b.n = n;
    b.xin = xin;
    b.theta = theta;
    b.hs = hs;
    b.gout = gout;
    b.glogq = S.glogq.as<float>();
    b.gin = gin;
    b.gths = S.gthsw.as<uint8_t>();
    b.gps = S.gpsw.as<uint8_t>();
    b.err = S.err.as<int>();
    if (int rc = flow_launch_bwd_wide(ctx, b, S.sms)) return rc;
    WideWgradArgs w{};
    w.n = n;
    w.H = S.H;
    w.nh = S.NH;
    w.da = S.da[l];
    w.db = S.db[l];
    w.nch = S.nch;
    w.ncol2 = ((16 + S.nch) + 63) & ~63;
    for (int i = 0; i < S.da[l]; ++i) w.cond[i] = static_cast<int8_t>(S.cond[l][i]);
    w.xin = xin;
    w.ch = S.chb.as<int32_t>();
    w.hs = hs;
    w.gps = b.gps;
    w.gths = b.gths;
    w.part = S.part_f.as<float>();
    w.nparam = S.np_flow;
    w.off_w1 = S.off_w1[l];
    w.off_e = S.off_e[l];
    w.off_w3 = S.off_w3[l];
    for (int k = 0; k < S.NH - 1; ++k) w.off_w2[k] = S.off_w2x[l][k];
    w.err = S.err.as<int>();
    const int halves = S.H / 128;
    auto add = [&](int kind, int m, int mh, int np) {
        w.item[w.nitems++] = WideWgradItem{static_cast<int8_t>(kind), static_cast<int8_t>(m),
                                           static_cast<int8_t>(mh), static_cast<int8_t>(np)};
    };
    for (int mh = 0; mh < halves; ++mh) {
        add(0, 0, mh, 0);
        if (S.db[l] == 5) add(0, 0, mh, 1);
        for (int m = 0; m < S.NH - 1; ++m) add(1, m, mh, 0);
        add(2, 0, mh, 0);
    }
    return flow_launch_wgrad_wide(ctx, w, kNsplit);
}

// Flow forward (density direction, saving), channel-weight network + loss,
// flow backward and weight gradients, Adam (lr = 0: gradients only, into
// S.grad), the step's loss into loss_dev[slot]. Inputs already in the
// training buffers: X_0 = u, ch, logf, feat, logprior.
int train_pass(chili_ctx *ctx, long long n, float lr, int slot) {
    FlowState &S = *ctx->flow;
    const long long tiles = (n + 127) / 128;
    float *X = S.X.as<float>();
    const size_t xs = static_cast<size_t>(S.D) * n;
    const size_t thn = static_cast<size_t>(kMaxDB * kPerDim) * n;
    CK(cudaMemsetAsync(S.logq.p, 0, sizeof(float) * n, ctx->stream));
    for (int l = 0; l < S.L; ++l)
        if (int rc = layer_forward(ctx, l, 0, true, n, X + xs * l, X + xs * (l + 1), S.chb.as<int32_t>(),
                                   S.logq.as<float>(), S.thetas.as<float>() + thn * l))
            return rc;
    AlphaTcArgs aa{};
    aa.n = n;
    aa.L = S.AL;
    aa.tiles = S.atiles.as<uint8_t>();
    aa.w = S.prm.as<float>() + S.off_alpha;
    aa.feat = S.feat.as<float>();
    aa.logprior = S.logprior.as<float>();
    aa.ch = S.chb.as<int32_t>();
    aa.logf = S.logf.as<float>();
    aa.logbeta = S.logbeta.as<float>();
    aa.logq = S.logq.as<float>();
    aa.glogq = S.glogq.as<float>();
    aa.part = S.part_a.as<float>();
    aa.loss_part = S.loss_part.as<double>();
    aa.err = S.err.as<int>();
    if (int rc = flow_launch_alpha(ctx, aa)) return rc;
    float *gcur = S.g0.as<float>(), *gnext = S.g1.as<float>();
    for (int l = S.L - 1; l >= 0; --l) {
        if (S.streamed) {
            if (int rc = layer_backward_streamed(ctx, l, n, X + xs * l, S.thetas.as<float>() + thn * l,
                                                 l == S.L - 1 ? nullptr : gcur, gnext))
                return rc;
            std::swap(gcur, gnext);
            continue;
        }
        BwdArgs b{};
        b.L = layer_dev(S, l);
        b.n = n;
        b.xin = X + xs * l;
        b.theta = S.thetas.as<float>() + thn * l;
        b.h1s = S.h1s.as<uint8_t>() + static_cast<size_t>(l) * tiles * kHTile;
        b.h2s = S.h2s.as<uint8_t>() + static_cast<size_t>(l) * tiles * kHTile;
        b.gout = l == S.L - 1 ? nullptr : gcur;
        b.glogq = S.glogq.as<float>();
        b.gin = gnext;
        b.gths = S.gths.as<uint8_t>();
        b.gp2s = S.gp2s.as<uint8_t>();
        b.gp1s = S.gp1s.as<uint8_t>();
        b.err = S.err.as<int>();
        if (int rc = flow_launch_bwd(ctx, b, S.sms)) return rc;
        WgradArgs w{};
        w.n = n;
        w.da = S.da[l];
        w.nch = S.nch;
        w.ncol2 = ((16 + S.nch) + 63) & ~63;
        for (int i = 0; i < S.da[l]; ++i) w.cond[i] = static_cast<int8_t>(S.cond[l][i]);
        w.xin = X + xs * l;
        w.ch = S.chb.as<int32_t>();
        w.h1s = b.h1s;
        w.h2s = b.h2s;
        w.gths = b.gths;
        w.gp2s = b.gp2s;
        w.gp1s = b.gp1s;
        w.part = S.part_f.as<float>();
        w.nparam = S.np_flow;
        w.off_w1 = S.off_w1[l];
        w.off_e = S.off_e[l];
        w.off_w2 = S.off_w2[l];
        w.off_w3 = S.off_w3[l];
        w.P = S.db[l] * kPerDim;
        w.err = S.err.as<int>();
        if (int rc = launch_wgrad(ctx, w)) return rc;
        std::swap(gcur, gnext);
    }
    ++S.adam_t;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, static_cast<float>(S.adam_t));
    const float c2 = 1.f - std::pow(b2, static_cast<float>(S.adam_t));
    float *grad = lr == 0.f ? S.grad.as<float>() : nullptr;
    k_flow_adam<<<static_cast<unsigned>((S.np_flow + 255) / 256), 256, 0, ctx->stream>>>(
        S.prm.as<float>(), S.m.as<float>(), S.v.as<float>(), S.part_f.as<float>(), kNsplit, S.np_flow, lr, b1, b2,
        1e-8f, c1, c2, grad);
    LAUNCHED();
    k_flow_adam<<<static_cast<unsigned>((S.AL.total + 255) / 256), 256, 0, ctx->stream>>>(
        S.prm.as<float>() + S.off_alpha, S.m.as<float>() + S.off_alpha, S.v.as<float>() + S.off_alpha,
        S.part_a.as<float>(), kAlphaSplit, S.AL.total, lr, b1, b2, 1e-8f, c1, c2, grad ? grad + S.off_alpha : nullptr);
    LAUNCHED();
    if (lr == 0.f) --S.adam_t;
    else if (int rc = pack_tiles(ctx)) return rc;
    k_loss_fold<<<1, 1, 0, ctx->stream>>>(S.loss_part.as<double>(), kAlphaSplit, 1.0 / static_cast<double>(n),
                                          S.loss_dev.as<double>() + slot);
    LAUNCHED();
    return CHILI_OK;
}

// m points of the flow path. Training (train = true): u uniform and c ~ beta
// from counters ctr0 ..., written to u/ch, and the batch rows (log F,
// features, log prior, F when fval is given). Sampling: u and ch given, the
// rows of the chunk, then the values v of the points (the channel-weight
// network on the tensor cores). Both: VEGAS map, FSMapper, PreProcess, then
// every channel's density through the phased weight pass.
int flow_points(chili_ctx *ctx, bool train, long long m, uint64_t seed, uint64_t ctr0, float *u, int32_t *ch,
                const float *logq, double *fval) {
    FlowState &S = *ctx->flow;
    CK(S.fmom.ensure(sizeof(double) * 4 * S.n_ext * m));
    CK(S.flist.ensure(sizeof(int32_t) * m));
    CK(S.fcount.ensure(sizeof(long long)));
    float *logf = S.logf.as<float>(), *feat = S.feat.as<float>(), *logprior = S.logprior.as<float>();
    if (!train) {
        CK(S.slogf.ensure(sizeof(float) * m));
        CK(S.sfeat.ensure(sizeof(float) * std::max(S.F, 1) * m));
        CK(S.slogprior.ensure(sizeof(float) * S.nch * m));
        CK(S.sfval.ensure(sizeof(double) * m));
        logf = S.slogf.as<float>();
        feat = S.sfeat.as<float>();
        logprior = S.slogprior.as<float>();
        fval = S.sfval.as<double>();
    }
    CK(cudaMemsetAsync(S.fcount.p, 0, sizeof(long long), ctx->stream));
    const unsigned gb = static_cast<unsigned>((m + 127) / 128);
    k_flow_rows_init<<<gb, 128, 0, ctx->stream>>>(m, S.nch, S.F, S.logbeta.as<float>(), logf, feat, logprior, fval);
    LAUNCHED();
    GenArgs g{};
    g.progs = ctx->progs.as<ChannelProgram>();
    g.grids = ctx->edges.as<double>();
    g.cp = S.cp.as<double>();
    g.f = ctx->f_dev.as<IntegrandDesc>();
    g.nch = S.nch;
    g.dims = S.D;
    g.bins = ctx->bins;
    g.n_ext = S.n_ext;
    g.seed = seed;
    g.ctr0 = ctr0;
    g.m = m;
    g.u = u;
    g.ch = ch;
    g.mom_soa = S.fmom.as<double>();
    g.list = S.flist.as<int32_t>();
    g.count = S.fcount.as<long long>();
    {
        KTimer kt_(ctx, KT_FLOW_BATCH);
        if (train) k_flow_gen<true><<<gb, 128, 0, ctx->stream>>>(g);
        else k_flow_gen<false><<<gb, 128, 0, ctx->stream>>>(g);
    }
    LAUNCHED();
    {
        // the listed count stays on the device: the weight pass and the rows
        // are launched for all m points and end at the device's count
        CombineArgs c{};
        c.list = S.flist.as<int32_t>();
        c.count = S.fcount.as<long long>();
        c.m = m;
        c.nch = S.nch;
        c.n_ext = S.n_ext;
        c.sqrts = ctx->sqrts;
        c.f = ctx->f_dev.as<IntegrandDesc>();
        c.beta = S.beta.as<float>();
        c.logbeta = S.logbeta.as<float>();
        c.log_fscale = S.log_fscale;
        c.logf = logf;
        c.fval = fval;
        c.feat = feat;
        c.logprior = logprior;
        if (int rc = pipeline_run(ctx, S.fmom.as<double>(), m, S.flist.as<int32_t>(), ch, S.fcount.as<long long>(),
                                  m, ctx->bins, false, nullptr, nullptr, [&](long long base, long long T) -> int {
                                      CombineArgs t = c;
                                      t.node_soa = ctx->node_soa.as<double>();
                                      t.dcv = ctx->dcv.as<double>();
                                      t.vwv = ctx->vwv.as<double>();
                                      t.ich_tile = ctx->ich_tile.as<int32_t>();
                                      t.base = base;
                                      t.T = T;
                                      return flow_launch_combine(ctx, t, static_cast<unsigned>((T + 127) / 128));
                                  }))
            return rc;
    }
    if (train) return CHILI_OK;
    // the values: alpha_c F / (beta_c q) of every row, 0 for rows without one
    AlphaTcArgs e{};
    e.n = m;
    e.L = S.AL;
    e.tiles = S.atiles.as<uint8_t>();
    e.w = S.prm.as<float>() + S.off_alpha;
    e.feat = feat;
    e.logprior = logprior;
    e.ch = ch;
    e.logf = logf;
    e.logbeta = S.logbeta.as<float>();
    e.logq = logq;
    e.fval = fval;
    e.v = S.fv.as<double>();
    e.err = S.err.as<int>();
    return flow_launch_alpha_eval(ctx, e, S.sms);
}

// The flow over n points (xin, xout [D][n] on the device): the layers in
// order (mode 0, density direction) or in reverse (mode 1, sampling).
int flow_pass(chili_ctx *ctx, const float *xin_dev, const int32_t *ch_dev, long long n, int mode, float *xout_dev,
              float *logq_dev) {
    FlowState &S = *ctx->flow;
    const size_t xs = static_cast<size_t>(S.D) * n;
    CK(S.sx0.ensure(sizeof(float) * xs));
    CK(S.sx1.ensure(sizeof(float) * xs));
    CK(cudaMemsetAsync(logq_dev, 0, sizeof(float) * n, ctx->stream));
    const float *cur = xin_dev;
    float *bufs[2] = {S.sx0.as<float>(), S.sx1.as<float>()};
    for (int k = 0; k < S.L; ++k) {
        const int l = mode == 0 ? k : S.L - 1 - k;
        float *out = k == S.L - 1 ? xout_dev : bufs[k & 1];
        if (int rc = layer_forward(ctx, l, mode, false, n, cur, out, ch_dev, logq_dev, nullptr)) return rc;
        cur = out;
    }
    return CHILI_OK;
}

}  // namespace

void flow_release(chili_ctx *ctx) {
    if (!ctx || !ctx->flow) return;
    FlowState &S = *ctx->flow;
    for (DevBuf *b : {&S.prm, &S.m, &S.v, &S.grad, &S.wtiles, &S.atiles, &S.slogf, &S.sfeat, &S.slogprior, &S.sfval,
                      &S.part_f, &S.part_a, &S.loss_part, &S.loss_dev,
                      &S.beta, &S.logbeta, &S.cp, &S.X, &S.chb, &S.logf, &S.fval, &S.feat, &S.logprior, &S.logq,
                      &S.glogq, &S.g0, &S.g1, &S.thetas, &S.h1s, &S.h2s, &S.gths, &S.gp2s, &S.gp1s, &S.scal,
                      &S.hsw, &S.gpsw, &S.gthsw,
                      &S.sx0, &S.sx1, &S.sz, &S.su, &S.sch, &S.slq, &S.spart, &S.sfold, &S.fv,
                      &S.fmom, &S.flist, &S.fcount, &S.err})
        b->release();
    delete ctx->flow;
    ctx->flow = nullptr;
}

extern "C" {

int chili_gpu_flow_init(chili_ctx *ctx, const chili_flow_params *params) {
    if (!ctx || !params) return fail(ctx, CHILI_ERR_INVALID_ARG, "null argument");
    if (int rc = set_device(ctx)) return rc;
    if (int rc = need_channels(ctx)) return rc;
    if (int rc = need_grids(ctx)) return rc;
    if (!ctx->f_set) return fail(ctx, CHILI_ERR_STATE, "no integrand set");
    if (!ctx->have_pp) return fail(ctx, CHILI_ERR_LIMIT, "channel set exceeds the point-program limits");
    if (ctx->g_nch != ctx->nch || ctx->dims != ctx->ndims)
        return fail(ctx, CHILI_ERR_STATE, "grids do not match the channel set");
    if (params->layers < 1 || params->layers > 32 || params->batch < 128 || params->batch > (1 << 24))
        return fail(ctx, CHILI_ERR_INVALID_ARG, "layers in [1, 32], batch in [128, 2^24]");
    const int F = n_features(ctx->n_ext);
    if (ctx->nch > kMaxFlowCh || F > kMaxFeat - 1)
        return fail(ctx, CHILI_ERR_LIMIT, "learned proposal limited to 48 channels and 31 features");
    flow_release(ctx);
    ctx->flow = new FlowState();
    FlowState &S = *ctx->flow;
    S.D = ctx->ndims;
    S.nch = ctx->nch;
    S.L = params->layers;
    S.F = F;
    S.n_ext = ctx->n_ext;
    S.batch = params->batch;
    S.lr = static_cast<float>(params->lr);
    S.H = params->hidden ? params->hidden : kH;
    S.NH = params->depth ? params->depth : 2;
    if ((S.H != 128 && S.H != 256) || S.NH < 2 || S.NH > kWMaxNH) {
        flow_release(ctx);
        return fail(ctx, CHILI_ERR_INVALID_ARG, "conditioner: hidden 128 or 256, depth 2..4");
    }
    S.streamed = S.H != kH || S.NH != 2 || ctx->flow_streamed;
    cudaDeviceGetAttribute(&S.sms, cudaDevAttrMultiProcessorCount, ctx->device);
    flow_masks(S.D, S.L, S.cond, S.trans);
    long long off = 0;
    S.layers.resize(S.L);
    for (int l = 0; l < S.L; ++l) {
        const int da = static_cast<int>(S.cond[l].size()), db = static_cast<int>(S.trans[l].size());
        if (da > kMaxDA || db > kMaxDB || da < 1 || db < 1) {
            flow_release(ctx);
            return fail(ctx, CHILI_ERR_LIMIT, "coupling split outside 1..16 conditioning / 1..5 transformed dims");
        }
        S.da.push_back(da);
        S.db.push_back(db);
        FlowLayer &L = S.layers[l];
        std::memset(&L, 0, sizeof(L));
        L.da = da;
        L.db = db;
        L.nch = S.nch;
        for (int i = 0; i < da; ++i) L.cond[i] = static_cast<int8_t>(S.cond[l][i]);
        for (int j = 0; j < db; ++j) L.trans[j] = static_cast<int8_t>(S.trans[l][j]);
        const long long H = S.H;
        S.off_w1.push_back(off);
        off += H * da;
        S.off_e.push_back(off);
        off += S.nch * H;
        S.off_w2.push_back(off);
        S.off_w2x.emplace_back();
        for (int k = 0; k < S.NH - 1; ++k) {
            S.off_w2x.back().push_back(off);
            off += H * H;
        }
        S.off_w3.push_back(off);
        off += db * kPerDim * H;
        WideLayer W{};
        W.H = S.H;
        W.nh = S.NH;
        W.da = da;
        W.db = db;
        W.nch = S.nch;
        for (int i = 0; i < da; ++i) W.cond[i] = L.cond[i];
        for (int j = 0; j < db; ++j) W.trans[j] = L.trans[j];
        S.wlayers.push_back(W);
    }
    S.np_flow = off;
    S.off_alpha = off;
    S.AL = alpha_layout(F, S.nch);
    S.np = off + S.AL.total;
    // initial parameters: identity flow, channel weights = the prior
    std::vector<float> p(S.np, 0.f);
    uint64_t rs = params->init_seed;
    for (int l = 0; l < S.L; ++l) {
        const int da = S.da[l], db = S.db[l];
        const int H = S.H;
        const double b1 = std::sqrt(6.0 / da), b2 = std::sqrt(6.0 / H);
        for (int i = 0; i < H * da; ++i) p[S.off_w1[l] + i] = static_cast<float>(b1 * unif_pm1(rs));
        for (int k = 0; k < S.NH - 1; ++k)
            for (int i = 0; i < H * H; ++i) p[S.off_w2x[l][k] + i] = static_cast<float>(b2 * unif_pm1(rs));
        const float did = static_cast<float>(std::log(std::expm1(1.0 - 1e-3)));
        for (int j = 0; j < db; ++j)
            for (int k = 0; k <= kBins; ++k) p[S.off_w3[l] + (j * kPerDim + 2 * kBins + k) * H + (H - 1)] = did;
    }
    {
        const double ba1 = std::sqrt(6.0 / F), ba2 = std::sqrt(6.0 / kAH);
        for (int i = 0; i < kAH * F; ++i) p[S.off_alpha + S.AL.a1 + i] = static_cast<float>(ba1 * unif_pm1(rs));
        for (int i = 0; i < kAH * kAH; ++i) p[S.off_alpha + S.AL.a2 + i] = static_cast<float>(ba2 * unif_pm1(rs));
    }
    CK(S.prm.ensure(sizeof(float) * S.np));
    CK(S.m.ensure(sizeof(float) * S.np));
    CK(S.v.ensure(sizeof(float) * S.np));
    CK(S.grad.ensure(sizeof(float) * S.np));
    CK(cudaMemcpyAsync(S.prm.p, p.data(), sizeof(float) * S.np, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemsetAsync(S.m.p, 0, sizeof(float) * S.np, ctx->stream));
    CK(cudaMemsetAsync(S.v.p, 0, sizeof(float) * S.np, ctx->stream));
    const size_t wbytes = static_cast<size_t>(S.L) * (S.streamed ? wide_layer_bytes(S.H, S.NH) : kWLayerBytes);
    CK(S.wtiles.ensure(wbytes));
    CK(cudaMemsetAsync(S.wtiles.p, 0, wbytes, ctx->stream));
    CK(S.atiles.ensure(kAWBytes));
    for (int l = 0; l < S.L; ++l)
        S.wlayers[l].w = S.wtiles.as<uint8_t>() + static_cast<size_t>(l) * wide_layer_bytes(S.H, S.NH);
    CK(S.part_f.ensure(sizeof(float) * kNsplit * S.np_flow));
    CK(S.part_a.ensure(sizeof(float) * kAlphaSplit * S.AL.total));
    CK(S.loss_part.ensure(sizeof(double) * kAlphaSplit));
    CK(S.loss_dev.ensure(sizeof(double) * 4096));
    CK(S.beta.ensure(sizeof(float) * S.nch));
    CK(S.logbeta.ensure(sizeof(float) * S.nch));
    CK(S.cp.ensure(sizeof(double) * S.nch));
    CK(S.err.ensure(sizeof(int)));
    CK(cudaMemsetAsync(S.err.p, 0, sizeof(int), ctx->stream));
    CK(S.scal.ensure(sizeof(double) * 2));
    // beta = the multichannel channel weights
    S.beta_host.assign(S.nch, 1.0 / S.nch);
    if (ctx->alpha_set) {
        std::vector<double> a(S.nch);
        CK(cudaMemcpyAsync(a.data(), alpha_ptr(ctx), sizeof(double) * S.nch, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        double tot = 0;
        for (double x : a) tot += x;
        if (tot > 0 && std::isfinite(tot)) S.beta_host = a;
    }
    if (int rc = upload_beta(ctx)) return rc;
    if (int rc = pack_tiles(ctx)) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return CHILI_OK;
}

int64_t chili_gpu_flow_nparams(const chili_ctx *ctx) { return (ctx && ctx->flow) ? ctx->flow->np : -1; }

int chili_gpu_flow_get_params(chili_ctx *ctx, float *prm) {
    if (!ctx || !prm) return fail(ctx, CHILI_ERR_INVALID_ARG, "null argument");
    if (int rc = need_flow(ctx)) return rc;
    if (int rc = set_device(ctx)) return rc;
    Arg o;
    if (int rc = resolve(ctx, prm, sizeof(float) * ctx->flow->np, 0, false, o)) return rc;
    CK(cudaMemcpyAsync(o.dev, ctx->flow->prm.p, o.bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    if (int rc = finish_out(ctx, o)) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return CHILI_OK;
}

int chili_gpu_flow_set_params(chili_ctx *ctx, const float *prm) {
    if (!ctx || !prm) return fail(ctx, CHILI_ERR_INVALID_ARG, "null argument");
    if (int rc = need_flow(ctx)) return rc;
    if (int rc = set_device(ctx)) return rc;
    Arg in;
    if (int rc = resolve(ctx, prm, sizeof(float) * ctx->flow->np, 0, true, in)) return rc;
    CK(cudaMemcpyAsync(ctx->flow->prm.p, in.dev, in.bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemsetAsync(ctx->flow->m.p, 0, sizeof(float) * ctx->flow->np, ctx->stream));
    CK(cudaMemsetAsync(ctx->flow->v.p, 0, sizeof(float) * ctx->flow->np, ctx->stream));
    ctx->flow->adam_t = 0;
    if (int rc = pack_tiles(ctx)) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return CHILI_OK;
}

int chili_gpu_flow_get_beta(chili_ctx *ctx, double *beta) {
    if (!ctx || !beta) return fail(ctx, CHILI_ERR_INVALID_ARG, "null argument");
    if (int rc = need_flow(ctx)) return rc;
    double tot = 0;
    for (double b : ctx->flow->beta_host) tot += b;
    for (int c = 0; c < ctx->flow->nch; ++c) beta[c] = ctx->flow->beta_host[c] / tot;
    return CHILI_OK;
}

int chili_gpu_flow_set_beta(chili_ctx *ctx, const double *beta) {
    if (!ctx || !beta) return fail(ctx, CHILI_ERR_INVALID_ARG, "null argument");
    if (int rc = need_flow(ctx)) return rc;
    if (int rc = set_device(ctx)) return rc;
    double tot = 0;
    for (int c = 0; c < ctx->flow->nch; ++c) {
        if (!(beta[c] >= 0) || !std::isfinite(beta[c]))
            return fail(ctx, CHILI_ERR_INVALID_ARG, "beta must be finite and >= 0");
        tot += beta[c];
    }
    if (!(tot > 0)) return fail(ctx, CHILI_ERR_INVALID_ARG, "beta sums to 0");
    ctx->flow->beta_host.assign(beta, beta + ctx->flow->nch);
    return upload_beta(ctx);
}

static int density_or_sample(chili_ctx *ctx, const float *xin, const int32_t *ch, int64_t n, float *xout, float *logq,
                             int mode) {
    if (!ctx || !xin || !ch || n <= 0) return fail(ctx, CHILI_ERR_INVALID_ARG, "null argument or n <= 0");
    if (int rc = need_flow(ctx)) return rc;
    if (int rc = set_device(ctx)) return rc;
    FlowState &S = *ctx->flow;
    const size_t xb = sizeof(float) * S.D * n;
    Arg ai, ac, ao, aq;
    if (int rc = resolve(ctx, xin, xb, 0, true, ai)) return rc;
    if (int rc = resolve(ctx, ch, sizeof(int32_t) * n, 1, true, ac)) return rc;
    if (int rc = resolve(ctx, xout, xout ? xb : 0, 2, false, ao)) return rc;
    if (int rc = resolve(ctx, logq, logq ? sizeof(float) * n : 0, 3, false, aq)) return rc;
    CK(S.sz.ensure(xb));
    CK(S.su.ensure(xb));
    CK(S.slq.ensure(sizeof(float) * n));
    k_transpose_f<<<static_cast<unsigned>((n * S.D + 255) / 256), 256, 0, ctx->stream>>>(
        static_cast<const float *>(ai.dev), S.sz.as<float>(), n, S.D, 1);
    LAUNCHED();
    if (int rc = flow_pass(ctx, S.sz.as<float>(), static_cast<const int32_t *>(ac.dev), n, mode, S.su.as<float>(),
                           S.slq.as<float>()))
        return rc;
    if (ao.dev) {
        k_transpose_f<<<static_cast<unsigned>((n * S.D + 255) / 256), 256, 0, ctx->stream>>>(
            S.su.as<float>(), static_cast<float *>(ao.dev), n, S.D, 0);
        LAUNCHED();
    }
    if (aq.dev) CK(cudaMemcpyAsync(aq.dev, S.slq.p, sizeof(float) * n, cudaMemcpyDeviceToDevice, ctx->stream));
    if (int rc = finish_out(ctx, ao)) return rc;
    if (int rc = finish_out(ctx, aq)) return rc;
    return check_err(ctx);
}

int chili_gpu_flow_density(chili_ctx *ctx, const float *u, const int32_t *ch, int64_t n, float *z, float *logq) {
    return density_or_sample(ctx, u, ch, n, z, logq, 0);
}

int chili_gpu_flow_sample_u(chili_ctx *ctx, const float *z, const int32_t *ch, int64_t n, float *u, float *logq) {
    return density_or_sample(ctx, z, ch, n, u, logq, 1);
}

int chili_gpu_flow_loss_grad(chili_ctx *ctx, const float *u, const int32_t *ch, const float *logf,
                             const float *feat, const float *logprior, int64_t n, double *loss, float *grad) {
    if (!ctx || !u || !ch || !logf || !feat || !logprior || n < 128)
        return fail(ctx, CHILI_ERR_INVALID_ARG, "null argument or n < 128");
    if (int rc = need_flow(ctx)) return rc;
    if (int rc = set_device(ctx)) return rc;
    FlowState &S = *ctx->flow;
    if (int rc = ensure_train(ctx, n)) return rc;
    Arg au, ac, al, af, ap;
    if (int rc = resolve(ctx, u, sizeof(float) * S.D * n, 0, true, au)) return rc;
    if (int rc = resolve(ctx, ch, sizeof(int32_t) * n, 1, true, ac)) return rc;
    if (int rc = resolve(ctx, logf, sizeof(float) * n, 2, true, al)) return rc;
    if (int rc = resolve(ctx, feat, sizeof(float) * S.F * n, 3, true, af)) return rc;
    if (int rc = resolve(ctx, logprior, sizeof(float) * S.nch * n, 4, true, ap)) return rc;
    const unsigned g = static_cast<unsigned>((n * std::max(S.D, std::max(S.F, S.nch)) + 255) / 256);
    k_transpose_f<<<g, 256, 0, ctx->stream>>>(static_cast<const float *>(au.dev), S.X.as<float>(), n, S.D, 1);
    LAUNCHED();
    k_transpose_f<<<g, 256, 0, ctx->stream>>>(static_cast<const float *>(af.dev), S.feat.as<float>(), n, S.F, 1);
    LAUNCHED();
    k_transpose_f<<<g, 256, 0, ctx->stream>>>(static_cast<const float *>(ap.dev), S.logprior.as<float>(), n, S.nch, 1);
    LAUNCHED();
    CK(cudaMemcpyAsync(S.chb.p, ac.dev, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(S.logf.p, al.dev, sizeof(float) * n, cudaMemcpyDeviceToDevice, ctx->stream));
    if (int rc = train_pass(ctx, n, 0.f, 0)) return rc;
    if (int rc = check_err(ctx)) return rc;
    if (loss) CK(cudaMemcpy(loss, S.loss_dev.p, sizeof(double), cudaMemcpyDeviceToHost));
    if (grad) {
        Arg ag;
        if (int rc = resolve(ctx, grad, sizeof(float) * S.np, 5, false, ag)) return rc;
        CK(cudaMemcpyAsync(ag.dev, S.grad.p, sizeof(float) * S.np, cudaMemcpyDeviceToDevice, ctx->stream));
        if (int rc = finish_out(ctx, ag)) return rc;
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return CHILI_OK;
}

int chili_gpu_flow_train(chili_ctx *ctx, int steps, uint64_t seed, uint64_t counter_base, double *loss) {
    if (!ctx || steps < 0 || steps > 4096) return fail(ctx, CHILI_ERR_INVALID_ARG, "steps in [0, 4096]");
    if (int rc = need_flow(ctx)) return rc;
    if (int rc = set_device(ctx)) return rc;
    FlowState &S = *ctx->flow;
    const long long n = S.batch;
    if (int rc = ensure_train(ctx, n)) return rc;
    if (!S.have_scale) {
        // F scale: mean of F over one batch of the plain proposal
        if (int rc = flow_points(ctx, true, n, seed, counter_base, S.X.as<float>(), S.chb.as<int32_t>(), nullptr,
                                 S.fval.as<double>()))
            return rc;
        k_sum_pos<<<1, 256, 0, ctx->stream>>>(S.fval.as<double>(), n, S.scal.as<double>());
        LAUNCHED();
        double sc[2];
        CK(cudaMemcpyAsync(sc, S.scal.p, sizeof(sc), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        const double mean = sc[0] / static_cast<double>(n);
        S.log_fscale = (mean > 0 && std::isfinite(mean)) ? std::log(mean) : 0.0;
        S.have_scale = true;
    }
    for (int s = 0; s < steps; ++s) {
        if (int rc = flow_points(ctx, true, n, seed, counter_base + static_cast<uint64_t>(s) * n, S.X.as<float>(),
                                 S.chb.as<int32_t>(), nullptr, nullptr))
            return rc;
        if (int rc = train_pass(ctx, n, S.lr, s)) return rc;
    }
    if (int rc = check_err(ctx)) return rc;
    if (loss && steps > 0) {
        Arg o;
        if (int rc = resolve(ctx, loss, sizeof(double) * steps, 0, false, o)) return rc;
        CK(cudaMemcpyAsync(o.dev, S.loss_dev.p, sizeof(double) * steps, cudaMemcpyDeviceToDevice, ctx->stream));
        if (int rc = finish_out(ctx, o)) return rc;
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return CHILI_OK;
}

int chili_gpu_flow_iterate(chili_ctx *ctx, uint64_t ncalls, uint64_t seed, uint64_t counter_base, int adapt_beta,
                           chili_stats *stats_out, chili_flow_iter_info *info) {
    if (!ctx || ncalls < 1 || ncalls > (1ull << 40)) return fail(ctx, CHILI_ERR_INVALID_ARG, "ncalls in [1, 2^40]");
    if (int rc = need_flow(ctx)) return rc;
    if (int rc = set_device(ctx)) return rc;
    FlowState &S = *ctx->flow;
    const int width = kPhysFixed + 2 * S.nch;
    const long long chunk = std::min<long long>(kSampleChunk, static_cast<long long>(ncalls));
    const unsigned blocks = static_cast<unsigned>((chunk + kPhysBlock - 1) / kPhysBlock);
    const size_t xs = static_cast<size_t>(S.D) * chunk;
    CK(S.sch.ensure(sizeof(int32_t) * chunk));
    CK(S.slq.ensure(sizeof(float) * chunk));
    CK(S.spart.ensure(sizeof(double) * blocks * width));
    CK(S.sfold.ensure(sizeof(double) * width));
    CK(S.sz.ensure(sizeof(float) * xs));
    CK(S.su.ensure(sizeof(float) * xs));
    CK(S.fv.ensure(sizeof(double) * chunk));
    std::vector<double> tot(width, 0.0), fold(width);
    for (uint64_t done = 0; done < ncalls;) {
        const long long m = std::min<long long>(chunk, static_cast<long long>(ncalls - done));
        k_flow_draw<<<static_cast<unsigned>((m + 255) / 256), 256, 0, ctx->stream>>>(
            S.cp.as<double>(), S.nch, S.D, seed, counter_base + done, m, S.sz.as<float>(), S.sch.as<int32_t>(),
            S.slq.as<float>(), S.fv.as<double>());
        LAUNCHED();
        if (int rc = flow_pass(ctx, S.sz.as<float>(), S.sch.as<int32_t>(), m, 1, S.su.as<float>(), S.slq.as<float>()))
            return rc;
        if (int rc = flow_points(ctx, false, m, seed, 0, S.su.as<float>(), S.sch.as<int32_t>(), S.slq.as<float>(),
                                 nullptr))
            return rc;
        const unsigned nbk = static_cast<unsigned>((m + kPhysBlock - 1) / kPhysBlock);
        k_flow_stats<<<nbk, kPhysBlock, 0, ctx->stream>>>(S.fv.as<double>(), S.sch.as<int32_t>(), S.beta.as<float>(),
                                                          S.nch, m, S.spart.as<double>());
        LAUNCHED();
        k_flow_fold<<<static_cast<unsigned>(width), 256, 0, ctx->stream>>>(S.spart.as<double>(),
                                                                            static_cast<int>(nbk), width,
                                                                            S.sfold.as<double>());
        LAUNCHED();
        CK(cudaMemcpyAsync(fold.data(), S.sfold.p, sizeof(double) * width, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        for (int q = 0; q < width; ++q) tot[q] = q == 3 ? std::max(tot[q], fold[q]) : tot[q] + fold[q];
        done += static_cast<uint64_t>(m);
    }
    if (int rc = check_err(ctx)) return rc;
    if (stats_out) {
        stats_out->n = tot[0];
        stats_out->min = 0;
        stats_out->max = tot[3];
        stats_out->sum = tot[1];
        stats_out->sum2 = tot[2];
        stats_out->n_finite = tot[4];
    }
    if (info) {
        info->points = static_cast<uint64_t>(tot[0]);
        info->nonzero = static_cast<uint64_t>(tot[4]);
        info->nonfinite = static_cast<uint64_t>(tot[5]);
        info->weight_max = tot[3];
        info->unweighting_efficiency = tot[3] > 0 ? (tot[1] / tot[0]) / tot[3] : 0.0;
    }
    if (adapt_beta) {
        std::vector<double> nb(S.nch);
        double mx = 0;
        for (int c = 0; c < S.nch; ++c) {
            const double nc = tot[kPhysFixed + c], t2 = tot[kPhysFixed + S.nch + c];
            nb[c] = nc > 0 ? std::sqrt(t2 / nc) : 0.0;
            mx = std::max(mx, nb[c]);
        }
        if (mx > 0) {
            for (int c = 0; c < S.nch; ++c) nb[c] = std::max(nb[c], 1e-4 * mx);
            S.beta_host = nb;
            if (int rc = upload_beta(ctx)) return rc;
        }
    }
    return CHILI_OK;
}

int chili_gpu_tc_selftest(chili_ctx *ctx, int mode, int K, int N, const float *A, const float *B, float *C) {
    if (!ctx || !A || !B || !C) return fail(ctx, CHILI_ERR_INVALID_ARG, "null argument");
    if (mode < 0 || mode > 3 || K < 16 || K > 256 || K % 16 || N < 16 || N > 256 || N % 16)
        return fail(ctx, CHILI_ERR_INVALID_ARG, "mode 0..3, K and N multiples of 16 in [16, 256]");
    if (int rc = set_device(ctx)) return rc;
    const size_t na = 128 * static_cast<size_t>(K), nbb = static_cast<size_t>(N) * K, nc = 128 * static_cast<size_t>(N);
    DevBuf &da = ctx->stage[0], &db = ctx->stage[1], &dc = ctx->stage[2], &de = ctx->stage[3];
    CK(da.ensure(sizeof(float) * na));
    CK(db.ensure(sizeof(float) * nbb));
    CK(dc.ensure(sizeof(float) * nc));
    CK(de.ensure(sizeof(int)));
    CK(cudaMemcpyAsync(da.p, A, sizeof(float) * na, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(db.p, B, sizeof(float) * nbb, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemsetAsync(de.p, 0, sizeof(int), ctx->stream));
    CK(cudaFuncSetAttribute(k_tc_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, kSelftestSmem));
    k_tc_selftest<<<1, 128, kSelftestSmem, ctx->stream>>>(mode, K, N, da.as<float>(), db.as<float>(), dc.as<float>(),
                                                          de.as<int>());
    LAUNCHED();
    int e = 0;
    CK(cudaMemcpyAsync(C, dc.p, sizeof(float) * nc, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(&e, de.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (e) return fail(ctx, CHILI_ERR_TIMEOUT, "tensor-core self test: wait gave up");
    return CHILI_OK;
}

}  // extern "C"
