// flow_phys.cuh -- the FP64 phase-space side of the learned proposal and its
// channel-weight network.
//
// Estimator (multi-channel importance sampling with point-dependent channel
// weights, Heimel et al., "MadNIS", SciPost Phys. 15 (2023) 141): channel c is
// drawn with probability beta_c, u from the channel's flow q_c, x = VEGAS_c(u)
// (Jacobian J), p = FSMapper_c(x); the point's value is
//     v = alpha_c(p) f(p) dens_c(p) J / (beta_c q_c(u)),
// dens_c the reference's FSMapper weight of channel c at p (Channel.cc:40-61).
// For any alpha(p) >= 0 with sum_c alpha_c(p) = 1, E[v] is the integral.
//
// alpha(p) = softmax(MLP(phi(p)) + log prior(p)): phi = log pair invariants
// log(s_ij/S) and log(|t_1j|/S) of the outgoing legs, scaled to ~[-1, 1];
// prior_c = beta_c g_c(p) / sum_k beta_k g_k(p), g_k = 1/D_k the channels'
// densities (Integrand::GenerateWeight, Integrand.hh:112-123). With the last
// layer zero and the flow the identity, v = f(p) / sum_k beta_k g_k(p): the
// plain multichannel estimator itself, which training then improves on.
#pragma once

#include <math_constants.h>

#include "flow.cuh"
#include "mc_device.cuh"

namespace chili_flow {

using namespace chili_dev;

constexpr int kAH = 64;        // hidden units of the channel-weight network
constexpr int kMaxFeat = 32;
constexpr int kMaxAlphaCh = 64;
constexpr int kAlphaBlock = 64;

// Offsets of the channel-weight network's parameters in its flat f32 block.
struct AlphaLayout {
    int F, nch;
    int a1, c1, a2, c2, a3, c3, total;
};

__host__ __device__ inline AlphaLayout alpha_layout(int F, int nch) {
    AlphaLayout L;
    L.F = F;
    L.nch = nch;
    L.a1 = 0;
    L.c1 = L.a1 + kAH * F;
    L.a2 = L.c1 + kAH;
    L.c2 = L.a2 + kAH * kAH;
    L.a3 = L.c2 + kAH;
    L.c3 = L.a3 + nch * kAH;
    L.total = L.c3 + nch;
    return L;
}

__host__ __device__ inline int n_features(int n_ext) {
    const int n_out = n_ext - 2;
    return n_out * (n_out - 1) / 2 + n_out;
}

// Features of one point (momenta mom[0..n_ext)).
__device__ __forceinline__ void point_features(const V4 *mom, int n_ext, double sqrts, float *feat) {
    const double S = sqrts * sqrts;
    int f = 0;
    for (int i = 2; i < n_ext; ++i)
        for (int j = i + 1; j < n_ext; ++j) {
            const double s = mass2(mom[i] + mom[j]) / S;
            feat[f++] = static_cast<float>(log(fmax(s, 1e-12)) / 8.0 + 1.0);
        }
    for (int j = 2; j < n_ext; ++j) {
        const double tt = fabs(mass2(mom[0] + mom[j])) / S;
        feat[f++] = static_cast<float>(log(fmax(tt, 1e-12)) / 8.0 + 1.0);
    }
}

__device__ __forceinline__ V4 soa_v4(const double *__restrict__ soa, int s, long long m, long long i) {
    return V4{soa[(4 * s + 0) * m + i], soa[(4 * s + 1) * m + i], soa[(4 * s + 2) * m + i],
              soa[(4 * s + 3) * m + i]};
}

// Channel-weight network forward for one point: the logits of every channel
// and their log-sum-exp.
template <int NCH, int NF>
__device__ __forceinline__ void alpha_forward(const float *__restrict__ w, const AlphaLayout &L, const float (&feat)[NF],
                                              const float *logprior, float (&a1)[kAH], float (&a2)[kAH],
                                              float (&lg)[NCH], float &lse) {
#pragma unroll 4
    for (int i = 0; i < kAH; ++i) {
        float s = w[L.c1 + i];
#pragma unroll
        for (int f = 0; f < NF; ++f)
            if (f < L.F) s += w[L.a1 + i * L.F + f] * feat[f];
        a1[i] = lrelu(s);
    }
#pragma unroll 4
    for (int j = 0; j < kAH; ++j) {
        float s = w[L.c2 + j];
#pragma unroll
        for (int i = 0; i < kAH; ++i) s += w[L.a2 + j * kAH + i] * a1[i];
        a2[j] = lrelu(s);
    }
    float mx = -INFINITY;
#pragma unroll
    for (int k = 0; k < NCH; ++k) {
        float s = -INFINITY;
        if (k < L.nch) {
            s = w[L.c3 + k] + logprior[k];
#pragma unroll
            for (int j = 0; j < kAH; ++j) s += w[L.a3 + k * kAH + j] * a2[j];
        }
        lg[k] = s;
        mx = fmaxf(mx, s);
    }
    float se = 0.f;
#pragma unroll
    for (int k = 0; k < NCH; ++k)
        if (k < L.nch) se += expf(lg[k] - mx);
    lse = mx + logf(se);
}

// Channel-weight network: forward, variance-loss terms, backward, weight
// gradients (this block's partial), for one training batch. Also writes
// d loss / d log q for the flow's backward pass.
//   l_i = alpha_c^2 F^2 / (beta_c^2 q)  (F = f dens J / F_scale), loss = mean l_i
struct AlphaTrainArgs {
    long long n;
    AlphaLayout L;
    const float *w;         // parameters (flat)
    const float *feat;      // [F][n]
    const float *logprior;  // [nch][n]
    const int32_t *ch;
    const float *logf;      // [n], -inf for a zero / invalid point
    const float *logbeta;   // [nch]
    const float *logq;      // [n]
    float *glogq;           // [n]
    float *part;            // [gridDim.x][L.total]
    double *loss_part;      // [gridDim.x]
};

template <int NCH, int NF>
__global__ void __launch_bounds__(kAlphaBlock) k_alpha_train(AlphaTrainArgs a) {
    constexpr int R = kAlphaBlock, LD = kAH + 1, LF = NF + 1, LC = NCH + 1;
    extern __shared__ float sa[];
    const AlphaLayout L = a.L;
    float *w = sa;                        // L.total
    float *s_a1 = w + ((L.total + 3) & ~3);
    float *s_a2 = s_a1 + R * LD;
    float *s_g1 = s_a2 + R * LD;
    float *s_g2 = s_g1 + R * LD;
    float *s_gl = s_g2 + R * LD;          // [R][NCH+1]
    float *s_f = s_gl + R * LC;           // [R][NF+1]
    const int t = threadIdx.x;
    for (int i = t; i < L.total; i += R) w[i] = a.w[i];
    __syncthreads();
    float acc2[kAH], acc3[NCH], acc1[NF];
#pragma unroll
    for (int i = 0; i < kAH; ++i) acc2[i] = 0.f;
#pragma unroll
    for (int k = 0; k < NCH; ++k) acc3[k] = 0.f;
#pragma unroll
    for (int f = 0; f < NF; ++f) acc1[f] = 0.f;
    float gc1 = 0.f, gc2 = 0.f, gc3 = 0.f;
    double lsum = 0.0;
    const long long ntiles = (a.n + R - 1) / R;
    const float invn = 1.f / static_cast<float>(a.n);
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long long row = tile * R + t;
        const bool valid = row < a.n;
        float lg[NCH], lse;
        {
            float feat[NF], lp[NCH];
#pragma unroll
            for (int f = 0; f < NF; ++f) feat[f] = (valid && f < L.F) ? a.feat[f * a.n + row] : 0.f;
#pragma unroll
            for (int k = 0; k < NCH; ++k) lp[k] = (valid && k < L.nch) ? a.logprior[k * a.n + row] : 0.f;
            float a1[kAH], a2[kAH];
            alpha_forward<NCH, NF>(w, L, feat, lp, a1, a2, lg, lse);
#pragma unroll
            for (int i = 0; i < kAH; ++i) {
                s_a1[t * LD + i] = a1[i];
                s_a2[t * LD + i] = a2[i];
            }
#pragma unroll
            for (int f = 0; f < NF; ++f) s_f[t * LF + f] = feat[f];
        }
        int c = valid ? a.ch[row] : 0;
        c = (c >= 0 && c < L.nch) ? c : 0;
        float lac = lg[0];
#pragma unroll
        for (int k = 1; k < NCH; ++k)
            if (k == c) lac = lg[k];
        lac -= lse;
        float ell = 0.f;
        if (valid) {
            const float e = 2.f * lac + 2.f * a.logf[row] - 2.f * a.logbeta[c] - a.logq[row];
            ell = isfinite(e) ? expf(e) : 0.f;
            if (!isfinite(ell)) ell = 0.f;
            a.glogq[row] = -ell * invn;
        }
        lsum += ell;
        const float gsel = 2.f * ell * invn;
        // g_logits = gsel (delta_kc - alpha_k)
#pragma unroll
        for (int k = 0; k < NCH; ++k) {
            const float al = k < L.nch ? expf(lg[k] - lse) : 0.f;
            lg[k] = gsel * ((k == c ? 1.f : 0.f) - al);
            s_gl[t * LC + k] = lg[k];
        }
#pragma unroll 4
        for (int j = 0; j < kAH; ++j) {
            float sg = 0.f;
#pragma unroll
            for (int k = 0; k < NCH; ++k)
                if (k < L.nch) sg += w[L.a3 + k * kAH + j] * lg[k];
            s_g2[t * LD + j] = sg * (s_a2[t * LD + j] > 0.f ? 1.f : kSlope);
        }
#pragma unroll 4
        for (int i = 0; i < kAH; ++i) {
            float sg = 0.f;
#pragma unroll 8
            for (int j = 0; j < kAH; ++j) sg += w[L.a2 + j * kAH + i] * s_g2[t * LD + j];
            s_g1[t * LD + i] = sg * (s_a1[t * LD + i] > 0.f ? 1.f : kSlope);
        }
        __syncthreads();
        // thread t owns row t of dA2, column t of dA3, row t of dA1
        for (int r = 0; r < R; ++r) {
            const float gr2 = s_g2[r * LD + t], gr1 = s_g1[r * LD + t], ar2 = s_a2[r * LD + t];
#pragma unroll
            for (int i = 0; i < kAH; ++i) acc2[i] += gr2 * s_a1[r * LD + i];
#pragma unroll
            for (int k = 0; k < NCH; ++k) acc3[k] += s_gl[r * LC + k] * ar2;
#pragma unroll
            for (int f = 0; f < NF; ++f) acc1[f] += gr1 * s_f[r * LF + f];
            gc1 += gr1;
            gc2 += gr2;
            if (t < NCH) gc3 += s_gl[r * LC + t];
        }
        __syncthreads();
    }
    float *out = a.part + static_cast<long long>(blockIdx.x) * L.total;
#pragma unroll
    for (int i = 0; i < kAH; ++i) out[L.a2 + t * kAH + i] = acc2[i];
#pragma unroll
    for (int k = 0; k < NCH; ++k)
        if (k < L.nch) out[L.a3 + k * kAH + t] = acc3[k];
#pragma unroll
    for (int f = 0; f < NF; ++f)
        if (f < L.F) out[L.a1 + t * L.F + f] = acc1[f];
    out[L.c1 + t] = gc1;
    out[L.c2 + t] = gc2;
    if (t < L.nch) out[L.c3 + t] = gc3;
    // loss partial
    __shared__ double red[kAlphaBlock];
    red[t] = lsum;
    __syncthreads();
    if (t == 0) {
        double sl = 0;
        for (int i = 0; i < R; ++i) sl += red[i];
        a.loss_part[blockIdx.x] = sl;
    }
}

template <int NCH, int NF>
constexpr size_t alpha_train_smem(int total) {
    return sizeof(float) * (((total + 3) & ~3) + 4 * kAlphaBlock * (kAH + 1) + kAlphaBlock * (NCH + 1) +
                            kAlphaBlock * (NF + 1));
}

// Flow-path points, step 2, after the phased weight pass of a tile: every
// channel's density D_k = dens_k vw_k, w0 = 1 / sum_k beta_k / D_k, the
// integrand. Training: log F (F = f D_c / F_scale), features and log prior
// of the batch row. Sampling: the channel-weight network and
// v = alpha_c f D_c / (beta_c q_c) at the point's index (NaN when not finite).
// The channel-weight network as the sampling pass keeps it in shared memory:
// every block 16-byte aligned and W1's rows padded to NF columns, so that the
// products read four weights per shared load.
template <int NCH, int NF>
struct AlphaSmem {
    static constexpr int kC1 = 0, kA1 = kAH, kC2 = kA1 + kAH * NF, kA2 = kC2 + kAH, kC3 = kA2 + kAH * kAH,
                         kA3 = kC3 + NCH, kTotal = kA3 + NCH * kAH;
};

template <int NCH, int NF>
__device__ __forceinline__ void alpha_to_smem(const float *__restrict__ w, const AlphaLayout &L, float *s) {
    using S = AlphaSmem<NCH, NF>;
    for (int q = threadIdx.x; q < S::kTotal; q += blockDim.x) {
        float v = 0.f;
        if (q < S::kA1) v = w[L.c1 + q];
        else if (q < S::kC2) {
            const int i = (q - S::kA1) / NF, f = (q - S::kA1) % NF;
            v = f < L.F ? w[L.a1 + i * L.F + f] : 0.f;
        } else if (q < S::kA2) v = w[L.c2 + q - S::kC2];
        else if (q < S::kC3) v = w[L.a2 + q - S::kA2];
        else if (q < S::kA3) v = (q - S::kC3) < L.nch ? w[L.c3 + q - S::kC3] : 0.f;
        else {
            const int k = (q - S::kA3) / kAH, j = (q - S::kA3) % kAH;
            v = k < L.nch ? w[L.a3 + k * kAH + j] : 0.f;
        }
        s[q] = v;
    }
}

// alpha_forward on the shared-memory copy (float4 weight reads).
template <int NCH, int NF>
__device__ __forceinline__ void alpha_forward_smem(const float *__restrict__ s, int nch, const float (&feat)[NF],
                                                   const float *logprior, float (&lg)[NCH], float &lse) {
    using S = AlphaSmem<NCH, NF>;
    float a1[kAH];
#pragma unroll
    for (int i = 0; i < kAH; ++i) {
        float acc = s[S::kC1 + i];
        const float4 *wr = reinterpret_cast<const float4 *>(s + S::kA1 + i * NF);
#pragma unroll
        for (int q = 0; q < NF / 4; ++q) {
            const float4 w4 = wr[q];
            acc += w4.x * feat[4 * q] + w4.y * feat[4 * q + 1] + w4.z * feat[4 * q + 2] + w4.w * feat[4 * q + 3];
        }
        a1[i] = lrelu(acc);
    }
#pragma unroll
    for (int k = 0; k < NCH; ++k) lg[k] = k < nch ? s[S::kC3 + k] + logprior[k] : -INFINITY;
    // the second hidden layer four units at a time, each group added into
    // the logits at once (the same order of additions as a whole second
    // layer followed by the last one, without holding all of it; a rolled
    // loop, so that the registers hold the first layer and one group)
#pragma unroll 1
    for (int q = 0; q < kAH / 4; ++q) {
        float h[4];
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            const int j = 4 * q + jj;
            float acc = s[S::kC2 + j];
            const float4 *wr = reinterpret_cast<const float4 *>(s + S::kA2 + j * kAH);
#pragma unroll
            for (int r = 0; r < kAH / 4; ++r) {
                const float4 w4 = wr[r];
                acc += w4.x * a1[4 * r] + w4.y * a1[4 * r + 1] + w4.z * a1[4 * r + 2] + w4.w * a1[4 * r + 3];
            }
            h[jj] = lrelu(acc);
        }
#pragma unroll
        for (int k = 0; k < NCH; ++k) {
            if (k < nch) {
                const float4 w4 = reinterpret_cast<const float4 *>(s + S::kA3 + k * kAH)[q];
                lg[k] += w4.x * h[0] + w4.y * h[1] + w4.z * h[2] + w4.w * h[3];
            }
        }
    }
    float mx = -INFINITY;
#pragma unroll
    for (int k = 0; k < NCH; ++k) mx = fmaxf(mx, lg[k]);
    float se = 0.f;
#pragma unroll
    for (int k = 0; k < NCH; ++k)
        if (k < nch) se += expf(lg[k] - mx);
    lse = mx + logf(se);
}

// log(x) of a positive double to float precision: exponent exactly, the
// mantissa's log in f32 (the log priors are f32 values).
__device__ __forceinline__ float log_d2f(double x) {
    int e;
    const double mnt = frexp(x, &e);
    return __logf(static_cast<float>(mnt)) + static_cast<float>(e) * 0.69314718055994531f;
}

struct CombineArgs {
    const double *node_soa;  // tile nodes [node][4][T]
    const double *dcv, *vwv; // tile densities [channel][T]
    const int32_t *ich_tile;
    const int32_t *list;
    const long long *count;
    long long base, T, m;
    int nch, n_ext;
    double sqrts;
    const IntegrandDesc *f;
    const float *beta, *logbeta;
    // training
    double log_fscale;
    float *logf;       // [m]
    double *fval;      // [m] or null
    float *feat;       // [F][m]
    float *logprior;   // [nch][m]
    // sampling
    const float *logq; // [m]
    const float *w;    // network parameters
    AlphaLayout L;
    double *v;         // [m]
};

template <bool TRAIN, int NCH, int NF>
__global__ void __launch_bounds__(128, TRAIN ? 1 : 4) k_flow_combine(CombineArgs a) {
    extern __shared__ __align__(16) float cw[];  // the network (sampling), AlphaSmem layout
    if (!TRAIN) {
        alpha_to_smem<NCH, NF>(a.w, a.L, cw);
        __syncthreads();
    }
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    const long long r = a.base + i;
    if (i >= a.T || r >= *a.count) return;
    const long long k = a.list[r];
    const int c = a.ich_tile[i];
    V4 mom[CHILI_MAX_EXT];
    for (int s = 0; s < a.n_ext; ++s) mom[s] = soa_v4(a.node_soa, s, a.T, i);
    // g_j = 1 / D_j; a channel whose D_j is +inf contributes nothing to the
    // mixture (g_j = 0, its prior and weight 0), as its term alpha_j / D_j
    // does in the plain combined weight; the sampled channel's D_c must be
    // finite and positive
    double acc = 0.0, Dc = 0.0;
    bool ok = true;
    for (int j = 0; j < a.nch; ++j) {
        const double Dj = a.dcv[static_cast<long long>(j) * a.T + i] * a.vwv[static_cast<long long>(j) * a.T + i];
        ok = ok && (Dj > 0);  // NaN and non-positive densities: no value
        acc += static_cast<double>(a.beta[j]) / Dj;
        if (j == c) Dc = Dj;
    }
    const double w0 = 1.0 / acc;
    const double fv = eval_momenta(a.f, mom, a.n_ext);
    const double F = fv * Dc;
    ok = ok && isfinite(Dc) && (w0 > 0) && isfinite(w0) && (F > 0) && isfinite(F);
    float lp[NCH > 0 ? NCH : 1];
    if (ok) {
        const float lw0 = log_d2f(w0);
        for (int j = 0; j < a.nch; ++j) {
            const double Dj = a.dcv[static_cast<long long>(j) * a.T + i] * a.vwv[static_cast<long long>(j) * a.T + i];
            lp[j] = isinf(Dj) ? -INFINITY : a.logbeta[j] - log_d2f(Dj) + lw0;
        }
    }
    float featv[kMaxFeat];
    if (ok) point_features(mom, a.n_ext, a.sqrts, featv);
    if (TRAIN) {
        if (!ok) return;  // the row keeps logf = -inf
        if (a.fval) a.fval[k] = F;
        a.logf[k] = static_cast<float>(log(F) - a.log_fscale);
        const int nf = n_features(a.n_ext);
        for (int q = 0; q < nf; ++q) a.feat[q * a.m + k] = featv[q];
        for (int j = 0; j < a.nch; ++j) a.logprior[j * a.m + k] = lp[j];
    } else {
        double v = 0;
        if (ok) {
            // the network's padded input columns must read 0, not whatever
            // the local memory beyond this point's nf features holds (0 x
            // inf would be NaN)
            const int nf = n_features(a.n_ext);
            float feat[NF];
#pragma unroll
            for (int q = 0; q < NF; ++q) feat[q] = (q < nf && q < kMaxFeat) ? featv[q] : 0.f;
            float lg[NCH], lse;
            alpha_forward_smem<NCH, NF>(cw, a.L.nch, feat, lp, lg, lse);
            float lac = lg[0];
#pragma unroll
            for (int q = 1; q < NCH; ++q)
                if (q == c) lac = lg[q];
            lac -= lse;
            v = exp(static_cast<double>(lac - a.logbeta[c] - a.logq[k])) * F;
            if (!isfinite(v)) v = CUDART_NAN;
        }
        a.v[k] = v;
    }
}

#ifndef CHILI_FLOW_LAYERS_ONLY
// Flow-path points, step 1 (training: TRAIN = true, u uniform from the
// counter-based generator and c ~ beta; sampling: u from the inverse flow,
// c drawn before it): x = VEGAS_c(u), p = FSMapper_c(x), PreProcess; the
// accepted points are listed (any order: every point's result is written at
// its own index) and their external momenta stored [leg][component][m].
struct GenArgs {
    const ChannelProgram *progs;
    const double *grids;
    const double *cp;
    const IntegrandDesc *f;
    int nch, dims, bins, n_ext;
    uint64_t seed, ctr0;
    long long m;
    float *u;          // [D][m]: written (training) or read (sampling)
    int32_t *ch;       // [m]: written (training) or read (sampling)
    double *mom_soa;   // [n_ext][4][m]
    int32_t *list;     // [m]
    long long *count;  // listed points
};

template <bool TRAIN>
__global__ void __launch_bounds__(128) k_flow_gen(GenArgs a) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= a.m) return;
    const int D = a.dims;
    double r[CHILI_MAX_DIMS + 1];
    int c;
    if (TRAIN) {
        load_uniforms(a.seed, a.ctr0 + i, nullptr, D + 1, r);
        c = select_channel(a.cp, a.nch, r[D]);
        for (int d = 0; d < D; ++d) a.u[d * a.m + i] = static_cast<float>(r[d]);
        a.ch[i] = c;
    } else {
        c = a.ch[i];
        for (int d = 0; d < D; ++d) r[d] = fmin(static_cast<double>(a.u[d * a.m + i]), 0.99999999999999989);
    }
    double jac;
    V4 mom[CHILI_MAX_SLOTS];
    double m2[CHILI_MAX_SLOTS];
    if (!grid_map_checked(a.grids + static_cast<size_t>(c) * D * (a.bins + 1), D, a.bins, r, jac)) return;
    fs_generate(a.progs + c, r, mom, m2);
    if (!preprocess(a.f, mom)) return;
    const long long k = static_cast<long long>(atomicAdd(reinterpret_cast<unsigned long long *>(a.count), 1ull));
    a.list[k] = static_cast<int32_t>(i);
    for (int s = 0; s < a.n_ext; ++s) {
        a.mom_soa[(4 * s + 0) * a.m + i] = mom[s].e;
        a.mom_soa[(4 * s + 1) * a.m + i] = mom[s].x;
        a.mom_soa[(4 * s + 2) * a.m + i] = mom[s].y;
        a.mom_soa[(4 * s + 3) * a.m + i] = mom[s].z;
    }
}

// Training rows default to a rejected point: log F = -inf, log prior = log beta.
__global__ void k_flow_rows_init(long long m, int nch, int F, const float *__restrict__ logbeta, float *__restrict__ logf,
                                 float *__restrict__ feat, float *__restrict__ logprior, double *__restrict__ fval) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= m) return;
    logf[i] = -INFINITY;
    if (fval) fval[i] = 0;
    for (int q = 0; q < F; ++q) feat[q * m + i] = 0.f;
    for (int j = 0; j < nch; ++j) logprior[j * m + i] = logbeta[j];
}

// Flow-path sampling, step 1: channel c ~ beta, z uniform in [0,1)^D
// (the flow's base point), log q = 0, v = 0.
__global__ void k_flow_draw(const double *__restrict__ cp, int nch, int dims, uint64_t seed, uint64_t ctr0,
                            long long n, float *__restrict__ z, int32_t *__restrict__ ch, float *__restrict__ logq,
                            double *__restrict__ v) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    double r[CHILI_MAX_DIMS + 1];
    load_uniforms(seed, ctr0 + i, nullptr, dims + 1, r);
    ch[i] = select_channel(cp, nch, r[dims]);
    for (int d = 0; d < dims; ++d) z[d * n + i] = fminf(static_cast<float>(r[d]), 0.99999994f);
    logq[i] = 0.f;
    v[i] = 0.0;
}

// StatsData partial of a block of points: [n, sum, sum2, max, nonzero,
// nonfinite] + per channel [n_c, sum (beta_c v)^2]; NaN values count as 0.
constexpr int kPhysBlock = 128;
constexpr int kPhysFixed = 6;

__global__ void __launch_bounds__(kPhysBlock) k_flow_stats(const double *__restrict__ vals,
                                                           const int32_t *__restrict__ ch,
                                                           const float *__restrict__ beta, int nch, long long n,
                                                           double *__restrict__ part) {
    __shared__ double s_ch[2 * kMaxAlphaCh];
    const int t = threadIdx.x;
    for (int q = t; q < 2 * nch; q += blockDim.x) s_ch[q] = 0;
    __syncthreads();
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + t;
    double v = 0;
    bool bad = false;
    if (i < n) {
        v = vals[i];
        if (!isfinite(v)) {
            bad = true;
            v = 0;
        }
        const int c = ch[i];
        const double T = v * static_cast<double>(beta[c]);
        atomicAdd(s_ch + c, 1.0);
        atomicAdd(s_ch + nch + c, T * T);
    }
    const double cnt = i < n ? 1.0 : 0.0;
    double q0 = cnt, q1 = v, q2 = v * v, q3 = v, q4 = v != 0 ? 1.0 : 0.0, q5 = bad ? 1.0 : 0.0;
    q0 = warp_sum(q0); q1 = warp_sum(q1); q2 = warp_sum(q2); q3 = warp_max(q3); q4 = warp_sum(q4); q5 = warp_sum(q5);
    __shared__ double red[kPhysBlock / 32][kPhysFixed];
    if ((t & 31) == 0) {
        red[t >> 5][0] = q0; red[t >> 5][1] = q1; red[t >> 5][2] = q2;
        red[t >> 5][3] = q3; red[t >> 5][4] = q4; red[t >> 5][5] = q5;
    }
    __syncthreads();
    double *out = part + static_cast<long long>(blockIdx.x) * (kPhysFixed + 2 * nch);
    if (t < kPhysFixed) {
        double sr = 0.0;
        for (int wq = 0; wq < kPhysBlock / 32; ++wq) sr = t == 3 ? fmax(sr, red[wq][3]) : sr + red[wq][t];
        out[t] = sr;
    }
    for (int q = t; q < 2 * nch; q += blockDim.x) out[kPhysFixed + q] = s_ch[q];
}


// Ordered fold of the block partials: out[0..5] = n, sum, sum2, max,
// nonzero, nonfinite; out[6..] = per channel n_c, sum T_c^2.
__global__ void k_flow_fold(const double *__restrict__ part, int nblocks, int width, double *__restrict__ out) {
    const int q = threadIdx.x + blockIdx.x * blockDim.x;
    if (q >= width) return;
    double s = 0;
    for (int b = 0; b < nblocks; ++b) {
        const double v = part[static_cast<long long>(b) * width + q];
        s = q == 3 ? fmax(s, v) : s + v;
    }
    out[q] = s;
}

// Ordered sum of the loss partials.
__global__ void k_loss_fold(const double *__restrict__ part, int nblocks, double scale, double *__restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s = 0;
    for (int b = 0; b < nblocks; ++b) s += part[b];
    *out = s * scale;
}

// Sum and count of positive values of a double array (one block).
__global__ void k_sum_pos(const double *__restrict__ v, long long n, double *__restrict__ out) {
    __shared__ double red[256];
    double s = 0, c = 0;
    for (long long i = threadIdx.x; i < n; i += 256) {
        s += v[i];
        c += v[i] > 0 ? 1.0 : 0.0;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0;
        for (int k = 0; k < 256; ++k) tot += red[k];
        out[0] = tot;
    }
    __syncthreads();
    red[threadIdx.x] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0;
        for (int k = 0; k < 256; ++k) tot += red[k];
        out[1] = tot;
    }
}

// [n][D] row-major <-> [D][n]
__global__ void k_transpose_f(const float *__restrict__ in, float *__restrict__ out, long long n, int D, int to_soa) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= n * D) return;
    const long long r = i / D;
    const int d = static_cast<int>(i % D);
    if (to_soa) out[d * n + r] = in[i];
    else out[i] = in[d * n + r];
}

#endif  // CHILI_FLOW_LAYERS_ONLY

}  // namespace chili_flow
