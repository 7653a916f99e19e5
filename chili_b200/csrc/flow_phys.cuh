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

// The channel-weight network's bf16 weight tiles (flow_alpha_tc.cuh): A1
// (hidden x feature), A2 (out x in), A3 (channel x hidden), 64 x 64 each.
constexpr int kATile = 64 * 64 * 2;
constexpr int kAWBytes = 3 * kATile;

// Arguments of the channel-weight network's tensor-core kernel (one row per
// point: features, log prior, channel, log F, log q).
struct AlphaTcArgs {
    long long n;          // rows
    AlphaLayout L;
    const uint8_t *tiles; // kAWBytes (k_alpha_pack)
    const float *w;       // f32 parameters (the biases are read from here)
    const float *feat;    // [F][n]
    const float *logprior;// [nch][n]
    const int32_t *ch;    // [n]
    const float *logf;    // [n]: training log F (-inf: no value); sampling: -inf marks a row without value
    const float *logbeta; // [nch]
    const float *logq;    // [n]
    // training
    float *glogq;         // [n]
    float *part;          // [gridDim.x][L.total]
    double *loss_part;    // [gridDim.x]
    // sampling
    const double *fval;   // [n] F of the row
    double *v;            // [n] the value alpha_c F / (beta_c q)
    int *err;
};

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

// Flow-path points, step 2, after the phased weight pass of a tile: every
// channel's density D_k = dens_k vw_k, w0 = 1 / sum_k beta_k / D_k, the
// integrand; the point's row for the channel-weight network (flow_alpha_tc.cuh):
// log F (F = f D_c / F_scale, and F itself when fval is given), features and
// log prior. Rows of points without a value keep log F = -inf.
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
    double log_fscale;
    float *logf;       // [m]
    double *fval;      // [m] or null
    float *feat;       // [F][m]
    float *logprior;   // [nch][m]
};

template <int NCH>
__global__ void __launch_bounds__(128) k_flow_combine(CombineArgs a) {
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
    if (!ok) return;  // the row keeps logf = -inf
    float lp[NCH > 0 ? NCH : 1];
    const float lw0 = log_d2f(w0);
    for (int j = 0; j < a.nch; ++j) {
        const double Dj = a.dcv[static_cast<long long>(j) * a.T + i] * a.vwv[static_cast<long long>(j) * a.T + i];
        lp[j] = isinf(Dj) ? -INFINITY : a.logbeta[j] - log_d2f(Dj) + lw0;
    }
    float featv[kMaxFeat];
    point_features(mom, a.n_ext, a.sqrts, featv);
    if (a.fval) a.fval[k] = F;
    a.logf[k] = static_cast<float>(log(F) - a.log_fscale);
    const int nf = n_features(a.n_ext);
    for (int q = 0; q < nf; ++q) a.feat[q * a.m + k] = featv[q];
    for (int j = 0; j < a.nch; ++j) a.logprior[j * a.m + k] = lp[j];
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
// nonzero, nonfinite; out[6..] = per channel n_c, sum T_c^2. One CTA per
// field (gridDim.x = width): thread t folds partials t, t + 256, ... in
// order, then a fixed tree over the threads (deterministic).
__global__ void __launch_bounds__(256) k_flow_fold(const double *__restrict__ part, int nblocks, int width,
                                                   double *__restrict__ out) {
    const int q = blockIdx.x;
    const bool mx = q == 3;
    double s = 0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        const double v = part[static_cast<long long>(b) * width + q];
        s = mx ? fmax(s, v) : s + v;
    }
    __shared__ double red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] = mx ? fmax(red[threadIdx.x], red[threadIdx.x + h])
                                                   : red[threadIdx.x] + red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[q] = red[0];
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
