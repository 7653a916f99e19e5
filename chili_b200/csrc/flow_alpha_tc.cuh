// flow_alpha_tc.cuh -- the channel-weight network of the learned proposal on
// the tensor cores: alpha(p) = softmax(MLP(phi(p)) + log prior(p)), an MLP of
// F features -> 64 -> 64 -> nch logits (leaky ReLU), bf16 operands and f32
// accumulation (tcgen05, accumulators in tensor memory), biases and the
// softmax in f32 (Heimel et al., "MadNIS", SciPost Phys. 15 (2023) 141, for
// the multi-channel weights with an analytic prior).
//
// One CTA of 128 threads works on tiles of 128 points (thread t = point row t
// = tensor-memory lane t). Per tile:
//   z1 = a0 A1^T (+ c1), h1 = lrelu(z1)       a0 = [features | 1 | 0], K = 32
//   z2 = h1 A2^T (+ c2), h2 = lrelu(z2)       K = 64
//   logits = h2 A3^T + c3 + log prior         N = 16 or 64 channel columns
// Training (k_alpha_train_tc) adds the variance loss, the backward products
//   g_h2 = g_l A3,  g_p2 = g_h2 * lrelu'(z2),  g_h1 = g_p2 A2,  g_p1 = g_h1 * lrelu'(z1)
// and the weight gradients with K = the points, accumulated in tensor memory
// over the CTA's tiles:
//   dA3^T = h2^T g_l,  dA2^T = h1^T g_p2,  dA1 = g_p1^T a0.
// The bias gradients come out of the same products: column 64 of the h1 and
// h2 tiles and column F of a0 hold the constant 1, so row 64 of dA3^T and
// dA2^T and column F of dA1 are the column sums of g_l, g_p2 and g_p1. (The
// constant columns take no part in the forward products: those read columns
// 0..63 of h1 and h2, and the A1 tile is zero from column F on.)
// Sampling (k_alpha_eval_tc) keeps one activation tile (a0, then h1, then
// h2) and 128 tensor-memory columns, so that four CTAs share an SM.
// Operand tiles use the SW128 layout of tc.cuh; the weight tiles serve as
// K-major operands forward and as MN-major operands (their transposes)
// backward, without copies. A tile's row inputs are loaded at its start, all
// loads in flight together.
#pragma once

#include "flow_phys.cuh"

namespace chili_flow {

constexpr int kAThreads = 128;
// training shared memory: weights, a0 [128 x 64], h1 and h2 [128 x 128],
// g_l [128 x 64], g_p2 [128 x 64], g_p1 [128 x 128], f32 biases
constexpr int kASmemTrain = kAWBytes + 128 * 64 * 2 + 2 * kHTile + 128 * 64 * 2 * 2 + kHTile + 3 * 64 * 4 + 64 + 1024;
// sampling: weights, one [128 x 64] tile, biases (42.8 KB), requested as
// 48 KB so that at most four CTAs (4 x 128 tensor-memory columns) share an SM
constexpr int kASmemEvalUsed = kAWBytes + 128 * 64 * 2 + 3 * 64 * 4 + 64 + 1024;
constexpr int kASmemEval = 48 * 1024;
static_assert(kASmemEvalUsed <= kASmemEval, "sampling shared memory");
// training tensor-memory columns: z1 / g_h2, z2 / g_h1, logits, and the
// three weight-gradient accumulators
constexpr uint32_t kTZ1 = 0, kTZ2 = 64, kTLg = 128, kTdA3 = 192, kTdA2 = 256, kTdA1 = 320;

// f32 parameters (AlphaLayout) -> the three bf16 weight tiles, zero padded.
__global__ void k_alpha_pack(const float *__restrict__ w, AlphaLayout L, uint8_t *__restrict__ tiles) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * 64 * 64) return;
    const int m = i / 4096, r = (i % 4096) / 64, c = i % 64;
    float v = 0.f;
    if (m == 0) v = c < L.F ? w[L.a1 + r * L.F + c] : 0.f;
    else if (m == 1) v = w[L.a2 + r * kAH + c];
    else v = r < L.nch ? w[L.a3 + r * kAH + c] : 0.f;
    *reinterpret_cast<uint16_t *>(tiles + m * kATile + sw128_off(r, c, 64)) =
        static_cast<uint16_t>(pack_bf16x2(v, 0.f) & 0xFFFFu);
}


// lrelu of 32 accumulator columns plus a bias, with the sign mask
__device__ __forceinline__ uint32_t bias_lrelu32(float (&v)[32], const float *bias) {
    uint32_t mk = 0;
#pragma unroll
    for (int j = 0; j < 32; ++j) {
        const float z = v[j] + bias[j];
        mk |= (z > 0.f ? 1u : 0u) << j;
        v[j] = z > 0.f ? z : kSlope * z;
    }
    return mk;
}

// The inputs of one row: the a0 row (features, 1 at column F, zero beyond;
// all zero for rows past n), the log prior (-inf beyond nch), channel, log F
// and log q. Every load is issued before the first is used.
template <int NCHP>
struct AlphaRow {
    float a0[32];
    float lp[NCHP];
    float lf, lq;
    int c;
};

template <int NCHP>
__device__ __forceinline__ void load_alpha_row(const AlphaTcArgs &a, long long row, bool valid, AlphaRow<NCHP> &R) {
    const long long n = a.n;
    const long long rr = valid ? row : 0;
    const int F = a.L.F, nch = a.L.nch;
#pragma unroll
    for (int f = 0; f < 32; ++f) R.a0[f] = f < F ? __ldg(a.feat + static_cast<long long>(f) * n + rr) : 0.f;
#pragma unroll
    for (int k = 0; k < NCHP; ++k) R.lp[k] = k < nch ? __ldg(a.logprior + static_cast<long long>(k) * n + rr) : 0.f;
    R.lf = __ldg(a.logf + rr);
    R.lq = __ldg(a.logq + rr);
    const int c = __ldg(a.ch + rr);
    R.c = (c >= 0 && c < nch) ? c : 0;
#pragma unroll
    for (int f = 0; f < 32; ++f) R.a0[f] = valid ? (f == F ? 1.f : R.a0[f]) : 0.f;
    if (!valid) R.lf = -INFINITY;
}

// logits (accumulators + c3 + log prior) -> log alpha of every channel's
// logit in lg (lg[k] - lse), lse; returns log alpha_c.
template <int NCHP>
__device__ __forceinline__ float alpha_softmax(float (&lg)[NCHP], const float *c3, const float (&lp)[NCHP], int nch,
                                               int c, float &lse) {
    float mx = -INFINITY;
#pragma unroll
    for (int k = 0; k < NCHP; ++k) {
        const float s = k < nch ? lg[k] + c3[k] + lp[k] : -INFINITY;
        lg[k] = s;
        mx = fmaxf(mx, s);
    }
    float se = 0.f;
#pragma unroll
    for (int k = 0; k < NCHP; ++k)
        if (k < nch) se += expf(lg[k] - mx);
    lse = mx + logf(se);
    float lac = lg[0];
#pragma unroll
    for (int k = 1; k < NCHP; ++k)
        if (k == c) lac = lg[k];
    return lac - lse;
}

// NCHP logits columns of this thread's lane
template <int NCHP>
__device__ __forceinline__ void load_logits(uint32_t taddr, float (&lg)[NCHP]) {
    if constexpr (NCHP == 16) {
        tmem_ld16(taddr, lg);
    } else {
#pragma unroll
        for (int h = 0; h < NCHP / 32; ++h) {
            float v[32];
            tmem_ld32(taddr + 32 * h, v);
#pragma unroll
            for (int k = 0; k < 32; ++k) lg[32 * h + k] = v[k];
        }
    }
}

// Weight tiles and biases into shared memory (all threads).
__device__ __forceinline__ void alpha_stage(const AlphaTcArgs &a, uint8_t *sm, float *sB) {
    copy_block(sm, a.tiles, kAWBytes);
    for (int i = threadIdx.x; i < 192; i += blockDim.x) {
        const int q = i / 64, j = i % 64;
        float b = 0.f;
        if (q == 0) b = a.w[a.L.c1 + j];
        else if (q == 1) b = a.w[a.L.c2 + j];
        else b = j < a.L.nch ? a.w[a.L.c3 + j] : 0.f;
        sB[i] = b;
    }
}

// --------------------------------------------------------------- training
// Forward, variance loss (l = alpha_c^2 F^2 / (beta_c^2 q), mean over the
// batch; d loss / d log q into glogq), backward and this CTA's partial of
// every parameter's gradient (in the AlphaLayout order) and of the loss.
template <int NCHP>
__global__ void __launch_bounds__(kAThreads, 1) k_alpha_train_tc(AlphaTcArgs a) {
    static_assert(NCHP == 16 || NCHP == 64, "channel columns");
    extern __shared__ uint8_t smem_raw[];
    uint8_t *sm = align1024(smem_raw);
    uint8_t *sW1 = sm, *sW2 = sm + kATile, *sW3 = sm + 2 * kATile;
    uint8_t *sA0 = sm + kAWBytes;            // [128 x 64]
    uint8_t *sH1 = sA0 + 128 * 64 * 2;        // [128 x 128]
    uint8_t *sH2 = sH1 + kHTile;              // [128 x 128]
    uint8_t *sGL = sH2 + kHTile;              // [128 x 64]
    uint8_t *sGP2 = sGL + 128 * 64 * 2;       // [128 x 64]
    uint8_t *sGP1 = sGP2 + 128 * 64 * 2;      // [128 x 128]
    float *sB = reinterpret_cast<float *>(sGP1 + kHTile);  // c1 [64], c2 [64], c3 [64]
    uint64_t *bar = reinterpret_cast<uint64_t *>(sB + 192);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);
    constexpr uint32_t kCols = 512;
    const int t = threadIdx.x, wp = t >> 5;
    const AlphaLayout L = a.L;
    const long long n = a.n;
    const long long ntiles = (n + 127) / 128;

    if (t == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    if (wp == 0) tmem_alloc(tslot, kCols);
    alpha_stage(a, sm, sB);
    {
        // constant columns: a0 [32, 64) zero; h1, h2: column 64 = 1, 65..127
        // zero; g_p1: 64..127 zero
        float z[32], one[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            z[j] = 0.f;
            one[j] = j == 0 ? 1.f : 0.f;
        }
        store_row32(sA0, 128, t, 32, z);
        store_row32(sH1, 128, t, 64, one);
        store_row32(sH1, 128, t, 96, z);
        store_row32(sH2, 128, t, 64, one);
        store_row32(sH2, 128, t, 96, z);
        store_row32(sGP1, 128, t, 64, z);
        store_row32(sGP1, 128, t, 96, z);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = *tslot;
    const uint32_t lane = tbase + (static_cast<uint32_t>(wp * 32) << 16);
    const uint32_t aW1 = smem_u32(sW1), aW2 = smem_u32(sW2), aW3 = smem_u32(sW3), aA0 = smem_u32(sA0),
                   aH1 = smem_u32(sH1), aH2 = smem_u32(sH2), aGL = smem_u32(sGL), aGP2 = smem_u32(sGP2),
                   aGP1 = smem_u32(sGP1);
    constexpr uint32_t id_h = idesc_bf16(128, 64, false, false);      // z1, z2
    constexpr uint32_t id_l = idesc_bf16(128, NCHP, false, false);    // logits
    constexpr uint32_t id_gh = idesc_bf16(128, 64, false, true);      // g_h2, g_h1 (weights MN-major)
    constexpr uint32_t id_w3 = idesc_bf16(128, NCHP, true, true);     // dA3^T
    constexpr uint32_t id_w2 = idesc_bf16(128, 64, true, true);       // dA2^T
    constexpr uint32_t id_w1 = idesc_bf16(128, 32, true, true);       // dA1
    bool ok = true;
    uint32_t phase = 0;
    bool first = true;
    double lsum = 0.0;
    const float invn = 1.f / static_cast<float>(n);
    auto wait_mma = [&]() {
        ok = mbar_wait(bar, phase, kWaitLimit) && ok;
        phase ^= 1;
        tc_fence_after();
    };
    auto sync_issue = [&]() -> bool {
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (t != 0) return false;
        tc_fence_after();
        return true;
    };

    for (long long tile = blockIdx.x; __syncthreads_and(ok) && tile < ntiles; tile += gridDim.x) {
        const long long row = tile * 128 + t;
        const bool valid = row < n;
        AlphaRow<NCHP> R;
        load_alpha_row<NCHP>(a, row, valid, R);
        const int c = R.c;
        store_row32(sA0, 128, t, 0, R.a0);
        if (sync_issue()) {
            mma_bf16(tbase + kTZ1, desc_k(aA0, 128, 0), desc_k(aW1, 64, 0), id_h, 0);
            mma_bf16(tbase + kTZ1, desc_k(aA0, 128, 16), desc_k(aW1, 64, 16), id_h, 1);
            mma_commit(bar);
        }
        wait_mma();
        uint32_t m1[2], m2[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            float v[32];
            tmem_ld32(lane + kTZ1 + 32 * h, v);
            m1[h] = bias_lrelu32(v, sB + 32 * h);
            store_row32(sH1, 128, t, 32 * h, v);
        }
        if (sync_issue()) {
#pragma unroll
            for (int k = 0; k < 4; ++k) mma_bf16(tbase + kTZ2, desc_k(aH1, 128, 16 * k), desc_k(aW2, 64, 16 * k), id_h, k > 0);
            mma_commit(bar);
        }
        wait_mma();
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            float v[32];
            tmem_ld32(lane + kTZ2 + 32 * h, v);
            m2[h] = bias_lrelu32(v, sB + 64 + 32 * h);
            store_row32(sH2, 128, t, 32 * h, v);
        }
        if (sync_issue()) {
#pragma unroll
            for (int k = 0; k < 4; ++k) mma_bf16(tbase + kTLg, desc_k(aH2, 128, 16 * k), desc_k(aW3, 64, 16 * k), id_l, k > 0);
            mma_commit(bar);
        }
        wait_mma();
        float lg[NCHP], lse;
        load_logits<NCHP>(lane + kTLg, lg);
        const float lac = alpha_softmax<NCHP>(lg, sB + 128, R.lp, L.nch, c, lse);
        // variance-loss term and d loss / d logits = gsel (delta_kc - alpha_k)
        float ell = 0.f;
        if (valid) {
            const float e = 2.f * lac + 2.f * R.lf - 2.f * a.logbeta[c] - R.lq;
            ell = isfinite(e) ? expf(e) : 0.f;
            if (!isfinite(ell)) ell = 0.f;
            a.glogq[row] = -ell * invn;
        }
        lsum += ell;
        const float gsel = 2.f * ell * invn;
        {
            float gl[32];
#pragma unroll
            for (int h = 0; h < (NCHP + 31) / 32; ++h) {
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int k = 32 * h + j;
                    float g = 0.f;
                    if (k < NCHP && k < L.nch) g = gsel * ((k == c ? 1.f : 0.f) - expf(lg[k] - lse));
                    gl[j] = g;
                }
                store_row32(sGL, 128, t, 32 * h, gl);
            }
        }
        // g_h2 = g_l A3 (A3 as an MN-major operand: K = channels)
        if (sync_issue()) {
#pragma unroll
            for (int k = 0; k < NCHP / 16; ++k)
                mma_bf16(tbase + kTZ1, desc_k(aGL, 128, 16 * k), desc_mn(aW3, 64, 16 * k), id_gh, k > 0);
            mma_commit(bar);
        }
        wait_mma();
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            float v[32];
            tmem_ld32(lane + kTZ1 + 32 * h, v);
#pragma unroll
            for (int j = 0; j < 32; ++j) v[j] *= ((m2[h] >> j) & 1u) ? 1.f : kSlope;
            store_row32(sGP2, 128, t, 32 * h, v);
        }
        // g_h1 = g_p2 A2
        if (sync_issue()) {
#pragma unroll
            for (int k = 0; k < 4; ++k)
                mma_bf16(tbase + kTZ2, desc_k(aGP2, 128, 16 * k), desc_mn(aW2, 64, 16 * k), id_gh, k > 0);
            mma_commit(bar);
        }
        wait_mma();
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            float v[32];
            tmem_ld32(lane + kTZ2 + 32 * h, v);
#pragma unroll
            for (int j = 0; j < 32; ++j) v[j] *= ((m1[h] >> j) & 1u) ? 1.f : kSlope;
            store_row32(sGP1, 128, t, 32 * h, v);
        }
        // weight gradients, K = the 128 points of the tile
        if (sync_issue()) {
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const uint32_t acc = (!first || k > 0) ? 1u : 0u;
                mma_bf16(tbase + kTdA3, desc_mn(aH2, 128, 16 * k), desc_mn(aGL, 128, 16 * k), id_w3, acc);
                mma_bf16(tbase + kTdA2, desc_mn(aH1, 128, 16 * k), desc_mn(aGP2, 128, 16 * k), id_w2, acc);
                mma_bf16(tbase + kTdA1, desc_mn(aGP1, 128, 16 * k), desc_mn(aA0, 128, 16 * k), id_w1, acc);
            }
            mma_commit(bar);
        }
        first = false;
        wait_mma();  // the tiles are rewritten by the next tile
    }
    // this CTA's partial: thread t holds row t of every accumulator
    float *out = a.part + static_cast<long long>(blockIdx.x) * L.total;
    for (int h = 0; h < NCHP / 16; ++h) {
        float v[16];
        if (first) {
#pragma unroll
            for (int j = 0; j < 16; ++j) v[j] = 0.f;
        } else {
            tmem_ld16(lane + kTdA3 + 16 * h, v);
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int k = 16 * h + j;
            if (k < L.nch) {
                if (t < kAH) out[L.a3 + k * kAH + t] = v[j];
                else if (t == kAH) out[L.c3 + k] = v[j];
            }
        }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        float v[32];
        if (first) {
#pragma unroll
            for (int j = 0; j < 32; ++j) v[j] = 0.f;
        } else {
            tmem_ld32(lane + kTdA2 + 32 * h, v);
        }
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            const int o = 32 * h + j;
            if (t < kAH) out[L.a2 + o * kAH + t] = v[j];
            else if (t == kAH) out[L.c2 + o] = v[j];
        }
    }
    {
        float v[32];
        if (first) {
#pragma unroll
            for (int j = 0; j < 32; ++j) v[j] = 0.f;
        } else {
            tmem_ld32(lane + kTdA1, v);
        }
        if (t < kAH) {
#pragma unroll
            for (int f = 0; f < 32; ++f) {
                if (f < L.F) out[L.a1 + t * L.F + f] = v[f];
                else if (f == L.F) out[L.c1 + t] = v[f];
            }
        }
    }
    __shared__ double red[kAThreads];
    red[t] = lsum;
    __syncthreads();
    if (t == 0) {
        double sl = 0;
        for (int i = 0; i < kAThreads; ++i) sl += red[i];
        a.loss_part[blockIdx.x] = sl;
    }
    if (!ok && t == 0) atomicExch(a.err, 4);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (wp == 0) tmem_dealloc(tbase, kCols);
}

// --------------------------------------------------------------- sampling
// The value of every row: v = alpha_c F / (beta_c q) (F = a.fval, q from
// log q), 0 for rows without a value (log F = -inf), NaN when not finite.
// One [128 x 64] activation tile: a0, then h1 (after z1's product has read
// a0), then h2; tensor memory: z1 and then the logits in columns 0..63, z2
// in 64..127.
template <int NCHP>
__global__ void __launch_bounds__(kAThreads, 4) k_alpha_eval_tc(AlphaTcArgs a) {
    static_assert(NCHP == 16 || NCHP == 64, "channel columns");
    extern __shared__ uint8_t smem_raw[];
    uint8_t *sm = align1024(smem_raw);
    uint8_t *sW1 = sm, *sW2 = sm + kATile, *sW3 = sm + 2 * kATile;
    uint8_t *sX = sm + kAWBytes;                              // [128 x 64]
    float *sB = reinterpret_cast<float *>(sX + 128 * 64 * 2);  // c1 [64], c2 [64], c3 [64]
    uint64_t *bar = reinterpret_cast<uint64_t *>(sB + 192);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);
    constexpr uint32_t kCols = 128;
    const int t = threadIdx.x, wp = t >> 5;
    const long long n = a.n;
    const long long ntiles = (n + 127) / 128;
    if (t == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    if (wp == 0) tmem_alloc(tslot, kCols);
    alpha_stage(a, sm, sB);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = *tslot;
    const uint32_t lane = tbase + (static_cast<uint32_t>(wp * 32) << 16);
    const uint32_t aW1 = smem_u32(sW1), aW2 = smem_u32(sW2), aW3 = smem_u32(sW3), aX = smem_u32(sX);
    constexpr uint32_t id_h = idesc_bf16(128, 64, false, false);
    constexpr uint32_t id_l = idesc_bf16(128, NCHP, false, false);
    bool ok = true;
    uint32_t phase = 0;
    auto wait_mma = [&]() {
        ok = mbar_wait(bar, phase, kWaitLimit) && ok;
        phase ^= 1;
        tc_fence_after();
    };
    auto sync_issue = [&]() -> bool {
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (t != 0) return false;
        tc_fence_after();
        return true;
    };
    for (long long tile = blockIdx.x; __syncthreads_and(ok) && tile < ntiles; tile += gridDim.x) {
        const long long row = tile * 128 + t;
        const bool valid = row < n;
        AlphaRow<NCHP> R;
        load_alpha_row<NCHP>(a, row, valid, R);
        const double fv = __ldg(a.fval + (valid ? row : 0));
        store_row32(sX, 128, t, 0, R.a0);
        if (sync_issue()) {
            mma_bf16(tbase, desc_k(aX, 128, 0), desc_k(aW1, 64, 0), id_h, 0);
            mma_bf16(tbase, desc_k(aX, 128, 16), desc_k(aW1, 64, 16), id_h, 1);
            mma_commit(bar);
        }
        wait_mma();
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            float v[32];
            tmem_ld32(lane + 32 * h, v);
            bias_lrelu32(v, sB + 32 * h);
            store_row32(sX, 128, t, 32 * h, v);
        }
        if (sync_issue()) {
#pragma unroll
            for (int k = 0; k < 4; ++k) mma_bf16(tbase + 64, desc_k(aX, 128, 16 * k), desc_k(aW2, 64, 16 * k), id_h, k > 0);
            mma_commit(bar);
        }
        wait_mma();
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            float v[32];
            tmem_ld32(lane + 64 + 32 * h, v);
            bias_lrelu32(v, sB + 64 + 32 * h);
            store_row32(sX, 128, t, 32 * h, v);
        }
        if (sync_issue()) {
#pragma unroll
            for (int k = 0; k < 4; ++k) mma_bf16(tbase, desc_k(aX, 128, 16 * k), desc_k(aW3, 64, 16 * k), id_l, k > 0);
            mma_commit(bar);
        }
        wait_mma();
        float lg[NCHP], lse;
        load_logits<NCHP>(lane, lg);
        const float lac = alpha_softmax<NCHP>(lg, sB + 128, R.lp, a.L.nch, R.c, lse);
        if (valid) {
            double v = 0.0;
            if (R.lf != -INFINITY) {
                v = exp(static_cast<double>(lac - a.logbeta[R.c] - R.lq)) * fv;
                if (!isfinite(v)) v = CUDART_NAN;
            }
            a.v[row] = v;
        }
    }
    if (!ok && t == 0) atomicExch(a.err, 5);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (wp == 0) tmem_dealloc(tbase, kCols);
}

}  // namespace chili_flow
