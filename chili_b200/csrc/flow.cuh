// flow.cuh -- device side of the learned proposal: a channel-conditioned
// rational-quadratic spline coupling flow on the VEGAS uniforms (Durkan et
// al., "Neural Spline Flows", 2019). Chili has no learned proposal; this is
// new capability on top of its VEGAS + multichannel path.
//
// Coupling layer l: the conditioning coordinates a = x[cond] (da <= 16) and
// the point's channel c give the spline parameters of the transformed
// coordinates x[trans] (db <= 5):
//   h1 = lrelu(W1 (2a - 1) + E[c]),  h1[127] = 1   (E[c] through a one-hot
//                                    column c of the same product, K = 64)
//   h2 = lrelu(W2 h1),               h2[127] = 1      (unit 127 carries the bias)
//   theta = W3 h2                    (db x 49: 16 widths, 16 heights, 17 slopes)
// The three products run on the tensor cores (tcgen05, bf16 operands in
// shared memory, f32 accumulators in tensor memory), 128 points per tile, one
// point per thread in the epilogues; the spline is evaluated in f32.
//
// Training: per layer one forward kernel that also saves the bf16 activation
// tiles and theta, one backward kernel for the data gradients (spline
// backward, then two more tensor-core products), one weight-gradient kernel
// (three products summed over the points, K = points), and an Adam kernel.
#pragma once

#include <cstdint>

#include "tc.cuh"

namespace chili_flow {

using namespace chili_tc;

constexpr int kH = 128;           // hidden units of a conditioner layer (unit 127 is the constant 1)
constexpr int kBins = 16;          // spline bins
constexpr int kPerDim = 3 * kBins + 1;
constexpr int kMaxDB = 5;          // transformed dimensions per layer
constexpr int kMaxDA = 16;         // conditioning dimensions per layer
constexpr int kMaxFlowCh = 48;     // channels (one-hot columns 16..63 of the first product)
constexpr int kP = 256;            // padded spline-parameter columns (>= 5 * 49)
constexpr float kMinW = 1e-3f, kMinH = 1e-3f, kMinD = 1e-3f, kSlope = 0.01f;
constexpr uint32_t kWaitLimit = 1u << 22;

// bf16 weight tiles of one layer, contiguous: W1 [128][64] (columns 0..da-1:
// W1, columns 16..16+nch-1: the channel embedding E^T, so nch <= 48),
// W2 [128][128], W3 [256][128] (db*49 rows used), each an SW128 tile.
constexpr int kW1Bytes = 128 * 64 * 2, kW2Bytes = 128 * 128 * 2, kW3Bytes = kP * 128 * 2;
constexpr int kWBytes = kW1Bytes + kW2Bytes + kW3Bytes;
// The forward kernel's copy of W3 with every dimension's 49 rows at a
// 64-row boundary (rows 64 j .. 64 j + 48 for dimension j; the rest zero), so
// that each dimension's spline parameters land at an aligned block of 64
// accumulator columns. Stored per layer after the kWBytes of tiles.
constexpr int kPF = 64 * kMaxDB;
constexpr int kW3FBytes = kPF * 128 * 2;
constexpr int kWLayerBytes = kWBytes + kW3FBytes;
constexpr int kHTile = 128 * 128 * 2;   // one activation tile (128 points x 128 units)
constexpr int kGTile = 128 * kP * 2;    // one spline-gradient tile (128 points x 256)

struct FlowLayer {
    const uint8_t *wt;   // kWBytes of tiles (W1, W2, W3)
    const uint8_t *wtf;  // kW3FBytes: W3 in the forward kernel's padded row order
    const float *E;     // [nch][128] channel embedding (first-layer bias per channel)
    int da, db, nch;
    int8_t cond[kMaxDA];
    int8_t trans[8];
};

// ------------------------------------------------------------------ spline
__device__ __forceinline__ float softplus_f(float t) { return t > 20.f ? t : log1pf(__expf(t)); }
__device__ __forceinline__ float sigmoid_f(float t) { return 1.f / (1.f + __expf(-t)); }

// softmax of 16 logits (sm) and the bin sizes min + (1 - 16 min) sm
__device__ __forceinline__ void bin_sizes(const float *th, float minv, float (&sm)[kBins], float (&sz)[kBins]) {
    float m = th[0];
#pragma unroll
    for (int k = 1; k < kBins; ++k) m = fmaxf(m, th[k]);
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < kBins; ++k) {
        sm[k] = __expf(th[k] - m);
        s += sm[k];
    }
    const float inv = __frcp_rn(s), sc = 1.f - kBins * minv;
#pragma unroll
    for (int k = 0; k < kBins; ++k) {
        sm[k] *= inv;
        sz[k] = minv + sc * sm[k];
    }
}

struct SplineBin {
    int k;
    float x0, y0, wk, hk, d0, d1, t0, t1;  // t0, t1: raw slope logits of knots k, k+1
};

// The bin of v: the number of interior knots (cumulative sizes, in bin
// order) not above v, on the x knots (forward) or the y knots (inverse).
__device__ __forceinline__ SplineBin locate(const float *th, const float (&w)[kBins], const float (&h)[kBins],
                                            float v, bool inverse) {
    SplineBin b;
    b.k = 0;
    b.x0 = 0.f;
    b.y0 = 0.f;
    b.wk = w[0];
    b.hk = h[0];
    float cx = 0.f, cy = 0.f;
#pragma unroll
    for (int m = 0; m < kBins; ++m) {
        const bool in = (m == 0) || ((inverse ? cy : cx) <= v);
        if (in) {
            b.k = m;
            b.x0 = cx;
            b.y0 = cy;
            b.wk = w[m];
            b.hk = h[m];
        }
        cx += w[m];
        cy += h[m];
    }
    b.t0 = th[2 * kBins];
    b.t1 = th[2 * kBins + 1];
#pragma unroll
    for (int m = 1; m < kBins; ++m)
        if (m == b.k) {
            b.t0 = th[2 * kBins + m];
            b.t1 = th[2 * kBins + m + 1];
        }
    b.d0 = kMinD + softplus_f(b.t0);
    b.d1 = kMinD + softplus_f(b.t1);
    return b;
}

// y = RQS(x) and log dy/dx (forward, density direction)
__device__ __forceinline__ float rqs_forward(const float *th, float x, float &logj) {
    float smw[kBins], w[kBins], smh[kBins], h[kBins];
    bin_sizes(th, kMinW, smw, w);
    bin_sizes(th + kBins, kMinH, smh, h);
    const SplineBin b = locate(th, w, h, x, false);
    const float xi = (x - b.x0) / b.wk;
    const float s = b.hk / b.wk;
    const float om = xi * (1.f - xi);
    const float A = s * xi * xi + b.d0 * om;
    const float B = s + (b.d0 + b.d1 - 2.f * s) * om;
    const float C = b.d1 * xi * xi + 2.f * s * om + b.d0 * (1.f - xi) * (1.f - xi);
    logj = 2.f * __logf(s) + __logf(C) - 2.f * __logf(B);
    return b.y0 + b.hk * A / B;
}

// x = RQS^-1(y) and log dy/dx at x (sampling direction)
__device__ __forceinline__ float rqs_inverse(const float *th, float y, float &logj) {
    float smw[kBins], w[kBins], smh[kBins], h[kBins];
    bin_sizes(th, kMinW, smw, w);
    bin_sizes(th + kBins, kMinH, smh, h);
    const SplineBin b = locate(th, w, h, y, true);
    const float s = b.hk / b.wk;
    const float dl = b.d0 + b.d1 - 2.f * s;
    const float dy = y - b.y0;
    const float qa = b.hk * (s - b.d0) + dy * dl;
    const float qb = b.hk * b.d0 - dy * dl;
    const float qc = -s * dy;
    const float disc = fmaxf(qb * qb - 4.f * qa * qc, 0.f);
    const float xi = 2.f * qc / (-qb - sqrtf(disc));
    const float om = xi * (1.f - xi);
    const float B = s + dl * om;
    const float C = b.d1 * xi * xi + 2.f * s * om + b.d0 * (1.f - xi) * (1.f - xi);
    logj = 2.f * __logf(s) + __logf(C) - 2.f * __logf(B);
    return b.x0 + xi * b.wk;
}

// Gradients of gy*y + gj*log(dy/dx) with respect to the 49 parameters and x.
__device__ __forceinline__ float rqs_backward(const float *th, float x, float gy, float gj, float (&g)[kPerDim]) {
    float smw[kBins], w[kBins], smh[kBins], h[kBins];
    bin_sizes(th, kMinW, smw, w);
    bin_sizes(th + kBins, kMinH, smh, h);
    const SplineBin b = locate(th, w, h, x, false);
    const float xi = (x - b.x0) / b.wk;
    const float s = b.hk / b.wk;
    const float om = xi * (1.f - xi);
    const float dl = b.d0 + b.d1 - 2.f * s;
    const float A = s * xi * xi + b.d0 * om;
    const float B = s + dl * om;
    const float C = b.d1 * xi * xi + 2.f * s * om + b.d0 * (1.f - xi) * (1.f - xi);
    const float A_xi = 2.f * s * xi + b.d0 * (1.f - 2.f * xi), A_s = xi * xi, A_d0 = om;
    const float B_xi = dl * (1.f - 2.f * xi), B_s = 1.f - 2.f * om, B_d = om;
    const float C_xi = 2.f * b.d1 * xi + 2.f * s * (1.f - 2.f * xi) - 2.f * b.d0 * (1.f - xi);
    const float C_s = 2.f * om, C_d0 = (1.f - xi) * (1.f - xi), C_d1 = xi * xi;
    const float hB2 = b.hk / (B * B);
    const float iB = 1.f / B, iC = 1.f / C;
    const float g_xi = gy * hB2 * (A_xi * B - A * B_xi) + gj * (C_xi * iC - 2.f * B_xi * iB);
    const float g_s = gy * hB2 * (A_s * B - A * B_s) + gj * (2.f / s + C_s * iC - 2.f * B_s * iB);
    const float g_d0 = gy * hB2 * (A_d0 * B - A * B_d) + gj * (C_d0 * iC - 2.f * B_d * iB);
    const float g_d1 = gy * hB2 * (-A * B_d) + gj * (C_d1 * iC - 2.f * B_d * iB);
    const float g_hk = gy * A * iB + g_s / b.wk;
    const float g_x0 = -g_xi / b.wk;
    const float g_wk = -(g_xi * xi + g_s * s) / b.wk;
    const float g_y0 = gy;
    const float scw = 1.f - kBins * kMinW, sch = 1.f - kBins * kMinH;
    float dotw = 0.f, doth = 0.f;
#pragma unroll
    for (int m = 0; m < kBins; ++m) {
        const float gw = (m < b.k ? g_x0 : 0.f) + (m == b.k ? g_wk : 0.f);
        const float gh = (m < b.k ? g_y0 : 0.f) + (m == b.k ? g_hk : 0.f);
        g[m] = scw * gw;
        g[kBins + m] = sch * gh;
        dotw += g[m] * smw[m];
        doth += g[kBins + m] * smh[m];
    }
#pragma unroll
    for (int m = 0; m < kBins; ++m) {
        g[m] = smw[m] * (g[m] - dotw);
        g[kBins + m] = smh[m] * (g[kBins + m] - doth);
    }
    const float s0 = sigmoid_f(b.t0), s1 = sigmoid_f(b.t1);
#pragma unroll
    for (int m = 0; m <= kBins; ++m)
        g[2 * kBins + m] = (m == b.k ? g_d0 * s0 : 0.f) + (m == b.k + 1 ? g_d1 * s1 : 0.f);
    return g_xi / b.wk;
}

// rqs_backward with the 49 parameter gradients written straight into row r
// of a bf16 SW128 tile (columns c0 .. c0 + 48) instead of an array: the same
// value for every gradient, fewer live registers. Returns d/dx.
__device__ __forceinline__ float rqs_backward_st(const float *th, float x, float gy, float gj, uint8_t *tile, int r,
                                                 int c0) {
    float smw[kBins], w[kBins], smh[kBins], h[kBins];
    bin_sizes(th, kMinW, smw, w);
    bin_sizes(th + kBins, kMinH, smh, h);
    const SplineBin b = locate(th, w, h, x, false);
    const float xi = (x - b.x0) / b.wk;
    const float s = b.hk / b.wk;
    const float om = xi * (1.f - xi);
    const float dl = b.d0 + b.d1 - 2.f * s;
    const float A = s * xi * xi + b.d0 * om;
    const float B = s + dl * om;
    const float C = b.d1 * xi * xi + 2.f * s * om + b.d0 * (1.f - xi) * (1.f - xi);
    const float A_xi = 2.f * s * xi + b.d0 * (1.f - 2.f * xi), A_s = xi * xi, A_d0 = om;
    const float B_xi = dl * (1.f - 2.f * xi), B_s = 1.f - 2.f * om, B_d = om;
    const float C_xi = 2.f * b.d1 * xi + 2.f * s * (1.f - 2.f * xi) - 2.f * b.d0 * (1.f - xi);
    const float C_s = 2.f * om, C_d0 = (1.f - xi) * (1.f - xi), C_d1 = xi * xi;
    const float hB2 = b.hk / (B * B);
    const float iB = 1.f / B, iC = 1.f / C;
    const float g_xi = gy * hB2 * (A_xi * B - A * B_xi) + gj * (C_xi * iC - 2.f * B_xi * iB);
    const float g_s = gy * hB2 * (A_s * B - A * B_s) + gj * (2.f / s + C_s * iC - 2.f * B_s * iB);
    const float g_d0 = gy * hB2 * (A_d0 * B - A * B_d) + gj * (C_d0 * iC - 2.f * B_d * iB);
    const float g_d1 = gy * hB2 * (-A * B_d) + gj * (C_d1 * iC - 2.f * B_d * iB);
    const float g_hk = gy * A * iB + g_s / b.wk;
    const float g_x0 = -g_xi / b.wk;
    const float g_wk = -(g_xi * xi + g_s * s) / b.wk;
    const float g_y0 = gy;
    const float scw = 1.f - kBins * kMinW, sch = 1.f - kBins * kMinH;
    float dotw = 0.f, doth = 0.f;
#pragma unroll
    for (int m = 0; m < kBins; ++m) {
        const float gw = (m < b.k ? g_x0 : 0.f) + (m == b.k ? g_wk : 0.f);
        const float gh = (m < b.k ? g_y0 : 0.f) + (m == b.k ? g_hk : 0.f);
        dotw += (scw * gw) * smw[m];
        doth += (sch * gh) * smh[m];
    }
    auto put = [&](int col, float v) {
        *reinterpret_cast<uint16_t *>(tile + sw128_off(r, c0 + col, 128)) =
            static_cast<uint16_t>(pack_bf16x2(v, 0.f) & 0xFFFFu);
    };
#pragma unroll
    for (int m = 0; m < kBins; ++m) {
        const float gw = (m < b.k ? g_x0 : 0.f) + (m == b.k ? g_wk : 0.f);
        const float gh = (m < b.k ? g_y0 : 0.f) + (m == b.k ? g_hk : 0.f);
        put(m, smw[m] * (scw * gw - dotw));
        put(kBins + m, smh[m] * (sch * gh - doth));
    }
    const float s0 = sigmoid_f(b.t0), s1 = sigmoid_f(b.t1);
#pragma unroll
    for (int m = 0; m <= kBins; ++m)
        put(2 * kBins + m, (m == b.k ? g_d0 * s0 : 0.f) + (m == b.k + 1 ? g_d1 * s1 : 0.f));
    return g_xi / b.wk;
}

// ------------------------------------------------------------- helpers
__device__ __forceinline__ uint8_t *align1024(uint8_t *p) {
    const uint32_t a = smem_u32(p);
    return p + (((a + 1023u) & ~1023u) - a);
}

__device__ __forceinline__ float lrelu(float v) { return v > 0.f ? v : kSlope * v; }

// Writes 32 consecutive values of row r (columns c0..c0+31) of an SW128 tile
// with R rows as bf16.
__device__ __forceinline__ void store_row32(uint8_t *tile, int R, int r, int c0, const float (&v)[32]) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        uint4 pk;
        pk.x = pack_bf16x2(v[8 * q + 0], v[8 * q + 1]);
        pk.y = pack_bf16x2(v[8 * q + 2], v[8 * q + 3]);
        pk.z = pack_bf16x2(v[8 * q + 4], v[8 * q + 5]);
        pk.w = pack_bf16x2(v[8 * q + 6], v[8 * q + 7]);
        *reinterpret_cast<uint4 *>(tile + sw128_off(r, c0 + 8 * q, R)) = pk;
    }
}

// Reads 32 consecutive bf16 values (columns c0..c0+31) of row r of a tile.
__device__ __forceinline__ void load_row32(const uint8_t *tile, int R, int r, int c0, float (&v)[32]) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const uint4 pk = *reinterpret_cast<const uint4 *>(tile + sw128_off(r, c0 + 8 * q, R));
        v[8 * q + 0] = bf16_lo(pk.x);
        v[8 * q + 1] = bf16_hi(pk.x);
        v[8 * q + 2] = bf16_lo(pk.y);
        v[8 * q + 3] = bf16_hi(pk.y);
        v[8 * q + 4] = bf16_lo(pk.z);
        v[8 * q + 5] = bf16_hi(pk.z);
        v[8 * q + 6] = bf16_lo(pk.w);
        v[8 * q + 7] = bf16_hi(pk.w);
    }
}

// Cooperative copy of `bytes` (a multiple of 16 * blockDim.x) between
// 16-byte aligned buffers.
__device__ __forceinline__ void copy_block(void *dst, const void *src, int bytes) {
    const uint4 *s = static_cast<const uint4 *>(src);
    uint4 *d = static_cast<uint4 *>(dst);
    for (int i = threadIdx.x; i < bytes / 16; i += blockDim.x) d[i] = s[i];
}

// ------------------------------------------------- coupling layer, forward
// MODE 0: density direction x -> y = RQS(x) (training and log q of given
// points); MODE 1: sampling direction y -> x = RQS^-1(y). SAVE keeps the
// activation tiles and theta for the backward pass. logq[i] += sum log dy/dx.
struct LayerArgs {
    FlowLayer L;
    long long n;
    const float *xin;  // [D][n]
    float *xout;       // [D][n]
    const int32_t *ch;
    float *logq;
    uint8_t *h1s, *h2s;  // [tiles][kHTile] (SAVE)
    float *theta;        // [db*49][n] (SAVE)
    int *err;
};

// Shared memory of the forward kernel: W1, W2, the padded W3, A tile, H tile,
// the log-det partials of the four other thread groups of a point, and the
// next tile's conditioning coordinates [16][128] and channels [128], copied
// asynchronously while the current tile's splines run.
// Five thread groups of 128 (one thread per point each; TMEM lanes are shared
// by warps w, w+4, ..., w+16): groups 0-3 split the 128 hidden columns of the
// epilogues, group j evaluates the spline of dimension j.
constexpr int kFwdGroups = 5;
constexpr int kFwdThreads = 128 * kFwdGroups;
constexpr int kFwdSmem = kW1Bytes + kW2Bytes + kW3FBytes + 128 * 64 * 2 + kHTile + (kFwdGroups - 1) * 128 * 4 +
                         kMaxDA * 128 * 4 + 128 * 4 + 64 + 1024;

// theta of dimension j: the 64 accumulator columns 128 + 64 j .. (the first
// 49 used), two loads in flight.
__device__ __forceinline__ void theta_window(uint32_t lane_addr, int j, float (&v)[64]) {
    uint32_t r0[32], r1[32];
    tmem_ld32_async(lane_addr + static_cast<uint32_t>(128 + 64 * j), r0);
    tmem_ld32_async(lane_addr + static_cast<uint32_t>(128 + 64 * j + 32), r1);
    tmem_wait_ld();
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        v[i] = __uint_as_float(r0[i]);
        v[32 + i] = __uint_as_float(r1[i]);
    }
}

template <int DB, int MODE, bool SAVE>
__global__ void __launch_bounds__(kFwdThreads, 1) k_flow_layer(LayerArgs a) {
    static_assert(DB >= 1 && DB <= kFwdGroups, "one spline dimension per thread group");
    extern __shared__ uint8_t smem_raw[];
    uint8_t *sm = align1024(smem_raw);
    uint8_t *sW1 = sm, *sW2 = sm + kW1Bytes, *sW3 = sm + kW1Bytes + kW2Bytes;  // sW3: kPF padded rows
    uint8_t *sA = sW3 + kW3FBytes;
    uint8_t *sH = sA + 128 * 64 * 2;
    float *sL = reinterpret_cast<float *>(sH + kHTile);  // [4][128] log-det partials of groups 1..4
    float *sX = sL + (kFwdGroups - 1) * 128;                // [kMaxDA][128] conditioning coordinates
    int *sCh = reinterpret_cast<int *>(sX + kMaxDA * 128);  // [128] channels
    uint64_t *bar = reinterpret_cast<uint64_t *>(sCh + 128);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 2);
    const int t = threadIdx.x, wp = t >> 5;
    const int grp = wp >> 2;                 // 0..4: the thread group of this warp
    const int r = (wp & 3) * 32 + (t & 31);  // the point (TMEM lane) of this thread
    const long long n = a.n;
    const long long ntiles = (n + 127) / 128;

    if (t == 0) {
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
        fence_mbar_init();
    }
    if (wp == 0) tmem_alloc(tslot, 512);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = *tslot;
    const uint32_t lane_addr = tbase + (static_cast<uint32_t>((wp & 3) * 32) << 16);
    if (t == 0) {
        mbar_expect_tx(bar, kW1Bytes + kW2Bytes + kW3FBytes);
        bulk_g2s(sm, a.L.wt, kW1Bytes + kW2Bytes, bar);
        bulk_g2s(sW3, a.L.wtf, kW3FBytes, bar);
    }
    bool ok = mbar_wait(bar, 0, kWaitLimit);
    const uint32_t aW1 = smem_u32(sW1), aW2 = smem_u32(sW2), aW3 = smem_u32(sW3);
    const uint32_t aA = smem_u32(sA), aH = smem_u32(sH);
    constexpr uint32_t id_h = idesc_bf16(128, 128, false, false);
    // theta: dimensions 0 .. min(DB, 4) - 1 in one product (columns 128 ..),
    // dimension 4 in a second one (columns 384 .. 447)
    constexpr int kN1 = 64 * (DB < 4 ? DB : 4);
    constexpr uint32_t id_p1 = idesc_bf16(128, kN1, false, false);
    constexpr uint32_t id_p2 = idesc_bf16(128, 64, false, false);
    uint32_t phase = 0;
    const int da = a.L.da;
    // a tile's conditioning coordinates and channels into sX / sCh (rows past
    // n are not copied: the tile's users read them as invalid rows)
    auto prefetch = [&](long long tl) {
        const long long base = tl * 128;
        for (int e = t; e < (da + 1) * 128; e += kFwdThreads) {
            const int i = e >> 7, p = e & 127;
            const long long rw = base + p;
            if (rw >= n) continue;
            if (i < da) cp_async4(sX + e, a.xin + static_cast<long long>(a.L.cond[i]) * n + rw);
            else cp_async4(sCh + p, a.ch + rw);
        }
        cp_async_commit();
    };
    if (blockIdx.x < ntiles) prefetch(blockIdx.x);
    cp_async_wait_all();

    for (long long tile = blockIdx.x; __syncthreads_and(ok) && tile < ntiles; tile += gridDim.x) {
        const long long row = tile * 128 + r;
        const bool valid = row < n;
        // this thread's spline input and (group 0) the point's log q, loaded
        // now so that their latency hides behind the three products
        const int dsp = grp < DB ? a.L.trans[grp] : 0;
        const float xsp = (valid && grp < DB) ? a.xin[dsp * n + row] : 0.5f;
        const float lq0 = (valid && grp == 0) ? a.logq[row] : 0.f;
        if (grp < 2) {
            // A tile row, bf16: group 0 the conditioning coordinates (columns
            // 0..15) and one-hot columns 16..31, group 1 one-hot columns 32..63
            int c = valid ? sCh[r] : 0;
            c = (c >= 0 && c < a.L.nch) ? c : 0;  // channel indices come from callers: keep E reads in bounds
            float av[32];
            if (grp == 0) {
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    float v = 0.f;
                    if (i < da && valid) v = 2.f * fminf(fmaxf(sX[i * 128 + r], 0.f), 1.f) - 1.f;
                    av[i] = v;
                }
#pragma unroll
                for (int i = 16; i < 32; ++i) av[i] = (valid && i == 16 + c) ? 1.f : 0.f;
            } else {
#pragma unroll
                for (int i = 0; i < 32; ++i) av[i] = (valid && 32 + i == 16 + c) ? 1.f : 0.f;
            }
            store_row32(sA, 128, r, 32 * grp, av);
        } else if (grp == 2 && valid) {
            // identity coordinates pass through
            for (int i = 0; i < da; ++i) a.xout[a.L.cond[i] * n + row] = sX[i * 128 + r];
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (t == 0) {
            tc_fence_after();
#pragma unroll
            for (int k = 0; k < 4; ++k) mma_bf16(tbase, desc_k(aA, 128, 16 * k), desc_k(aW1, 128, 16 * k), id_h, k > 0);
            mma_commit(bar + 1);
        }
        ok = mbar_wait(bar + 1, phase, kWaitLimit) && ok;
        phase ^= 1;
        tc_fence_after();
        // h1 = lrelu(acc) (the product already holds E[c]); unit 127 = 1;
        // this group's 32 columns (groups 0-3)
        if (grp < 4) {
            const int c0 = 32 * grp;
            float v[32];
            tmem_ld32(lane_addr + c0, v);
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                v[j] = lrelu(v[j]);
                if (c0 + j == kH - 1) v[j] = 1.f;
            }
            store_row32(sH, 128, r, c0, v);
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (t == 0) {
            tc_fence_after();
#pragma unroll
            for (int k = 0; k < 8; ++k) mma_bf16(tbase, desc_k(aH, 128, 16 * k), desc_k(aW2, 128, 16 * k), id_h, k > 0);
            mma_commit(bar + 1);
        }
        if (SAVE) copy_block(a.h1s + tile * kHTile, sH, kHTile);
        ok = mbar_wait(bar + 1, phase, kWaitLimit) && ok;
        phase ^= 1;
        tc_fence_after();
        __syncthreads();  // the copy of h1 is complete before h2 overwrites it
        if (grp < 4) {
            const int c0 = 32 * grp;
            float v[32];
            tmem_ld32(lane_addr + c0, v);  // h2's accumulator reuses h1's columns
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                v[j] = lrelu(v[j]);
                if (c0 + j == kH - 1) v[j] = 1.f;
            }
            store_row32(sH, 128, r, c0, v);
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (t == 0) {
            tc_fence_after();
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                mma_bf16(tbase + 128, desc_k(aH, 128, 16 * k), desc_k(aW3, kPF, 16 * k), id_p1, k > 0);
                if (DB == 5)  // rows 256 .. 319 of the padded tile: 32 KB into each 64-column chunk
                    mma_bf16(tbase + 384, desc_k(aH, 128, 16 * k), desc_k(aW3 + 256 / 8 * 1024, kPF, 16 * k), id_p2,
                             k > 0);
            }
            mma_commit(bar + 1);
        }
        if (SAVE) copy_block(a.h2s + tile * kHTile, sH, kHTile);
        ok = mbar_wait(bar + 1, phase, kWaitLimit) && ok;
        phase ^= 1;
        tc_fence_after();
        // splines: dimension j = grp on group grp (DB <= kFwdGroups); one
        // copy of the spline code, the dimension a runtime value
        // sX / sCh were read before the first product of this tile: the next
        // tile's copies run beside the splines
        if (tile + gridDim.x < ntiles) prefetch(tile + gridDim.x);
        float lsum = 0.f;
        if (grp < DB) {
            const int j = grp;
            float th[64];
            theta_window(lane_addr, j, th);  // th[0 .. 48]: this dimension's parameters
            const int b0 = j * kPerDim;
            if (SAVE && valid) {
#pragma unroll
                for (int i = 0; i < kPerDim; ++i) a.theta[(b0 + i) * n + row] = th[i];
            }
            const float x = fminf(fmaxf(xsp, 0.f), 1.f);
            float lj;
            const float y = MODE == 0 ? rqs_forward(th, x, lj) : rqs_inverse(th, x, lj);
            if (valid) a.xout[dsp * n + row] = y;
            lsum += lj;
        }
        if (grp > 0) sL[(grp - 1) * 128 + r] = lsum;
        cp_async_wait_all();  // the next tile's copies of this thread, before the barrier publishes them
        tc_fence_before();
        __syncthreads();
        if (grp == 0 && valid) a.logq[row] = lq0 + (lsum + sL[r] + sL[128 + r] + sL[256 + r] + sL[384 + r]);
    }
    if (!ok && t == 0) atomicExch(a.err, 1);
    // every issued MMA has been waited for (or the wait gave up): release TMEM
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (wp == 0) tmem_dealloc(tbase, 512);
}

// ------------------------------------------------ coupling layer, backward
// Data gradients of one layer: spline backward (theta and x saved by the
// forward pass), then g_h2 = g_theta W3, g_p2 = g_h2 * lrelu'(h2),
// g_h1 = g_p2 W2, g_p1 = g_h1 * lrelu'(h1), g_a = g_p1 W1; writes the
// gradient of the layer input and the bf16 tiles of g_theta, g_p2 and g_p1
// for the weight-gradient kernel.
struct BwdArgs {
    FlowLayer L;
    long long n;
    const float *xin;    // layer input [D][n]
    const float *theta;  // [db*49][n]
    const uint8_t *h1s, *h2s;
    const float *gout;   // gradient of the layer output [D][n], or null (last layer)
    const float *glogq;  // d loss / d log q [n]
    float *gin;          // gradient of the layer input [D][n]
    uint8_t *gths, *gp2s, *gp1s;  // [tiles][kGTile], [tiles][kHTile], [tiles][kHTile]
    int *err;
};

// Five thread groups of 128 (one thread per point each, as in the forward
// kernel): group j runs the spline backward of dimension j; groups 0-3 split
// the epilogues' 128 hidden columns. The g_a partials of groups 1-3 reuse the
// g_theta tile's memory once its product and copy are done.
constexpr int kBwdGroups = 5;
constexpr int kBwdThreads = 128 * kBwdGroups;
constexpr int kBwdSmem = kWBytes + kGTile + kHTile + 64 + 1024;

template <int DB>
__global__ void __launch_bounds__(kBwdThreads, 1) k_flow_layer_bwd(BwdArgs a) {
    static_assert(DB >= 1 && DB <= kBwdGroups, "one spline dimension per thread group");
    extern __shared__ uint8_t smem_raw[];
    uint8_t *sm = align1024(smem_raw);
    uint8_t *sW1 = sm, *sW2 = sm + kW1Bytes, *sW3 = sm + kW1Bytes + kW2Bytes;
    uint8_t *sG = sm + kWBytes;
    uint8_t *sP = sG + kGTile;
    float *sGA = reinterpret_cast<float *>(sG);  // [3][16][128] g_a partials of groups 1-3 (after g_theta's use)
    uint64_t *bar = reinterpret_cast<uint64_t *>(sP + kHTile);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 2);
    const int t = threadIdx.x, wp = t >> 5;
    const int grp = wp >> 2;
    const int r = (wp & 3) * 32 + (t & 31);
    const long long n = a.n;
    const long long ntiles = (n + 127) / 128;
    if (t == 0) {
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
        fence_mbar_init();
    }
    if (wp == 0) tmem_alloc(tslot, 128);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = *tslot;
    const uint32_t lane_addr = tbase + (static_cast<uint32_t>((wp & 3) * 32) << 16);
    if (t == 0) {
        mbar_expect_tx(bar, kWBytes);
        bulk_g2s(sm, a.L.wt, kWBytes, bar);
    }
    bool ok = mbar_wait(bar, 0, kWaitLimit);
    const uint32_t aW2 = smem_u32(sW2), aW3 = smem_u32(sW3), aG = smem_u32(sG), aP = smem_u32(sP);
    constexpr uint32_t id_mn = idesc_bf16(128, 128, false, true);
    uint32_t phase = 0;
    const int da = a.L.da;
    // the group that zeroes g_theta's padding columns DB*49 .. 255
    constexpr int kPadGroup = DB < kBwdGroups ? DB : kBwdGroups - 1;
    for (long long tile = blockIdx.x; __syncthreads_and(ok) && tile < ntiles; tile += gridDim.x) {
        const long long row = tile * 128 + r;
        const bool valid = row < n;
        // spline backward of dimension grp -> g_theta (bf16 tile, row r)
        if (grp < DB) {
            const int b0 = grp * kPerDim;
            const int d = a.L.trans[grp];
            const long long rr = valid ? row : 0;
            float th[kPerDim];
#pragma unroll
            for (int i = 0; i < kPerDim; ++i) th[i] = a.theta[(b0 + i) * n + rr];
            const float x = fminf(fmaxf(a.xin[d * n + rr], 0.f), 1.f);
            const float gy = (valid && a.gout) ? a.gout[d * n + row] : 0.f;
            const float gl = valid ? a.glogq[row] : 0.f;
            const float gx = rqs_backward_st(th, x, gy, gl, sG, r, b0);
            if (valid) a.gin[d * n + row] = gx;
        }
        if (grp == kPadGroup)
            for (int col = DB * kPerDim; col < kP; ++col)
                *reinterpret_cast<uint16_t *>(sG + sw128_off(r, col, 128)) = 0;
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (t == 0) {
            tc_fence_after();
#pragma unroll
            for (int k = 0; k < kP / 16; ++k)
                mma_bf16(tbase, desc_k(aG, 128, 16 * k), desc_mn(aW3, kP, 16 * k), id_mn, k > 0);
            mma_commit(bar + 1);
        }
        copy_block(a.gths + tile * kGTile, sG, kGTile);
        ok = mbar_wait(bar + 1, phase, kWaitLimit) && ok;
        phase ^= 1;
        tc_fence_after();
        // g_p2 = g_h2 * lrelu'(h2), unit 127 -> 0; groups 0-3, 32 columns each
        if (grp < 4) {
            const uint8_t *h2t = a.h2s + tile * kHTile;
            const int c0 = 32 * grp;
            float v[32], hv[32];
            tmem_ld32(lane_addr + c0, v);
            load_row32(h2t, 128, r, c0, hv);
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                v[j] *= hv[j] > 0.f ? 1.f : kSlope;
                if (c0 + j == kH - 1 || !valid) v[j] = 0.f;
            }
            store_row32(sP, 128, r, c0, v);
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (t == 0) {
            tc_fence_after();
#pragma unroll
            for (int k = 0; k < 8; ++k) mma_bf16(tbase, desc_k(aP, 128, 16 * k), desc_mn(aW2, 128, 16 * k), id_mn, k > 0);
            mma_commit(bar + 1);
        }
        copy_block(a.gp2s + tile * kHTile, sP, kHTile);
        ok = mbar_wait(bar + 1, phase, kWaitLimit) && ok;
        phase ^= 1;
        tc_fence_after();
        __syncthreads();  // the copies of g_theta and g_p2 are complete before their tiles are reused
        // g_p1 = g_h1 * lrelu'(h1); g_a = bf16(g_p1) W1 on the CUDA cores,
        // this group's 32 units
        float ga[kMaxDA];
#pragma unroll
        for (int i = 0; i < kMaxDA; ++i) ga[i] = 0.f;
        if (grp < 4) {
            const uint8_t *h1t = a.h1s + tile * kHTile;
            const int c0 = 32 * grp;
            float v[32], hv[32];
            tmem_ld32(lane_addr + c0, v);
            load_row32(h1t, 128, r, c0, hv);
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                v[j] *= hv[j] > 0.f ? 1.f : kSlope;
                if (c0 + j == kH - 1 || !valid) v[j] = 0.f;
            }
            store_row32(sP, 128, r, c0, v);
#pragma unroll 4
            for (int j = 0; j < 32; ++j) {
                const int hcol = c0 + j;
                const float gq = bf16_hi(pack_bf16x2(0.f, v[j]));
                // W1[hcol][0..15]: two 16-byte chunks of row hcol of the W1 tile
                const uint4 w0 = *reinterpret_cast<const uint4 *>(sW1 + sw128_off(hcol, 0, 128));
                const uint4 w1 = *reinterpret_cast<const uint4 *>(sW1 + sw128_off(hcol, 8, 128));
                ga[0] += gq * bf16_lo(w0.x); ga[1] += gq * bf16_hi(w0.x);
                ga[2] += gq * bf16_lo(w0.y); ga[3] += gq * bf16_hi(w0.y);
                ga[4] += gq * bf16_lo(w0.z); ga[5] += gq * bf16_hi(w0.z);
                ga[6] += gq * bf16_lo(w0.w); ga[7] += gq * bf16_hi(w0.w);
                ga[8] += gq * bf16_lo(w1.x); ga[9] += gq * bf16_hi(w1.x);
                ga[10] += gq * bf16_lo(w1.y); ga[11] += gq * bf16_hi(w1.y);
                ga[12] += gq * bf16_lo(w1.z); ga[13] += gq * bf16_hi(w1.z);
                ga[14] += gq * bf16_lo(w1.w); ga[15] += gq * bf16_hi(w1.w);
            }
            if (grp > 0) {
#pragma unroll
                for (int i = 0; i < kMaxDA; ++i) sGA[((grp - 1) * kMaxDA + i) * 128 + r] = ga[i];
            }
        }
        __syncthreads();
        copy_block(a.gp1s + tile * kHTile, sP, kHTile);
        if (grp == 0 && valid) {
#pragma unroll
            for (int i = 0; i < kMaxDA; ++i)
                if (i < da) {
                    const int d = a.L.cond[i];
                    const float s3 = sGA[i * 128 + r] + sGA[(kMaxDA + i) * 128 + r] + sGA[(2 * kMaxDA + i) * 128 + r];
                    a.gin[d * n + row] = (a.gout ? a.gout[d * n + row] : 0.f) + 2.f * (ga[i] + s3);
                }
        }
        tc_fence_before();
    }
    if (!ok && t == 0) atomicExch(a.err, 2);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (wp == 0) tmem_dealloc(tbase, 128);
}

// Kernels launched only from flow.cu (the other translation units that
// include this header define CHILI_FLOW_LAYERS_ONLY).
#ifndef CHILI_FLOW_LAYERS_ONLY
// ------------------------------------------------------- weight gradients
// Product p (blockIdx.y) summed over this block's share of the point tiles
// (K = points), accumulated in tensor memory, then written as this block's
// partial (blockIdx.x) in the flat gradient layout:
//   p = 0: dW3[n][h]   = sum_r g_theta[r][n] h2[r][h]     (A = h2,   B = g_theta)
//   p = 1: dW2[o][i]   = sum_r g_p2[r][o]    h1[r][i]     (A = h1,   B = g_p2)
//   p = 2: dW1[h][i]   = sum_r g_p1[r][h]    a[r][i]      (A = g_p1, B = [a | 0 | onehot(c)])
//          dE[c][h]    = sum_{r: c_r = c} g_p1[r][h]
// Both operands are MN-major views of the saved row-major tiles.
struct WgradArgs {
    long long n;
    int da, nch, ncol2;  // ncol2: columns of the product-2 B tile (16 + nch, rounded up to 64)
    int8_t cond[kMaxDA];
    const float *xin;
    const int32_t *ch;
    const uint8_t *h1s, *h2s, *gths, *gp2s, *gp1s;
    float *part;          // [nsplit][nparam]
    long long nparam;     // stride between partials
    long long off_w1, off_e, off_w2, off_w3;
    int P;                // db*49
    int *err;
};

constexpr int kWgSmem = 2 * (kHTile + kGTile) + 64 + 1024;

__global__ void __launch_bounds__(128, 1) k_flow_wgrad(WgradArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *sm = align1024(smem_raw);
    uint8_t *sA[2] = {sm, sm + kHTile};
    uint8_t *sB[2] = {sm + 2 * kHTile, sm + 2 * kHTile + kGTile};
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + 2 * (kHTile + kGTile));
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 4);
    const int t = threadIdx.x, wp = t >> 5;
    const int p = blockIdx.y;
    const long long n = a.n;
    const long long ntiles = (n + 127) / 128;
    const int ncols = p == 0 ? kP : (p == 1 ? 128 : a.ncol2);
    const int bbytes = 128 * ncols * 2;
    const uint8_t *srcA = p == 0 ? a.h2s : (p == 1 ? a.h1s : a.gp1s);
    const uint8_t *srcB = p == 0 ? a.gths : (p == 1 ? a.gp2s : nullptr);
    const long long strideB = p == 0 ? kGTile : kHTile;
    if (t == 0) {
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
        mbar_init(bar + 2, 1);
        fence_mbar_init();
    }
    if (wp == 0) tmem_alloc(tslot, 256);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = *tslot;
    const uint32_t lane_addr = tbase + (static_cast<uint32_t>(wp * 32) << 16);
    const uint32_t idesc = idesc_bf16(128, ncols, true, true);
    bool ok = true;
    uint32_t ph_load[2] = {0, 0}, ph_mma = 0;
    bool first = true;
    auto issue_load = [&](long long tile, int s) {
        if (t == 0) {
            const uint32_t bytes = kHTile + (srcB ? bbytes : 0);
            mbar_expect_tx(bar + s, bytes);
            bulk_g2s(sA[s], srcA + tile * kHTile, kHTile, bar + s);
            if (srcB) bulk_g2s(sB[s], srcB + tile * strideB, bbytes, bar + s);
        }
    };
    long long tile = blockIdx.x;
    if (tile < ntiles) issue_load(tile, 0);
    int s = 0;
    for (; __syncthreads_and(ok) && tile < ntiles; tile += gridDim.x, s ^= 1) {
        if (p == 2) {
            // B tile: [a (da columns) | 0 | onehot(c) at column 16 + c], bf16
            const long long row = tile * 128 + t;
            const bool valid = row < n;
            const int c = valid ? a.ch[row] : -1;
            for (int c0 = 0; c0 < ncols; c0 += 32) {
                float v[32];
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int col = c0 + j;
                    float x = 0.f;
                    if (valid) {
                        if (col < a.da)
                            x = 2.f * fminf(fmaxf(a.xin[a.cond[col] * n + row], 0.f), 1.f) - 1.f;
                        else if (col == 16 + c)
                            x = 1.f;
                    }
                    v[j] = x;
                }
                store_row32(sB[s], 128, t, c0, v);
            }
            fence_async_smem();
        }
        ok = mbar_wait(bar + s, ph_load[s], kWaitLimit) && ok;
        ph_load[s] ^= 1;
        tc_fence_before();
        __syncthreads();
        if (t == 0) {
            tc_fence_after();
            const uint32_t aa = smem_u32(sA[s]), ab = smem_u32(sB[s]);
#pragma unroll
            for (int k = 0; k < 8; ++k)
                mma_bf16(tbase, desc_mn(aa, 128, 16 * k), desc_mn(ab, 128, 16 * k), idesc, (!first || k > 0) ? 1u : 0u);
            mma_commit(bar + 2);
        }
        first = false;
        // the other stage's buffers are free: its MMA was waited for at the
        // end of the previous iteration
        if (tile + gridDim.x < ntiles) issue_load(tile + gridDim.x, s ^ 1);
        ok = mbar_wait(bar + 2, ph_mma, kWaitLimit) && ok;
        ph_mma ^= 1;
    }
    tc_fence_after();
    // partial of this block: thread t holds accumulator row t (M index)
    float *out = a.part + static_cast<long long>(blockIdx.x) * a.nparam;
    for (int c0 = 0; c0 < ncols; c0 += 32) {
        float v[32];
        if (first) {
#pragma unroll
            for (int j = 0; j < 32; ++j) v[j] = 0.f;
        } else {
            tmem_ld32(lane_addr + c0, v);
        }
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            const int col = c0 + j;
            if (p == 0) {
                if (col < a.P) out[a.off_w3 + static_cast<long long>(col) * kH + t] = v[j];
            } else if (p == 1) {
                out[a.off_w2 + static_cast<long long>(col) * kH + t] = v[j];
            } else {
                if (col < a.da) out[a.off_w1 + static_cast<long long>(t) * a.da + col] = v[j];
                else if (col >= 16 && col < 16 + a.nch) out[a.off_e + static_cast<long long>(col - 16) * kH + t] = v[j];
            }
        }
    }
    if (!ok && t == 0) atomicExch(a.err, 3);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (wp == 0) tmem_dealloc(tbase, 256);
}

// ------------------------------------------------------------------- Adam
// g = sum of the partials in block order (deterministic); Adam with bias
// correction (Kingma & Ba 2015, algorithm 1) on the f32 master copy.
__global__ void k_flow_adam(float *__restrict__ prm, float *__restrict__ m, float *__restrict__ v,
                            const float *__restrict__ part, int nsplit, long long np, float lr, float b1, float b2,
                            float eps, float c1, float c2, float *__restrict__ grad_out) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= np) return;
    float g = 0.f;
    for (int s = 0; s < nsplit; ++s) g += part[s * np + i];
    if (grad_out) grad_out[i] = g;
    if (lr == 0.f) return;
    const float mi = b1 * m[i] + (1.f - b1) * g;
    const float vi = b2 * v[i] + (1.f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    prm[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// f32 master weights of one layer -> its bf16 tiles (zero padding); the W1
// tile also carries E^T in columns 16..16+nch-1.
__global__ void k_flow_pack(const float *__restrict__ w1, const float *__restrict__ E, const float *__restrict__ w2,
                            const float *__restrict__ w3, int da, int nch, int P, uint8_t *__restrict__ wt,
                            uint8_t *__restrict__ wtf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 128 * 64) {
        const int r = i / 64, c = i % 64;
        const float v = c < da ? w1[r * da + c] : ((c >= 16 && c < 16 + nch) ? E[(c - 16) * kH + r] : 0.f);
        *reinterpret_cast<uint16_t *>(wt + sw128_off(r, c, 128)) = static_cast<uint16_t>(pack_bf16x2(v, 0.f) & 0xFFFFu);
    }
    if (i < 128 * 128) {
        const int r = i / 128, c = i % 128;
        *reinterpret_cast<uint16_t *>(wt + kW1Bytes + sw128_off(r, c, 128)) =
            static_cast<uint16_t>(pack_bf16x2(w2[i], 0.f) & 0xFFFFu);
    }
    if (i < kP * 128) {
        const int r = i / 128, c = i % 128;
        const float v = r < P ? w3[r * 128 + c] : 0.f;
        *reinterpret_cast<uint16_t *>(wt + kW1Bytes + kW2Bytes + sw128_off(r, c, kP)) =
            static_cast<uint16_t>(pack_bf16x2(v, 0.f) & 0xFFFFu);
    }
    if (i < kPF * 128) {
        // padded copy: dimension j's parameter q at row 64 j + q
        const int r = i / 128, c = i % 128, j = r / 64, q = r % 64;
        const int src = j * kPerDim + q;
        const float v = (q < kPerDim && src < P) ? w3[src * 128 + c] : 0.f;
        *reinterpret_cast<uint16_t *>(wtf + sw128_off(r, c, kPF)) = static_cast<uint16_t>(pack_bf16x2(v, 0.f) & 0xFFFFu);
    }
}

// ------------------------------------------------------ tensor-core check
// C[128][N] = A op B for the three operand arrangements the flow uses:
// mode 0: A [128][K] K-major, B [N][K] K-major (C = A B^T)
// mode 1: A [K][128] MN-major, B [K][N] MN-major (C = A^T B)
// mode 2: A [128][K] K-major, B [K][N] MN-major (C = A B)
// K and N multiples of 16 in [16, 256]. Inputs f32, rounded to bf16.
constexpr int kSelftestSmem = 128 * 256 * 2 + 256 * 256 * 2 + 64 + 1024;

__global__ void __launch_bounds__(128, 1) k_tc_selftest(int mode, int K, int N, const float *A, const float *B,
                                                        float *C, int *err) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *sm = align1024(smem_raw);
    uint8_t *sA = sm;                  // A tile: at most 128 x 256 (or 256 x 128) bf16
    uint8_t *sB = sm + 128 * 256 * 2;  // B tile: at most 256 x 256 bf16
    uint64_t *bar = reinterpret_cast<uint64_t *>(sB + 256 * 256 * 2);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);
    const int t = threadIdx.x, wp = t >> 5;
    if (t == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    if (wp == 0) tmem_alloc(tslot, 256);
    const int KP = (K + 63) & ~63, NP = (N + 63) & ~63;
    for (int i = t; i < 128 * 256; i += 128) {
        if (mode == 1) {
            const int r = i / 128, c = i % 128;  // [K][128]
            if (r < K)
                *reinterpret_cast<uint16_t *>(sA + sw128_off(r, c, K)) =
                    static_cast<uint16_t>(pack_bf16x2(A[r * 128 + c], 0.f) & 0xFFFFu);
        } else {
            const int r = i / 256, c = i % 256;  // [128][K]
            if (c < KP)
                *reinterpret_cast<uint16_t *>(sA + sw128_off(r, c, 128)) =
                    static_cast<uint16_t>(pack_bf16x2(c < K ? A[r * K + c] : 0.f, 0.f) & 0xFFFFu);
        }
    }
    for (int i = t; i < 256 * 256; i += 128) {
        const int r = i / 256, c = i % 256;
        if (mode == 0) {  // [N][K]
            if (r < N && c < KP)
                *reinterpret_cast<uint16_t *>(sB + sw128_off(r, c, N)) =
                    static_cast<uint16_t>(pack_bf16x2(c < K ? B[r * K + c] : 0.f, 0.f) & 0xFFFFu);
        } else {  // [K][N]
            if (r < K && c < NP)
                *reinterpret_cast<uint16_t *>(sB + sw128_off(r, c, K)) =
                    static_cast<uint16_t>(pack_bf16x2(c < N ? B[r * N + c] : 0.f, 0.f) & 0xFFFFu);
        }
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = *tslot;
    if (t == 0 && mode != 3) {  // mode 3 issues nothing: its wait must give up
        const uint32_t aa = smem_u32(sA), ab = smem_u32(sB);
        const uint32_t id = idesc_bf16(128, N, mode == 1, mode != 0);
        for (int k = 0; k < K / 16; ++k) {
            const uint64_t da = mode == 1 ? desc_mn(aa, K, 16 * k) : desc_k(aa, 128, 16 * k);
            const uint64_t db = mode == 0 ? desc_k(ab, N, 16 * k) : desc_mn(ab, K, 16 * k);
            mma_bf16(tbase, da, db, id, k > 0);
        }
        mma_commit(bar);
    }
    const bool ok = mbar_wait(bar, 0, mode == 3 ? (1u << 16) : kWaitLimit);
    tc_fence_after();
    if (ok) {
        for (int c0 = 0; c0 < N; c0 += 16) {
            float v[16];
            tmem_ld16(tbase + (static_cast<uint32_t>(wp * 32) << 16) + c0, v);
            for (int j = 0; j < 16; ++j) C[t * N + c0 + j] = v[j];
        }
    } else if (t == 0) {
        atomicExch(err, 9);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (wp == 0) tmem_dealloc(tbase, 256);
}

#endif  // CHILI_FLOW_LAYERS_ONLY

}  // namespace chili_flow
