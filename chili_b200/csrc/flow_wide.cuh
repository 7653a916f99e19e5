// flow_wide.cuh -- coupling layers whose conditioner is too large for its
// weights to stay in shared memory: H = 128 or 256 hidden units and 2..4
// hidden layers (3 x 256: 448 KB of bf16 weights per layer, against 227 KB
// of shared memory per CTA).
//
// Conditioner (the same function as the resident-weight kernels of
// flow.cuh, with depth and width as parameters):
//   h_1 = lrelu(W1 (2a - 1) + E[c]),   h_k = lrelu(W2_{k-2} h_{k-1}),
//   theta = W3 h_nh,                   unit H-1 of every h is the constant 1.
//
// Weights of one layer in global memory, bf16 SW128 tiles (tc.cuh):
//   W1T [H][64]   columns 0..da-1 W1, 16..16+nch-1 E^T (one-hot product)
//   W2_m [H][H]   m = 0 .. nh-2
//   W3F [320][H]  W3 with dimension j's 49 rows at rows 64 j .. 64 j + 48
// Every CTA reads the same bytes, so they stay in L2. Each 128-point tile
// streams them through a ring of shared-memory stages: a producer warp
// fills stage s with 1-D bulk copies (cp.async.bulk, no multicast) as soon
// as the tensor core has released it (tcgen05.commit on the stage's "empty"
// mbarrier), while one thread issues the products on the stages already
// filled. The forward kernel streams 64-column blocks (K-major operands);
// the backward kernel streams 64-row slices of the same tiles (MN-major
// operands: four 8 KB pieces per slice). Every wait is bounded; a CTA that
// gives up sets an abort flag that ends the producer's waits, waits for its
// own copies in flight, releases its tensor memory and reports a code.
//
// The kernels are compiled only where CHILI_FLOW_WIDE_KERNELS is defined
// (flow_wide.cu); the argument structures are visible to every includer.
#pragma once

#include "flow.cuh"

namespace chili_flow {

constexpr int kWStages = 3;
constexpr int kWMaxNH = 4;             // hidden layers at most
constexpr int kFStage = kPF * 128;     // 40 KB: the largest forward chunk (64 columns of W3F)
constexpr int kBStage = 4 * 8192;      // 32 KB: a backward chunk (64 rows of a [*][256] tile)
constexpr int kGTileW = 128 * kPF * 2;  // g_theta tile, padded columns (dimension j at 64 j)
constexpr int kSlice = 8192;            // 64 rows x 128 B: one column block of a 64-row slice

__host__ __device__ constexpr long long wide_w1_bytes(int H) { return 128ll * H; }
__host__ __device__ constexpr long long wide_w2_bytes(int H) { return 2ll * H * H; }
__host__ __device__ constexpr long long wide_w3_bytes(int H) { return 2ll * kPF * H; }
__host__ __device__ constexpr long long wide_layer_bytes(int H, int nh) {
    return wide_w1_bytes(H) + (nh - 1) * wide_w2_bytes(H) + wide_w3_bytes(H);
}
__host__ __device__ constexpr int wide_act_bytes(int H) { return 128 * H * 2; }

struct WideLayer {
    const uint8_t *w;  // W1T | W2_0 .. W2_{nh-2} | W3F
    int H, nh, da, db, nch;
    int8_t cond[kMaxDA];
    int8_t trans[8];
};

// ------------------------------------------------------------ helpers
// Named barrier 1 over the n compute threads (the producer warp keeps out).
__device__ __forceinline__ void cbar_sync(int n) { asm volatile("bar.sync 1, %0;" ::"r"(n) : "memory"); }
__device__ __forceinline__ bool cbar_and(int n, bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 q, %1, 0;\n\t"
        "bar.red.and.pred p, 1, %2, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(r)
        : "r"(v ? 1u : 0u), "r"(n)
        : "memory");
    return r != 0;
}

// Bounded wait that also gives up when the compute threads have aborted.
__device__ __forceinline__ bool mbar_wait_or_abort(uint64_t *bar, uint32_t parity, uint32_t limit,
                                                   const volatile int *abort_flag) {
    for (uint32_t i = 0; i < limit; i += 64) {
        if (mbar_wait(bar, parity, 64)) return true;
        if (*abort_flag) return false;
    }
    return false;
}

// Copy of `bytes` (a multiple of 16) by threads 0 .. nthr-1.
__device__ __forceinline__ void copy_n(void *dst, const void *src, int bytes, int tid, int nthr) {
    const uint4 *s = static_cast<const uint4 *>(src);
    uint4 *d = static_cast<uint4 *>(dst);
    for (int i = tid; i < bytes / 16; i += nthr) d[i] = s[i];
}

// The producer warp: chunk c (0 .. nchunks-1) into stage c % kWStages once
// the products of the stage's previous chunk have completed. issue(c, dst,
// bar) runs on lane 0 and arms `bar` with the chunk's bytes.
template <class Issue>
__device__ void wide_producer(long long nchunks, uint8_t *stages, int stage_bytes, uint64_t *full, uint64_t *empty,
                              const volatile int *abort_flag, int *err, int code, Issue issue) {
    const int lane = threadIdx.x & 31;
    long long c = 0;
    bool ok = true;
    for (; c < nchunks; ++c) {
        // lane 0 waits and issues; the warp follows its decision
        int got = 0;
        if (lane == 0) {
            const int s = static_cast<int>(c % kWStages);
            const uint32_t par = static_cast<uint32_t>((c / kWStages) & 1) ^ 1u;
            got = mbar_wait_or_abort(empty + s, par, kWaitLimit, abort_flag) ? 1 : 0;
            if (got) issue(c, stages + static_cast<long long>(s) * stage_bytes, full + s);
        }
        got = __shfl_sync(0xffffffffu, got, 0);
        if (!got) {
            ok = false;
            break;
        }
    }
    if (lane == 0) {
        // copies in flight complete on their own: wait for each stage's last fill
        for (int s = 0; s < kWStages; ++s) {
            if (c > s) {
                const long long u = ((c - 1 - s) / kWStages) * kWStages + s;
                mbar_wait(full + s, static_cast<uint32_t>((u / kWStages) & 1), kWaitLimit);
            }
        }
        if (!ok && !*abort_flag) atomicExch(err, code);
    }
    __syncwarp();
}

// The consumer side (one thread): waits for chunk c to land in its stage
// (false: the bounded wait gave up).
__device__ __forceinline__ bool wide_take(uint64_t *full, long long c) {
    return mbar_wait(full + c % kWStages, static_cast<uint32_t>((c / kWStages) & 1), kWaitLimit);
}

// Forward chunk k of a tile (1 + nh * H/64 chunks): W1T, then the 64-column
// blocks of W2_0 .. W2_{nh-2}, then those of W3F. Contiguous.
__device__ __forceinline__ void wide_fwd_chunk(const WideLayer &L, int k, const uint8_t *&src, uint32_t &bytes) {
    const int H = L.H, nb = H / 64;
    if (k == 0) {
        src = L.w;
        bytes = static_cast<uint32_t>(wide_w1_bytes(H));
        return;
    }
    const int k2 = k - 1;
    const uint8_t *w2 = L.w + wide_w1_bytes(H);
    if (k2 < (L.nh - 1) * nb) {
        src = w2 + (k2 / nb) * wide_w2_bytes(H) + static_cast<long long>(k2 % nb) * H * 128;
        bytes = static_cast<uint32_t>(H * 128);
        return;
    }
    src = w2 + (L.nh - 1) * wide_w2_bytes(H) + static_cast<long long>(k2 - (L.nh - 1) * nb) * kPF * 128;
    bytes = static_cast<uint32_t>(kPF * 128);
}

// Backward chunk k of a tile (db + nh * H/64 chunks): 64-row slices of W3F
// (dimension k's padded rows), then of W2_{nh-2} .. W2_0, then of W1T; a
// slice of a [*][H] tile is H/64 pieces of 8 KB (one per column block), laid
// out as an SW128 tile of 64 rows.
__device__ __forceinline__ void wide_bwd_issue(const WideLayer &L, int k, uint8_t *dst, uint64_t *bar) {
    const int H = L.H, nb = H / 64;
    const uint8_t *w2 = L.w + wide_w1_bytes(H);
    const uint8_t *w3 = w2 + (L.nh - 1) * wide_w2_bytes(H);
    if (k < L.db) {
        mbar_expect_tx(bar, static_cast<uint32_t>(nb * kSlice));
        for (int cb = 0; cb < nb; ++cb)
            bulk_g2s(dst + cb * kSlice, w3 + static_cast<long long>(cb) * kPF * 128 + k * kSlice, kSlice, bar);
        return;
    }
    const int k2 = k - L.db;
    if (k2 < (L.nh - 1) * nb) {
        const int m = L.nh - 2 - k2 / nb, q = k2 % nb;
        mbar_expect_tx(bar, static_cast<uint32_t>(nb * kSlice));
        for (int cb = 0; cb < nb; ++cb)
            bulk_g2s(dst + cb * kSlice, w2 + m * wide_w2_bytes(H) + static_cast<long long>(cb) * H * 128 + q * kSlice,
                     kSlice, bar);
        return;
    }
    const int q = k2 - (L.nh - 1) * nb;
    mbar_expect_tx(bar, kSlice);
    bulk_g2s(dst, L.w + q * kSlice, kSlice, bar);
}

// h = lrelu(accumulator), unit H-1 = 1, into the activation tile; thread
// group grp (0..3) takes columns grp*H/4 ..
template <int H>
__device__ __forceinline__ void wide_hidden_epilogue(int grp, int r, uint32_t lane_addr, uint8_t *sH) {
    if (grp >= 4) return;
    constexpr int W = H / 4;
#pragma unroll
    for (int q = 0; q < W / 32; ++q) {
        const int c0 = grp * W + 32 * q;
        float v[32];
        tmem_ld32(lane_addr + c0, v);
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            v[j] = lrelu(v[j]);
            if (c0 + j == H - 1) v[j] = 1.f;
        }
        store_row32(sH, 128, r, c0, v);
    }
}

// g_p = accumulator * lrelu'(h) (h from the saved tile), unit H-1 and rows
// beyond n -> 0, into the gradient tile.
template <int H>
__device__ __forceinline__ void wide_grad_epilogue(int grp, int r, uint32_t lane_addr, const uint8_t *htile, bool valid,
                                                   uint8_t *sP) {
    constexpr int W = H / 4;
#pragma unroll
    for (int q = 0; q < W / 32; ++q) {
        const int c0 = grp * W + 32 * q;
        float v[32], hv[32];
        tmem_ld32(lane_addr + c0, v);
        load_row32(htile, 128, r, c0, hv);
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            v[j] *= hv[j] > 0.f ? 1.f : kSlope;
            if (c0 + j == H - 1 || !valid) v[j] = 0.f;
        }
        store_row32(sP, 128, r, c0, v);
    }
}

// 64 accumulator columns from taddr, two loads in flight.
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float (&v)[64]) {
    uint32_t r0[32], r1[32];
    tmem_ld32_async(taddr, r0);
    tmem_ld32_async(taddr + 32, r1);
    tmem_wait_ld();
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        v[i] = __uint_as_float(r0[i]);
        v[32 + i] = __uint_as_float(r1[i]);
    }
}

// ------------------------------------------------- coupling layer, forward
// MODE 0: density direction, MODE 1: sampling direction; SAVE keeps the
// hidden activation tiles (hs [nh][tiles][128 x H bf16]) and theta for the
// backward pass. logq[i] += sum log dy/dx.
struct WideFwdArgs {
    WideLayer L;
    long long n;
    const float *xin;  // [D][n]
    float *xout;       // [D][n]
    const int32_t *ch;
    float *logq;
    uint8_t *hs;   // SAVE
    float *theta;  // [db*49][n] (SAVE)
    int *err;
};

// Five thread groups of 128 (one point per thread; groups 0-3 split the
// hidden columns of the epilogues, group j evaluates dimension j's spline)
// and the producer warp.
constexpr int kWFwdCompute = 640;
constexpr int kWFwdThreads = kWFwdCompute + 32;
template <int H>
constexpr int wide_fwd_smem() {
    return 128 * 64 * 2 + wide_act_bytes(H) + kWStages * kFStage + 4 * 128 * 4 + 128 + 1024;
}

#ifdef CHILI_FLOW_WIDE_KERNELS
template <int H, int MODE, bool SAVE>
__global__ void __launch_bounds__(kWFwdThreads, 1) k_flow_layer_wide(WideFwdArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *sm = align1024(smem_raw);
    uint8_t *sA = sm;                        // [128][64]: 2a - 1 and the one-hot channel
    uint8_t *sH = sA + 128 * 64 * 2;         // [128][H]: the current hidden layer
    uint8_t *sS = sH + wide_act_bytes(H);    // weight stages
    float *sL = reinterpret_cast<float *>(sS + kWStages * kFStage);  // [4][128] log-det partials
    uint64_t *full = reinterpret_cast<uint64_t *>(sL + 4 * 128);
    uint64_t *empty = full + kWStages;
    uint64_t *accb = empty + kWStages;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(accb + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tslot + 1);
    const int t = threadIdx.x, wp = t >> 5;
    const long long n = a.n;
    const long long ntiles = (n + 127) / 128;
    constexpr int nb = H / 64;
    const int nh = a.L.nh;
    const int per_tile = 1 + nh * nb;

    if (t == 0) {
        for (int s = 0; s < kWStages; ++s) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, 1);
        }
        mbar_init(accb, 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (wp == 0) tmem_alloc(tslot, 512);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = *tslot;
    const long long my_tiles =
        static_cast<long long>(blockIdx.x) < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    if (wp == kWFwdCompute / 32) {
        const WideLayer L = a.L;
        wide_producer(my_tiles * per_tile, sS, kFStage, full, empty, abort_flag, a.err, 12,
                      [&](long long c, uint8_t *dst, uint64_t *bar) {
                          const uint8_t *src;
                          uint32_t bytes;
                          wide_fwd_chunk(L, static_cast<int>(c % per_tile), src, bytes);
                          mbar_expect_tx(bar, bytes);
                          bulk_g2s(dst, src, bytes, bar);
                      });
    } else {
        const int grp = wp >> 2;
        const int r = (wp & 3) * 32 + (t & 31);
        const uint32_t lane_addr = tbase + (static_cast<uint32_t>((wp & 3) * 32) << 16);
        const uint32_t aA = smem_u32(sA), aH = smem_u32(sH), aS = smem_u32(sS);
        const int DB = a.L.db, da = a.L.da;
        const uint32_t id_h = idesc_bf16(128, H, false, false);
        const uint32_t id_p1 = idesc_bf16(128, 64 * (DB < 4 ? DB : 4), false, false);
        const uint32_t id_p2 = idesc_bf16(128, 64, false, false);
        constexpr int act = wide_act_bytes(H);
        uint32_t acc_phase = 0;
        long long cc = 0;  // chunks consumed (thread 0)
        bool ok = true;
        for (long long tile = blockIdx.x;; tile += gridDim.x) {
            const bool go = cbar_and(kWFwdCompute, ok);
            if (!go || tile >= ntiles) {
                ok = go;
                break;
            }
            const long long row = tile * 128 + r;
            const bool valid = row < n;
            // this thread's spline input and (group 0) the point's log q,
            // loaded now so that their latency hides behind the products
            const int dsp = grp < DB ? a.L.trans[grp] : 0;
            const float xsp = (valid && grp < DB) ? a.xin[dsp * n + row] : 0.5f;
            const float lq0 = (valid && grp == 0) ? a.logq[row] : 0.f;
            if (grp < 2) {
                int c = valid ? a.ch[row] : 0;
                c = (c >= 0 && c < a.L.nch) ? c : 0;  // channel indices come from callers
                float av[32];
                if (grp == 0) {
#pragma unroll
                    for (int i = 0; i < 16; ++i) {
                        float v = 0.f;
                        if (i < da && valid) v = 2.f * fminf(fmaxf(a.xin[a.L.cond[i] * n + row], 0.f), 1.f) - 1.f;
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
                for (int i = 0; i < da; ++i) a.xout[a.L.cond[i] * n + row] = a.xin[a.L.cond[i] * n + row];
            }
            fence_async_smem();
            tc_fence_before();
            cbar_sync(kWFwdCompute);
            // h_1 = lrelu(W1 a + E[c])
            if (t == 0) {
                tc_fence_after();
                const bool g = wide_take(full, cc);
                const uint32_t st = aS + static_cast<uint32_t>(cc % kWStages) * kFStage;
                if (g)
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        mma_bf16(tbase, desc_k(aA, 128, 16 * k), desc_k(st, H, 16 * k), id_h, k > 0);
                mma_commit(empty + cc % kWStages);
                ++cc;
                mma_commit(accb);
                ok = ok && g;
            }
            ok = mbar_wait(accb, acc_phase, kWaitLimit) && ok;
            acc_phase ^= 1;
            tc_fence_after();
            wide_hidden_epilogue<H>(grp, r, lane_addr, sH);
            fence_async_smem();
            tc_fence_before();
            cbar_sync(kWFwdCompute);
            // h_{m+2} = lrelu(W2_m h_{m+1})
            for (int m = 0; m < nh - 1; ++m) {
                if (t == 0) {
                    tc_fence_after();
                    for (int q = 0; q < nb; ++q) {
                        const bool g = wide_take(full, cc);
                        const uint32_t st = aS + static_cast<uint32_t>(cc % kWStages) * kFStage;
                        if (g)
#pragma unroll
                            for (int k = 0; k < 4; ++k)
                                mma_bf16(tbase, desc_k(aH, 128, 64 * q + 16 * k), desc_k(st, H, 16 * k), id_h,
                                         (q | k) > 0);
                        mma_commit(empty + cc % kWStages);
                        ++cc;
                        ok = ok && g;
                    }
                    mma_commit(accb);
                }
                if (SAVE) copy_n(a.hs + (m * ntiles + tile) * act, sH, act, t, kWFwdCompute);
                ok = mbar_wait(accb, acc_phase, kWaitLimit) && ok;
                acc_phase ^= 1;
                tc_fence_after();
                cbar_sync(kWFwdCompute);  // the copy of h is complete before it is overwritten
                wide_hidden_epilogue<H>(grp, r, lane_addr, sH);
                fence_async_smem();
                tc_fence_before();
                cbar_sync(kWFwdCompute);
            }
            // theta = W3 h_nh: dimensions 0 .. min(DB, 4) - 1 at accumulator
            // columns 0 .., dimension 4 at columns 256 .. 319
            if (t == 0) {
                tc_fence_after();
                for (int q = 0; q < nb; ++q) {
                    const bool g = wide_take(full, cc);
                    const uint32_t st = aS + static_cast<uint32_t>(cc % kWStages) * kFStage;
                    if (g) {
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            mma_bf16(tbase, desc_k(aH, 128, 64 * q + 16 * k), desc_k(st, kPF, 16 * k), id_p1,
                                     (q | k) > 0);
                            if (DB == 5)
                                mma_bf16(tbase + 256, desc_k(aH, 128, 64 * q + 16 * k),
                                         desc_k(st + 256 * 128, 64, 16 * k), id_p2, (q | k) > 0);
                        }
                    }
                    mma_commit(empty + cc % kWStages);
                    ++cc;
                    ok = ok && g;
                }
                mma_commit(accb);
            }
            if (SAVE) copy_n(a.hs + ((nh - 1) * ntiles + tile) * act, sH, act, t, kWFwdCompute);
            ok = mbar_wait(accb, acc_phase, kWaitLimit) && ok;
            acc_phase ^= 1;
            tc_fence_after();
            float lsum = 0.f;
            if (grp < DB) {  // dimension grp on group grp (DB <= 5)
                const int j = grp;
                float th[64];
                tmem_ld64(lane_addr + static_cast<uint32_t>(64 * j), th);
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
            tc_fence_before();
            cbar_sync(kWFwdCompute);
            if (grp == 0 && valid) a.logq[row] = lq0 + (lsum + sL[r] + sL[128 + r] + sL[256 + r] + sL[384 + r]);
        }
        if (!ok && t == 0) {
            *abort_flag = 1;
            atomicExch(a.err, 11);
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (wp == 0) tmem_dealloc(tbase, 512);
}
#endif  // CHILI_FLOW_WIDE_KERNELS

// ------------------------------------------------ coupling layer, backward
// Data gradients of one layer: spline backward (theta and x saved by the
// forward pass) -> g_theta; g_h_nh = g_theta W3; per hidden layer k from the
// last: g_p_k = g_h_k * lrelu'(h_k) (unit H-1 -> 0), g_h_{k-1} = g_p_k W2;
// g_a = g_p_1 W1. Writes the gradient of the layer input and the bf16 tiles
// of g_theta (padded columns) and of every g_p for the weight gradients.
struct WideBwdArgs {
    WideLayer L;
    long long n;
    const float *xin;    // layer input [D][n]
    const float *theta;  // [db*49][n]
    const uint8_t *hs;   // [nh][tiles][act]
    const float *gout;   // gradient of the layer output [D][n], or null (last layer)
    const float *glogq;  // d loss / d log q [n]
    float *gin;          // gradient of the layer input [D][n]
    uint8_t *gths;       // [tiles][kGTileW]
    uint8_t *gps;        // [nh][tiles][act]
    int *err;
};

constexpr int kWBwdCompute = 512;  // four groups of 128 (one point per thread)
constexpr int kWBwdThreads = kWBwdCompute + 32;
constexpr int kWBwdSmem = kGTileW + kWStages * kBStage + 128 + 1024;

#ifdef CHILI_FLOW_WIDE_KERNELS
template <int H>
__global__ void __launch_bounds__(kWBwdThreads, 1) k_flow_layer_bwd_wide(WideBwdArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *sm = align1024(smem_raw);
    uint8_t *sG = sm;  // g_theta [128][320]; the g_p tiles [128][H] reuse its first bytes
    uint8_t *sP = sm;
    uint8_t *sS = sm + kGTileW;
    uint64_t *full = reinterpret_cast<uint64_t *>(sS + kWStages * kBStage);
    uint64_t *empty = full + kWStages;
    uint64_t *accb = empty + kWStages;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(accb + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tslot + 1);
    const int t = threadIdx.x, wp = t >> 5;
    const long long n = a.n;
    const long long ntiles = (n + 127) / 128;
    constexpr int nb = H / 64;
    const int nh = a.L.nh, DB = a.L.db;
    const int per_tile = DB + nh * nb;

    if (t == 0) {
        for (int s = 0; s < kWStages; ++s) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, 1);
        }
        mbar_init(accb, 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (wp == 0) tmem_alloc(tslot, 256);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = *tslot;
    const long long my_tiles =
        static_cast<long long>(blockIdx.x) < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    if (wp == kWBwdCompute / 32) {
        const WideLayer L = a.L;
        wide_producer(my_tiles * per_tile, sS, kBStage, full, empty, abort_flag, a.err, 14,
                      [&](long long c, uint8_t *dst, uint64_t *bar) {
                          wide_bwd_issue(L, static_cast<int>(c % per_tile), dst, bar);
                      });
    } else {
        const int grp = wp >> 2;
        const int r = (wp & 3) * 32 + (t & 31);
        const uint32_t lane_addr = tbase + (static_cast<uint32_t>((wp & 3) * 32) << 16);
        const uint32_t aG = smem_u32(sG), aS = smem_u32(sS);
        const uint32_t id_h = idesc_bf16(128, H, false, true);
        const uint32_t id_ga = idesc_bf16(128, 64, false, true);
        constexpr int act = wide_act_bytes(H);
        const int da = a.L.da;
        uint32_t acc_phase = 0;
        long long cc = 0;
        bool ok = true;
        // one K step chain of a product: the stages of `chunks` consecutive
        // chunks, A = the gradient tile (K-major, 64 columns per chunk)
        auto product = [&](int chunks, uint32_t idesc) {
            tc_fence_after();
            for (int q = 0; q < chunks; ++q) {
                const bool g = wide_take(full, cc);
                const uint32_t st = aS + static_cast<uint32_t>(cc % kWStages) * kBStage;
                if (g)
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        mma_bf16(tbase, desc_k(aG, 128, 64 * q + 16 * k), desc_mn(st, 64, 16 * k), idesc,
                                 (q | k) > 0);
                mma_commit(empty + cc % kWStages);
                ++cc;
                ok = ok && g;
            }
            mma_commit(accb);
        };
        for (long long tile = blockIdx.x;; tile += gridDim.x) {
            const bool go = cbar_and(kWBwdCompute, ok);
            if (!go || tile >= ntiles) {
                ok = go;
                break;
            }
            const long long row = tile * 128 + r;
            const bool valid = row < n;
            const float gl = valid ? a.glogq[row] : 0.f;
            // spline backward -> g_theta, dimension j in columns 64 j .. 64 j + 48
#pragma unroll 1
            for (int j = grp; j < DB; j += 4) {
                const int b0 = j * kPerDim;
                float th[kPerDim], g[kPerDim];
#pragma unroll
                for (int i = 0; i < kPerDim; ++i) th[i] = valid ? a.theta[(b0 + i) * n + row] : 0.f;
                const int d = a.L.trans[j];
                const float x = valid ? fminf(fmaxf(a.xin[d * n + row], 0.f), 1.f) : 0.5f;
                const float gy = (valid && a.gout) ? a.gout[d * n + row] : 0.f;
                const float gx = rqs_backward(th, x, gy, valid ? gl : 0.f, g);
                if (valid) a.gin[d * n + row] = gx;
                float v[32];
#pragma unroll
                for (int i = 0; i < 32; ++i) v[i] = valid ? g[i] : 0.f;
                store_row32(sG, 128, r, 64 * j, v);
#pragma unroll
                for (int i = 0; i < 32; ++i) v[i] = (valid && 32 + i < kPerDim) ? g[32 + i] : 0.f;
                store_row32(sG, 128, r, 64 * j + 32, v);
            }
            fence_async_smem();
            tc_fence_before();
            cbar_sync(kWBwdCompute);
            if (t == 0) product(DB, id_h);  // g_h_nh = g_theta W3 (K: the DB padded row blocks)
            copy_n(a.gths + tile * kGTileW, sG, DB * 128 * 128, t, kWBwdCompute);
            ok = mbar_wait(accb, acc_phase, kWaitLimit) && ok;
            acc_phase ^= 1;
            tc_fence_after();
            cbar_sync(kWBwdCompute);  // the copy of g_theta is complete before g_p overwrites it
            wide_grad_epilogue<H>(grp, r, lane_addr, a.hs + ((nh - 1) * ntiles + tile) * act, valid, sP);
            fence_async_smem();
            tc_fence_before();
            cbar_sync(kWBwdCompute);
            for (int m = nh - 2; m >= 0; --m) {
                if (t == 0) product(nb, id_h);  // g_h_{m+1} = g_p_{m+2} W2_m (1-based layers)
                copy_n(a.gps + ((m + 1) * ntiles + tile) * act, sP, act, t, kWBwdCompute);
                ok = mbar_wait(accb, acc_phase, kWaitLimit) && ok;
                acc_phase ^= 1;
                tc_fence_after();
                cbar_sync(kWBwdCompute);
                wide_grad_epilogue<H>(grp, r, lane_addr, a.hs + (m * ntiles + tile) * act, valid, sP);
                fence_async_smem();
                tc_fence_before();
                cbar_sync(kWBwdCompute);
            }
            if (t == 0) product(nb, id_ga);  // g_a = g_p_1 W1 (columns 0 .. 15 used)
            copy_n(a.gps + tile * act, sP, act, t, kWBwdCompute);
            ok = mbar_wait(accb, acc_phase, kWaitLimit) && ok;
            acc_phase ^= 1;
            tc_fence_after();
            if (grp == 0) {
                float ga[16];
                tmem_ld16(lane_addr, ga);
                if (valid) {
#pragma unroll
                    for (int i = 0; i < kMaxDA; ++i)
                        if (i < da) {
                            const int d = a.L.cond[i];
                            a.gin[d * n + row] = (a.gout ? a.gout[d * n + row] : 0.f) + 2.f * ga[i];
                        }
                }
            }
            tc_fence_before();
        }
        if (!ok && t == 0) {
            *abort_flag = 1;
            atomicExch(a.err, 13);
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (wp == 0) tmem_dealloc(tbase, 256);
}
#endif  // CHILI_FLOW_WIDE_KERNELS

// ------------------------------------------------------- weight gradients
// One product (item blockIdx.y) summed over this block's share of the point
// tiles (K = points), M = 128 of the output's H-sized side, written as this
// block's partial (blockIdx.x) in the flat gradient layout:
//   kind 0: dW3[p][h]  = sum_r g_theta[r][p] h_nh[r][h]   (A = h_nh,  B = g_theta columns 256 np ..)
//   kind 1: dW2_m[o][i] = sum_r g_p_{m+2}[r][o] h_{m+1}[r][i]  (A = h_{m+1}, B = g_p_{m+2})
//   kind 2: dW1[h][i]  = sum_r g_p_1[r][h] a[r][i],  dE[c][h] = sum_{r: c_r = c} g_p_1[r][h]
//           (A = g_p_1, B = [a | 0 | onehot(c)] built here)
// (1-based hidden layers.) Both operands are MN-major views of the saved
// row-major tiles; A is the 32 KB column slice mh of a tile.
struct WideWgradItem {
    int8_t kind, m, mh, np;
};
struct WideWgradArgs {
    long long n;
    int H, nh, da, db, nch, ncol2;  // ncol2: columns of the kind-2 B tile (16 + nch, rounded up to 64)
    int8_t cond[kMaxDA];
    const float *xin;
    const int32_t *ch;
    const uint8_t *hs, *gps, *gths;
    float *part;       // [nsplit][nparam]
    long long nparam;  // stride between partials
    long long off_w1, off_e, off_w3, off_w2[kWMaxNH - 1];
    int nitems;
    WideWgradItem item[16];
    int *err;
};

constexpr int kWgA = 128 * 128 * 2;
constexpr int kWgB = 128 * 256 * 2;
constexpr int kWgWideSmem = 2 * (kWgA + kWgB) + 64 + 1024;

#ifdef CHILI_FLOW_WIDE_KERNELS
__global__ void __launch_bounds__(128, 1) k_flow_wgrad_wide(WideWgradArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *sm = align1024(smem_raw);
    uint8_t *sA[2] = {sm, sm + kWgA};
    uint8_t *sB[2] = {sm + 2 * kWgA, sm + 2 * kWgA + kWgB};
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + 2 * (kWgA + kWgB));
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 4);
    const int t = threadIdx.x, wp = t >> 5;
    const WideWgradItem it = a.item[blockIdx.y];
    const long long n = a.n;
    const long long ntiles = (n + 127) / 128;
    const int H = a.H;
    const long long act = wide_act_bytes(H);
    const int db4 = a.db < 4 ? a.db : 4;
    int ncols;
    const uint8_t *srcA, *srcB = nullptr;
    long long strideB = act, offB = 0;
    if (it.kind == 0) {
        srcA = a.hs + (a.nh - 1) * ntiles * act;
        srcB = a.gths;
        strideB = kGTileW;
        offB = static_cast<long long>(it.np) * 4 * 128 * 128;
        ncols = it.np == 0 ? 64 * db4 : 64;
    } else if (it.kind == 1) {
        srcA = a.hs + it.m * ntiles * act;
        srcB = a.gps + (it.m + 1) * ntiles * act;
        ncols = H;
    } else {
        srcA = a.gps;
        ncols = a.ncol2;
    }
    const long long offA = static_cast<long long>(it.mh) * kWgA;
    const int bbytes = 128 * ncols * 2;
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
            mbar_expect_tx(bar + s, static_cast<uint32_t>(kWgA + (srcB ? bbytes : 0)));
            bulk_g2s(sA[s], srcA + tile * act + offA, kWgA, bar + s);
            if (srcB) bulk_g2s(sB[s], srcB + tile * strideB + offB, static_cast<uint32_t>(bbytes), bar + s);
        }
    };
    long long tile = blockIdx.x;
    if (tile < ntiles) issue_load(tile, 0);
    int s = 0;
    for (; __syncthreads_and(ok) && tile < ntiles; tile += gridDim.x, s ^= 1) {
        if (it.kind == 2) {
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
        if (t == 0 && ok) {
            tc_fence_after();
            const uint32_t aa = smem_u32(sA[s]), ab = smem_u32(sB[s]);
#pragma unroll
            for (int k = 0; k < 8; ++k)
                mma_bf16(tbase, desc_mn(aa, 128, 16 * k), desc_mn(ab, 128, 16 * k), idesc, (!first || k > 0) ? 1u : 0u);
        }
        if (t == 0) mma_commit(bar + 2);
        first = false;
        // the other stage's buffers are free: its products were waited for at
        // the end of the previous iteration
        if (tile + gridDim.x < ntiles) issue_load(tile + gridDim.x, s ^ 1);
        ok = mbar_wait(bar + 2, ph_mma, kWaitLimit) && ok;
        ph_mma ^= 1;
    }
    // loads still in flight when the loop ended early (the one given up on,
    // and the one issued for the tile this block did not reach) complete on
    // their own: wait for them before the block exits
    if (t == 0 && tile < ntiles) {
        mbar_wait(bar + s, ph_load[s], kWaitLimit);
        mbar_wait(bar + (s ^ 1), ph_load[s ^ 1] ^ 1u, kWaitLimit);
    }
    tc_fence_after();
    float *out = a.part + static_cast<long long>(blockIdx.x) * a.nparam;
    const int mrow = it.mh * 128 + t;  // the output's H-side index of this thread
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
            if (it.kind == 0) {
                const int pc = 256 * it.np + col, jd = pc >> 6, q = pc & 63;
                if (jd < a.db && q < kPerDim) out[a.off_w3 + static_cast<long long>(jd * kPerDim + q) * H + mrow] = v[j];
            } else if (it.kind == 1) {
                out[a.off_w2[it.m] + static_cast<long long>(col) * H + mrow] = v[j];
            } else {
                if (col < a.da) out[a.off_w1 + static_cast<long long>(mrow) * a.da + col] = v[j];
                else if (col >= 16 && col < 16 + a.nch) out[a.off_e + static_cast<long long>(col - 16) * H + mrow] = v[j];
            }
        }
    }
    if (!ok && t == 0) atomicExch(a.err, 15);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (wp == 0) tmem_dealloc(tbase, 256);
}
#endif  // CHILI_FLOW_WIDE_KERNELS

// f32 master weights of one layer -> its bf16 tiles (region blockIdx.y:
// 0 W1T, 1 .. nh-1 W2_{region-1}, nh W3F; zero padding).
struct WidePackArgs {
    const float *prm;
    long long off_w1, off_e, off_w3, off_w2[kWMaxNH - 1];
    int H, nh, da, nch, db;
    uint8_t *w;
};

#ifdef CHILI_FLOW_WIDE_KERNELS
__global__ void k_flow_pack_wide(WidePackArgs a) {
    const int region = blockIdx.y;
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    const int H = a.H;
    float v;
    uint8_t *dst;
    if (region == 0) {
        if (i >= 64ll * H) return;
        const int r = static_cast<int>(i / 64), c = static_cast<int>(i % 64);
        v = c < a.da ? a.prm[a.off_w1 + static_cast<long long>(r) * a.da + c]
                     : ((c >= 16 && c < 16 + a.nch) ? a.prm[a.off_e + static_cast<long long>(c - 16) * H + r] : 0.f);
        dst = a.w + sw128_off(r, c, H);
    } else if (region < a.nh) {
        if (i >= static_cast<long long>(H) * H) return;
        const int r = static_cast<int>(i / H), c = static_cast<int>(i % H);
        v = a.prm[a.off_w2[region - 1] + i];
        dst = a.w + wide_w1_bytes(H) + (region - 1) * wide_w2_bytes(H) + sw128_off(r, c, H);
    } else {
        if (i >= static_cast<long long>(kPF) * H) return;
        const int r = static_cast<int>(i / H), c = static_cast<int>(i % H), j = r / 64, q = r % 64;
        v = (q < kPerDim && j < a.db) ? a.prm[a.off_w3 + static_cast<long long>(j * kPerDim + q) * H + c] : 0.f;
        dst = a.w + wide_w1_bytes(H) + (a.nh - 1) * wide_w2_bytes(H) + sw128_off(r, c, kPF);
    }
    *reinterpret_cast<uint16_t *>(dst) = static_cast<uint16_t>(pack_bf16x2(v, 0.f) & 0xFFFFu);
}
#endif  // CHILI_FLOW_WIDE_KERNELS

}  // namespace chili_flow
