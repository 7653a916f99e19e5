// common.cuh -- device value types, the counter-based generator and helpers
// shared by the kernels of libchili_b200.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace chili_dev {

constexpr double kPi = 3.14159265358979323846;  // M_PI
constexpr double kTwoPi = 2.0 * kPi;            // 2*M_PI, exact doubling

// std::min / std::max semantics (return the first argument unless the second
// compares strictly smaller / larger), which decide how NaN propagates.
__device__ __forceinline__ double std_min(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double std_max(double a, double b) { return (a < b) ? b : a; }

// ------------------------------------------------------------ four-vectors
// (E, px, py, pz), FP64, the component order of chili::FourVector.
struct V4 {
    double e, x, y, z;
};

__device__ __forceinline__ V4 v4(double e, double x, double y, double z) { return V4{e, x, y, z}; }
__device__ __forceinline__ V4 operator+(V4 a, V4 b) { return V4{a.e + b.e, a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V4 operator-(V4 a, V4 b) { return V4{a.e - b.e, a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V4 scale(V4 a, double s) { return V4{a.e * s, a.x * s, a.y * s, a.z * s}; }
// Products of momenta round every product and sum separately, in the
// reference's order (FourVector.cc operator*, FourVector.hh Pt2/P2), as its
// x86-64 build does: a contracted multiply-add would round differently, and
// the cancellation in the invariant mass of nearly collinear momenta (the
// compound currents of nested decays) amplifies that to ~1e-9.
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
// Minkowski product E E' - ((px px' + py py') + pz pz')
__device__ __forceinline__ double dot4(V4 a, V4 b) {
    return __dsub_rn(dmul(a.e, b.e), dadd(dadd(dmul(a.x, b.x), dmul(a.y, b.y)), dmul(a.z, b.z)));
}
__device__ __forceinline__ double mass2(V4 a) { return dot4(a, a); }
__device__ __forceinline__ double pt2(V4 a) { return dadd(dmul(a.x, a.x), dmul(a.y, a.y)); }
__device__ __forceinline__ double p2(V4 a) { return dadd(pt2(a), dmul(a.z, a.z)); }
__device__ __forceinline__ double dot3(V4 a, V4 b) { return dadd(dadd(dmul(a.x, b.x), dmul(a.y, b.y)), dmul(a.z, b.z)); }
__device__ __forceinline__ double rapidity(V4 a) {
    if (a.e == 0) return 99;
    return log((a.e + a.z) / (a.e - a.z)) / 2;
}
__device__ __forceinline__ double phi_0_2pi(V4 a) {
    const double p = atan2(a.y, a.x);
    if (p < 0) return p + kTwoPi;
    return p;
}
__device__ __forceinline__ double comp(const V4 &a, int i) {
    return i == 0 ? a.e : (i == 1 ? a.x : (i == 2 ? a.y : a.z));
}
__device__ __forceinline__ void set_comp(V4 &a, int i, double v) {
    if (i == 0) a.e = v;
    else if (i == 1) a.x = v;
    else if (i == 2) a.y = v;
    else a.z = v;
}

// ---------------------------------------------------------------- Philox
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11): 10 rounds of two 32x32->64 multiplies with a Weyl key
// schedule.  Point k of a run draws uniform j from the block
// ctr = {j/2, lo32(k), hi32(k), stream}, key = {lo32(seed), hi32(seed)}.
struct U4 {
    uint32_t a, b, c, d;
};

__host__ __device__ __forceinline__ U4 philox4x32_10(U4 ctr, uint32_t k0, uint32_t k1) {
    constexpr uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    constexpr uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = static_cast<uint64_t>(M0) * ctr.a;
        const uint64_t p1 = static_cast<uint64_t>(M1) * ctr.c;
        const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
        const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
        ctr = U4{hi1 ^ ctr.b ^ k0, lo1, hi0 ^ ctr.d ^ k1, lo0};
        k0 += W0;
        k1 += W1;
    }
    return ctr;
}

// 53 random bits -> [0, 1): (hi << 21 | lo >> 11) * 2^-53
__host__ __device__ __forceinline__ double u53(uint32_t hi, uint32_t lo) {
    const uint64_t bits = (static_cast<uint64_t>(hi) << 21) | (lo >> 11);
    return static_cast<double>(bits) * 0x1.0p-53;
}

// Uniforms 2q and 2q+1 of point `k` of stream `stream`.
__host__ __device__ __forceinline__ void uniform_pair(uint64_t seed, uint64_t k, uint32_t stream,
                                                     uint32_t q, double &u0, double &u1) {
    const U4 r = philox4x32_10(U4{q, static_cast<uint32_t>(k), static_cast<uint32_t>(k >> 32), stream},
                               static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32));
    u0 = u53(r.a, r.b);
    u1 = u53(r.c, r.d);
}

// Stream ids keep different consumers of one seed apart.
constexpr uint32_t kStreamPoints = 0;  // VEGAS / multichannel points
constexpr uint32_t kStreamAccept = 1;  // hit-or-miss uniforms of the unweighting stage

// ------------------------------------------------------------ reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = std_min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = std_max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// StatsData partial (Statistics.hh:62-142): n, min, max, sum, sum2, n_finite.
struct Stats6 {
    double n, mn, mx, sum, sum2, nfin;
};

}  // namespace chili_dev
