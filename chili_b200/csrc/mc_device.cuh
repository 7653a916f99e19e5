// mc_device.cuh -- types and device helpers shared by the kernels of
// libchili_b200 (kernels.cuh, pipeline.cuh, flow_phys.cuh): iteration
// accumulator and round records, the channel-selection rule, the checked
// grid map and the counter-based uniforms.
#pragma once

#include "channel_program.h"
#include "common.cuh"
#include "fsmapper.cuh"
#include "grid.cuh"
#include "integrands.cuh"

namespace chili_dev {

constexpr int kFwdBlock = 256;
constexpr int kWgtBlock = 128;
constexpr int kVegasBlock = 256;

// Iteration accumulator of a multichannel iteration (device resident).
struct IterAcc {
    double st[6];      // n, min, max, sum, sum2, n_finite
    double nan_count;  // NaN-value retries
    double nonfinite;  // dropped alpha-training terms (guard mode)
    double wmax;       // max value
    double dropped;    // histogram adds before the histogram (dim 0, FindBin SIZE_MAX)
    double rejected_pre;
    double pad;
    double atrain[CHILI_MAX_CHANNELS];
};

// Round control written by k_mc_scan / k_mc_finalize, read by the host.
struct RoundCtl {
    long long cut;        // counters consumed by this round
    long long n_acc;      // PreProcess-accepted points before the cut
    long long nan_round;  // of those, NaN retries
    long long pad;
};

constexpr int kPartFixed = 10;  // n, min, max, sum, sum2, nfin, nan, nonfin, wmax, dropped

// libstdc++ lower_bound over cp[0..n) (probe order of bits/stl_algobase.h).
__device__ __forceinline__ int lower_bound_d(const double *__restrict__ a, int n, double v) {
    int first = 0, len = n;
    while (len > 0) {
        const int half = len >> 1;
        const int mid = first + half;
        if (__ldg(a + mid) < v) {
            first = mid + 1;
            len = len - half - 1;
        } else {
            len = half;
        }
    }
    return first;
}

// Random::SelectIndex == std::discrete_distribution (Random.hh:43-45): the
// index of the first cumulative probability not below v.
__device__ __forceinline__ int select_channel(const double *__restrict__ cp, int nch, double v) {
    if (nch < 2) return 0;
    const int i = lower_bound_d(cp, nch, v);
    return i < nch ? i : nch - 1;
}

// Forward grid map with the bin index checked: returns false (x untouched
// beyond the failing dimension) when a uniform is outside [0, 1).
__device__ __forceinline__ bool grid_map_checked(const double *__restrict__ g, int dims, int bins, double *x,
                                                 double &jac) {
    jac = 1.0;
    const double fb = static_cast<double>(bins);
    for (int d = 0; d < dims; ++d) {
        const double pos = __dmul_rn(x[d], fb);
        if (!(pos >= 0.0 && pos < fb)) return false;
        const int idx = static_cast<int>(pos);
        const double loc = __dsub_rn(pos, static_cast<double>(idx));
        const double *e = g + d * (bins + 1);
        const double left = __ldg(e + idx);
        const double size = __dsub_rn(__ldg(e + idx + 1), left);
        x[d] = __dadd_rn(left, __dmul_rn(loc, size));
        jac = __dmul_rn(jac, __dmul_rn(size, fb));
    }
    return true;
}

__device__ __forceinline__ void load_uniforms(uint64_t seed, uint64_t k, const double *__restrict__ u_in,
                                              int n, double *out) {
    if (u_in) {
        for (int j = 0; j < n; ++j) out[j] = __ldg(u_in + k * n + j);
    } else {
        for (int q = 0; 2 * q < n; ++q) {
            double a, b;
            uniform_pair(seed, k, kStreamPoints, static_cast<uint32_t>(q), a, b);
            out[2 * q] = a;
            if (2 * q + 1 < n) out[2 * q + 1] = b;
        }
    }
}

}  // namespace chili_dev
