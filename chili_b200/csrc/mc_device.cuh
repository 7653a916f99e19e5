// mc_device.cuh -- types and device helpers shared by the kernels of
// libchili_b200 (kernels.cuh, pipeline.cuh, flow_phys.cuh): iteration
// accumulator and round records, the channel-selection rule, the checked
// grid map, the counter-based uniforms, the combined channel weight, the
// channel-weight update and the grid adaptation of one dimension.
#pragma once

#include <math_constants.h>

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

// ------------------------------------------------- shared by several kernels
// Integrand::GenerateWeight (Integrand.hh:112-123) for one point.  The
// uniform buffer x is shared by all channels and not cleared between them,
// as the reference's _rans; the chosen channel's copy lands in xs.
__device__ __forceinline__ double combined_weight(const ChannelProgram *__restrict__ progs,
                                                  const double *__restrict__ grids, const double *__restrict__ alpha,
                                                  int nch, int dims, int bins, int ich, V4 *mom, double *x,
                                                  double *xs, double *dens, int dens_stride) {
    for (int d = 0; d < dims; ++d) x[d] = 0.0;
    double acc = 0;
    const size_t gsz = static_cast<size_t>(dims) * (bins + 1);
    const double before = edge_before_table(dims, bins);
    for (int c = 0; c < nch; ++c) {
        const double dc = fs_weight(progs + c, mom, x);
        if (c == ich)
            for (int d = 0; d < dims; ++d) xs[d] = x[d];
        const double vw = grid_weight(grids + c * gsz, dims, bins, x, before);
        acc += __ldg(alpha + c) / dc / vw;
        if (dens) dens[static_cast<size_t>(c) * dens_stride] = dc;
    }
    return 1.0 / acc;
}


__device__ __forceinline__ void alpha_update(double *__restrict__ alpha, double *__restrict__ best, double *__restrict__ min_diff,
                               double *__restrict__ cp, const double *__restrict__ train, int nch, double beta,
                               double min_alpha, int mode) {
    if (mode == 1) {
        double nw[CHILI_MAX_CHANNELS];
        double sum_w = 0;
        for (int i = 0; i < nch; ++i) {
            nw[i] = alpha[i] * pow(train[i], beta);
            sum_w += nw[i];
        }
        double new_sum = 0;
        for (int i = 0; i < nch; ++i) {
            if (nw[i] == 0) continue;
            nw[i] /= sum_w;
            nw[i] = std_max(nw[i], min_alpha);
            new_sum += nw[i];
        }
        for (int i = 0; i < nch; ++i) alpha[i] = nw[i] / new_sum;
        double mx = 0;
        for (int i = 0; i + 1 < nch; ++i)
            for (int j = i + 1; j < nch; ++j) mx = std_max(mx, fabs(train[i] - train[j]));
        if (mx < *min_diff) {
            for (int i = 0; i < nch; ++i) best[i] = alpha[i];
            *min_diff = mx;
        }
    }
    if (nch >= 2) {
        double s = 0;
        for (int i = 0; i < nch; ++i) s += alpha[i];
        double c = 0;
        for (int i = 0; i < nch; ++i) {
            const double p = alpha[i] / s;
            c = (i == 0) ? p : c + p;
            cp[i] = c;
        }
        cp[nch - 1] = 1.0;
    }
}


// AdaptiveMap::Adapt (AdaptiveMap.cc:67-125) of dimension d of grid c by one
// block (WARP false; tmp: bins doubles of shared memory) or by one warp
// (WARP true: the lanes of the calling warp, tmp its own bins doubles).  The
// order-dependent sums and the rebinning run serially in thread (lane) 0 in
// the reference's order; smoothing and the importance factors in parallel.
template <bool WARP>
__device__ __forceinline__ void grid_adapt_impl(const double *__restrict__ g_old, double *__restrict__ g_new, int dims,
                                                int bins, double alpha, const double *__restrict__ train,
                                                int skip_zero, int *__restrict__ status, int d, int c, double *tmp) {
    const int tid = WARP ? static_cast<int>(threadIdx.x & 31) : static_cast<int>(threadIdx.x);
    const int nthr = WARP ? 32 : static_cast<int>(blockDim.x);
    auto sync = [] {
        if (WARP) __syncwarp();
        else __syncthreads();
    };
    const double *T = train + static_cast<size_t>(c) * dims * bins;
    const double *E = g_old + static_cast<size_t>(c) * dims * (bins + 1);
    double *EN = g_new + static_cast<size_t>(c) * dims * (bins + 1);
    const double *Ed = E + d * (bins + 1);
    double *ENd = EN + d * (bins + 1);
    if (skip_zero) {
        int nz = 0;
        for (int k = tid; k < dims * bins; k += nthr) nz |= (T[k] != 0);
        nz = WARP ? __any_sync(0xffffffffu, nz) : __syncthreads_or(nz);
        if (!nz) {
            for (int k = tid; k <= bins; k += nthr) ENd[k] = Ed[k];
            return;
        }
    }
    const double *o = T + d * bins;
    for (int b = tid; b < bins; b += nthr) {
        double s;
        if (b == 0) s = (o[0] + o[1]) / 2;
        else if (b == bins - 1) s = (o[bins - 2] + o[bins - 1]) / 2;
        else s = ((o[b - 1] + o[b]) + o[b + 1]) / 3;
        tmp[b] = s;
    }
    sync();
    double norm = 0;
    if (WARP) {
        if (tid == 0)
            for (int b = 0; b < bins; ++b) norm = (b == 0) ? tmp[0] : norm + tmp[b];
        norm = __shfl_sync(0xffffffffu, norm, 0);
    } else {
        __shared__ double norm_s;
        if (tid == 0) {
            double nm = 0;
            for (int b = 0; b < bins; ++b) nm = (b == 0) ? tmp[0] : nm + tmp[b];
            norm_s = nm;
        }
        __syncthreads();
        norm = norm_s;
    }
    if (norm == 0) {  // the reference leaves this dimension of new_hist at zero
        for (int k = tid; k <= bins; k += nthr) ENd[k] = 0.0;
        return;
    }
    for (int b = tid; b < bins; b += nthr) {
        if (tmp[b] != 0) {
            const double r = tmp[b] / norm;
            tmp[b] = pow((r - 1.0) / log(r), alpha);
        }
    }
    sync();
    if (tid == 0) {
        double avg = 0;
        for (int b = 0; b < bins; ++b) avg += tmp[b];
        avg /= static_cast<double>(bins);
        double cbin = 0;
        int ibin = 0;
        int bad = 0;
        const double nan = CUDART_NAN;
        ENd[0] = 0.0;
        for (int nb = 1; nb < bins; ++nb) {
            while (cbin < avg && ibin < bins) cbin += tmp[ibin++];
            if (cbin < avg) bad = 1;  // the reference would read past the histogram
            const int flat_prev = d * (bins + 1) + ibin - 1;
            const double prev = flat_prev >= 0 ? E[flat_prev] : nan;
            const double curr = Ed[ibin];
            if (ibin == 0) bad = 1;
            cbin -= avg;
            const double delta = (curr - prev) * cbin;
            const double t = ibin > 0 ? tmp[ibin - 1] : nan;
            ENd[nb] = curr - delta / t;
        }
        ENd[bins] = 1.0;
        if (bad) atomicOr(status, 1);
    }
    sync();
}

__device__ __forceinline__ void grid_adapt_block(const double *__restrict__ g_old, double *__restrict__ g_new, int dims,
                                                 int bins, double alpha, const double *__restrict__ train, int skip_zero,
                                                 int *__restrict__ status, int d, int c, double *tmp) {
    grid_adapt_impl<false>(g_old, g_new, dims, bins, alpha, train, skip_zero, status, d, c, tmp);
}

}  // namespace chili_dev
