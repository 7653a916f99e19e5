// grid.cuh -- device form of chili::AdaptiveMap (VEGAS grid).
//
// A grid set holds nch grids of `dims` x (bins+1) edges, each grid in the
// reference layout edges[dim*(bins+1) + k] (AdaptiveMap.hh:29-40), grids back
// to back.  The forward map and the bin search use explicitly rounded
// multiply/add so that x, J and bin indices are bit-identical to the
// reference's (compiled without FMA contraction) for identical inputs.
#pragma once

#include "common.cuh"

namespace chili_dev {

// Table reads: through the read-only path (global tables, NC = true) or
// plain loads (tables staged in shared memory, NC = false).
template <bool NC, class T>
__device__ __forceinline__ T tab_ld(const T *p) {
    if constexpr (NC) return __ldg(p);
    else return *p;
}

// std::lower_bound over edges[0..bins) with libstdc++'s probe sequence, then
// "- 1" as in AdaptiveMap::FindBin (AdaptiveMap.cc:34-38).  Returns -1 where
// the reference returns SIZE_MAX (x <= edges[0] or x NaN).
template <bool NC = true>
__device__ __forceinline__ int find_bin(const double *__restrict__ e, int bins, double x) {
    int first = 0, len = bins;
    while (len > 0) {
        const int half = len >> 1;
        const int mid = first + half;
        if (tab_ld<NC>(e + mid) < x) {
            first = mid + 1;
            len = len - half - 1;
        } else {
            len = half;
        }
    }
    return first - 1;
}

// The 8 bytes before the reference's edge table.  AdaptiveMap::width(0,
// SIZE_MAX) reads m_hist[-1]; under glibc malloc that is the size word of the
// vector's heap chunk: (8*dims*(bins+1) + 8) rounded up to 16, with the
// PREV_INUSE bit set (mmapped chunks, from 128 KiB up, round to pages and set
// IS_MMAPPED).  As a double it is a positive denormal; whether a channel's
// term then overflows to -inf or stays finite depends on its exact value, so
// the host computes it per grid shape (edge_before_table()).
__host__ __device__ inline double edge_before_table(int dims, int bins) {
    const unsigned long long req = 8ull * static_cast<unsigned long long>(dims) * (bins + 1);
    unsigned long long word;
    if (req + 8 >= 128ull * 1024) word = ((req + 16 + 4095) & ~4095ull) | 2ull;
    else {
        word = (req + 8 + 15) & ~15ull;
        word = (word < 32ull ? 32ull : word) | 1ull;
    }
    union {
        unsigned long long u;
        double d;
    } cv;
    cv.u = word;
    return cv.d;
}

// width(dim, bin) of the flat edge table, including the reference's reading
// of bin == SIZE_MAX: lower_edge at flat index dim*(bins+1) - 1 (the previous
// dimension's last edge, or the word before the table for dim 0).
template <bool NC = true>
__device__ __forceinline__ double bin_width(const double *__restrict__ g, int bins, int dim, int bin,
                                            double before) {
    const int base = dim * (bins + 1);
    if (bin >= 0) return __dsub_rn(tab_ld<NC>(g + base + bin + 1), tab_ld<NC>(g + base + bin));
    const double lower = dim > 0 ? tab_ld<NC>(g + base - 1) : before;
    return __dsub_rn(tab_ld<NC>(g + base), lower);
}

// AdaptiveMap::operator() (AdaptiveMap.cc:40-56) on one point: x in place,
// returns the Jacobian.
__device__ __forceinline__ double grid_map(const double *__restrict__ g, int dims, int bins, double *x) {
    double jac = 1.0;
    const double fb = static_cast<double>(bins);
    for (int d = 0; d < dims; ++d) {
        const double pos = __dmul_rn(x[d], fb);
        const int idx = static_cast<int>(pos);
        const double loc = __dsub_rn(pos, static_cast<double>(idx));
        const double *e = g + d * (bins + 1);
        const double left = __ldg(e + idx);
        const double size = __dsub_rn(__ldg(e + idx + 1), left);
        x[d] = __dadd_rn(left, __dmul_rn(loc, size));
        jac = __dmul_rn(jac, __dmul_rn(size, fb));
    }
    return jac;
}

// AdaptiveMap::GenerateWeight (AdaptiveMap.cc:58-65).
__device__ __forceinline__ double grid_weight(const double *__restrict__ g, int dims, int bins,
                                              const double *x, double before) {
    double jac = 1.0;
    const double fb = static_cast<double>(bins);
    for (int d = 0; d < dims; ++d) {
        const int b = find_bin(g + d * (bins + 1), bins, x[d]);
        jac = __dmul_rn(jac, __dmul_rn(bin_width(g, bins, d, b, before), fb));
    }
    return jac;
}

// Flat histogram slot of dimension d's bin b the way Integrand::AddTrainData
// and Vegas::operator() index it (train[d*bins + FindBin]); a FindBin of
// SIZE_MAX wraps to d*bins - 1, which for d == 0 lies before the histogram:
// that slot is reported as -1 (skipped).
__device__ __forceinline__ int train_slot(int d, int bins, int b) {
    const int s = d * bins + b;
    return s;  // b == -1 and d == 0 gives -1
}

// ------------------------------------------------------------ hinted search
// For a monotone edge table the cells of a uniform H-cell grid over [0, 1)
// bracket lower_bound: with cell(v) = clamp((int)(v*H), 0, H) (monotone in v),
// every edge in a cell below x's cell is < x and every edge in a cell above it
// is > x, so lower_bound(x) lies in [hint[c], hint[c+1]) where hint[j] counts
// the edges e[k], k < bins, with cell(e[k]) < j.  hint has H+1 entries per
// (grid, dim); sorted[] marks the tables the shortcut may use (monotone, no
// NaN); other tables and x outside [0, 1) take the plain search.
constexpr int kHintPerBin = 2;

__device__ __forceinline__ int edge_cell(double v, int H) {
    if (!(v > 0.0)) return 0;  // also NaN (excluded by sorted[] anyway)
    const double p = v * static_cast<double>(H);
    return p >= static_cast<double>(H) ? H : static_cast<int>(p);
}

template <bool NC = true>
__device__ __forceinline__ int find_bin_hinted(const double *__restrict__ e, const uint32_t *__restrict__ hint,
                                               bool sorted, int bins, int H, double x) {
    if (!sorted || !(x >= 0.0 && x < 1.0)) return find_bin<NC>(e, bins, x);
    const int c = static_cast<int>(x * static_cast<double>(H));  // < H for x < 1
    const uint32_t hp = tab_ld<NC>(hint + c);  // hint[c] | hint[c+1] << 16
    int first = static_cast<int>(hp & 0xffffu);
    int len = static_cast<int>(hp >> 16) - first;
    while (len > 0) {  // lower_bound inside the bracket
        const int half = len >> 1;
        const int mid = first + half;
        if (tab_ld<NC>(e + mid) < x) {
            first = mid + 1;
            len = len - half - 1;
        } else {
            len = half;
        }
    }
    return first - 1;
}

// The hint table of one (grid, dimension) row of edges e[0..bins], its
// widths w[k] = e[k+1] - e[k] and its monotone flag, built by one block
// (every thread of the block calls this).  hint[j] = first k in [0, bins)
// with cell(e[k]) >= j, packed with hint[j+1] in the upper 16 bits.
__device__ __forceinline__ void build_hint_row(const double *__restrict__ e, int bins, uint32_t *__restrict__ h,
                                               uint8_t *__restrict__ sorted, double *__restrict__ w) {
    const int H = kHintPerBin * bins;
    int bad = 0;
    for (int k = threadIdx.x; k < bins; k += blockDim.x) {
        const double a = e[k];
        if (a != a) bad = 1;
        if (k + 1 < bins && !(a <= e[k + 1])) bad = 1;
        w[k] = __dsub_rn(e[k + 1], a);
    }
    bad = __syncthreads_or(bad);
    if (threadIdx.x == 0) *sorted = bad ? 0 : 1;
    if (bad) return;
    for (int j = threadIdx.x; j < H; j += blockDim.x) {
        int lo[2];
        for (int q = 0; q < 2; ++q) {
            int first = 0, len = bins;
            while (len > 0) {
                const int half = len >> 1, mid = first + half;
                if (edge_cell(e[mid], H) < j + q) {
                    first = mid + 1;
                    len = len - half - 1;
                } else {
                    len = half;
                }
            }
            lo[q] = first;
        }
        h[j] = static_cast<uint32_t>(lo[0]) | (static_cast<uint32_t>(lo[1]) << 16);
    }
}

// width(dim, bin) from the precomputed table wt[dim*bins + bin] (the same
// subtraction as bin_width, done once per grid), the reference's reading of
// bin == SIZE_MAX from the edges.
template <bool NC = true>
__device__ __forceinline__ double bin_width_t(const double *__restrict__ g, const double *__restrict__ wt, int bins,
                                              int dim, int bin, double before) {
    if (bin >= 0) return tab_ld<NC>(wt + dim * bins + bin);
    return bin_width<NC>(g, bins, dim, bin, before);
}

}  // namespace chili_dev
