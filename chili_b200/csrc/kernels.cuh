// kernels.cuh -- the sm_100a kernels of libchili_b200.
//
// Plain VEGAS (Vegas::operator(), src/Integrator/Vegas.cc:18-52) runs as one
// fused kernel: counter-based uniforms -> grid map -> integrand -> StatsData
// partials and the per-bin f^2 J^2 histogram in shared memory.
//
// A multichannel iteration (MultiChannel::operator(),
// include/Channel/MultiChannel.hh:196-251) runs in rounds over contiguous
// counter ranges, so that the retry semantics of the sequential loop (points
// are tried in order until ncalls are accepted) hold exactly:
//   k_mc_forward   uniforms -> channel choice -> VEGAS map -> FSMapper
//                  forward -> PreProcess flag, momenta kept in HBM (SoA)
//   k_mc_scan      accepted counts per block -> exclusive offsets
//   k_mc_compact   ordered list of the PreProcess-accepted points
//   k_mc_weight    every channel's inverse map + grid weight -> combined
//                  weight and integrand, as per-point records
//   k_block_count, k_mc_scan, k_cut_finalize
//                  the cut: the `needed`-th point whose value is not NaN
//                  (NaN values are retried, MultiChannel.hh:230-236)
//   k_mc_accum     StatsData, channel histograms and alpha training over the
//                  records before the cut (block partials)
//   k_mc_reduce, k_mc_accumulate
//                  ordered fold of the partials into the iteration
//                  accumulator; PreProcess rejections count as zero calls
// The chunk is sized from the previous acceptance and NaN rates so that one
// round normally covers the iteration; a short chunk leads to another round.
#pragma once

#include "mc_device.cuh"
#include "phase_dev.cuh"

namespace chili_dev {

// ------------------------------------------------------------- grid kernels
// One block per (dim = blockIdx.x, grid = blockIdx.y): the hint table (as
// pairs hint[j] | hint[j+1] << 16, j < H), the monotone flag and the bin
// widths of that edge table.
__global__ void k_build_hints(const double *__restrict__ grids, int dims, int bins, uint32_t *__restrict__ hints,
                              uint8_t *__restrict__ sorted, double *__restrict__ widths) {
    const int d = blockIdx.x, c = blockIdx.y;
    const size_t row = static_cast<size_t>(c) * dims + d;
    build_hint_row(grids + row * (bins + 1), bins, hints + row * (kHintPerBin * bins), sorted + row,
                   widths + row * bins);
}

__global__ void k_grid_map(const double *__restrict__ g, int dims, int bins, const double *__restrict__ u,
                           double *__restrict__ x, double *__restrict__ jac, long long n) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    double r[CHILI_MAX_DIMS];
    for (int d = 0; d < dims; ++d) r[d] = u[i * dims + d];
    double j;
    if (!grid_map_checked(g, dims, bins, r, j)) {
        for (int d = 0; d < dims; ++d) r[d] = CUDART_NAN;
        j = CUDART_NAN;
    }
    for (int d = 0; d < dims; ++d) x[i * dims + d] = r[d];
    jac[i] = j;
}

// AdaptiveMap::FindBin / GenerateWeight through the hinted search that the
// iteration uses (grid.cuh, find_bin_hinted).
__global__ void k_grid_weight(const double *__restrict__ g, const uint32_t *__restrict__ hints,
                              const uint8_t *__restrict__ sorted, int dims, int bins, const double *__restrict__ x,
                              double *__restrict__ w, int32_t *__restrict__ bin, long long n) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    double jac = 1.0;
    const double fb = static_cast<double>(bins);
    const int H = kHintPerBin * bins;
    for (int d = 0; d < dims; ++d) {
        const int b = find_bin_hinted(g + d * (bins + 1), hints + d * H, sorted[d] != 0, bins, H,
                                      x[i * dims + d]);
        if (bin) bin[i * dims + d] = b;
        jac = __dmul_rn(jac, __dmul_rn(bin_width(g, bins, d, b, edge_before_table(dims, bins)), fb));
    }
    if (w) w[i] = jac;
}

// AdaptiveMap::Adapt (AdaptiveMap.cc:67-125) for grid blockIdx.y, dimension
// blockIdx.x: smoothing and importance factors in parallel over bins, the
// order-dependent sums and the rebinning serially in lane 0, in the
// reference's order.  With skip_zero, grids whose whole histogram is zero
// are copied unchanged (Integrand::Train, Integrand.hh:97-104).
// status bit 1: the rebinning ran past the last bin or before the first.
__global__ void k_grid_adapt(const double *__restrict__ g_old, double *__restrict__ g_new, int dims, int bins,
                             double alpha, const double *__restrict__ train, int skip_zero,
                             int *__restrict__ status) {
    extern __shared__ double tmp[];  // bins
    grid_adapt_block(g_old, g_new, dims, bins, alpha, train, skip_zero, status, blockIdx.x, blockIdx.y, tmp);
}

// AdaptiveMap::Split (AdaptiveMap.cc:127-160) of every grid.
__global__ void k_grid_split(const double *__restrict__ g_old, double *__restrict__ g_new, int ngrids, int dims,
                             int bins, int nsplit) {
    const long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    const long long total = static_cast<long long>(ngrids) * dims * bins;
    if (t >= total) return;
    const int bin = static_cast<int>(t % bins);
    const long long gd = t / bins;  // grid*dims + dim
    const int nb = nsplit * bins;
    const double *e = g_old + gd * (bins + 1);
    double *en = g_new + gd * (nb + 1);
    const double curr = e[bin];
    const double size = __dsub_rn(e[bin + 1], curr);
    for (int i = 0; i < nsplit; ++i)
        en[bin * nsplit + i] = __dadd_rn(curr, __ddiv_rn(__dmul_rn(static_cast<double>(i), size),
                                                          static_cast<double>(nsplit)));
    if (bin == bins - 1) en[nb] = 1.0;
}

// ------------------------------------------------------------- plain VEGAS
// One Vegas::operator() over n points (grid-stride).  Histogram in shared
// memory when it fits (smem_hist), else global atomics into hist.
// DIMS > 0: the dimension fixed at compile time (coordinates in registers);
// DIMS == 0: `dims` at run time (a local array).
template <int DIMS>
__device__ __forceinline__ void vegas_points(const double *__restrict__ g, int dims_rt, int bins, uint64_t seed,
                                             uint64_t ctr0, const double *__restrict__ u_in, long long n,
                                             const IntegrandDesc *__restrict__ f, double *__restrict__ part,
                                             double *__restrict__ hist, int smem_hist) {
    extern __shared__ double sh[];
    const int dims = DIMS > 0 ? DIMS : dims_rt;
    const int nh = dims * bins;
    if (smem_hist)
        for (int k = threadIdx.x; k < nh; k += blockDim.x) sh[k] = 0.0;
    __syncthreads();
    double* H = smem_hist ? sh : hist;
    double cnt = 0, sum = 0, sum2 = 0, mn = 1.7976931348623157e308, mx = 2.2250738585072014e-308, nf = 0;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        double r[DIMS > 0 ? DIMS : CHILI_MAX_DIMS];
        if (u_in) {
#pragma unroll
            for (int d = 0; d < dims; ++d) r[d] = __ldg(u_in + i * dims + d);
        } else {
            load_uniforms(seed, ctr0 + i, nullptr, dims, r);
        }
        double jac;
        double val;
        if (grid_map_checked(g, dims, bins, r, jac)) val = camel(f, r, dims) * jac;
        else val = CUDART_NAN;
        const double val2 = val * val;
        cnt += 1;
        sum += val;
        sum2 += val * val;
        mn = std_min(mn, val);
        mx = std_max(mx, val);
        nf += (val != 0);
#pragma unroll
        for (int j = 0; j < dims; ++j) {
            const int b = find_bin(g + j * (bins + 1), bins, r[j]);
            const int s = j * bins + b;
            if (s >= 0) atomicAdd(H + s, val2);
        }
    }
    cnt = warp_sum(cnt);
    sum = warp_sum(sum);
    sum2 = warp_sum(sum2);
    mn = warp_min(mn);
    mx = warp_max(mx);
    nf = warp_sum(nf);
    __shared__ double ws[32][6];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        ws[w][0] = cnt; ws[w][1] = mn; ws[w][2] = mx; ws[w][3] = sum; ws[w][4] = sum2; ws[w][5] = nf;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a[6] = {ws[0][0], ws[0][1], ws[0][2], ws[0][3], ws[0][4], ws[0][5]};
        for (int k = 1; k < (blockDim.x >> 5); ++k) {
            a[0] += ws[k][0]; a[1] = std_min(a[1], ws[k][1]); a[2] = std_max(a[2], ws[k][2]);
            a[3] += ws[k][3]; a[4] += ws[k][4]; a[5] += ws[k][5];
        }
        for (int k = 0; k < 6; ++k) part[blockIdx.x * 6 + k] = a[k];
    }
    if (smem_hist) {
        double *dst = hist + static_cast<size_t>(blockIdx.x) * nh;
        for (int k = threadIdx.x; k < nh; k += blockDim.x) dst[k] = sh[k];
    }
}

template <int DIMS>
__global__ void k_vegas_iter(const double *__restrict__ g, int dims_rt, int bins, uint64_t seed, uint64_t ctr0,
                             const double *__restrict__ u_in, long long n, const IntegrandDesc *__restrict__ f,
                             double *__restrict__ part, double *__restrict__ hist, int smem_hist) {
    vegas_points<DIMS>(g, dims_rt, bins, seed, ctr0, u_in, n, f, part, hist, smem_hist);
}

// Materialised VEGAS points on the camel: point i's uniforms (the counter
// stream of k_vegas_iter, ctr0 + i) through the grid, x_out[i][dims] and the
// point's weight f(x) J(u) to w_out[i].  The grid (dims x (bins+1) edges) is
// staged in shared memory; a block's points are assembled in shared memory
// and leave as contiguous 16-byte stores, so the only HBM traffic is the
// 8 (dims + 1) bytes written per point.  Persistent grid-stride over tiles
// of kGenTile points.
// DIMS > 0 fixes the dimension at compile time (the point's coordinates stay
// in registers); DIMS == 0 takes `dims` at run time (a local array).  PPT
// points per thread (independent dependency chains the scheduler overlaps):
// a tile is kGenTile * PPT points.
constexpr int kGenTile = 256;
template <int DIMS, int PPT>
__global__ void __launch_bounds__(kGenTile) k_vegas_generate(const double *__restrict__ g, int dims_rt, int bins,
                                                             uint64_t seed, uint64_t ctr0, long long n,
                                                             const IntegrandDesc *__restrict__ f,
                                                             double *__restrict__ x_out, double *__restrict__ w_out) {
    extern __shared__ __align__(16) double gsh[];
    constexpr int kTile = kGenTile * PPT;
    const int dims = DIMS > 0 ? DIMS : dims_rt;
    const int ne = dims * (bins + 1);
    double *xt = gsh + ((ne + 1) & ~1);  // kTile * dims x values, 16-byte aligned
    double *wt = xt + kTile * dims;      // kTile weights
    for (int k = threadIdx.x; k < ne; k += blockDim.x) gsh[k] = g[k];
    __syncthreads();
    const double fb = static_cast<double>(bins);
    const long long ntiles = (n + kTile - 1) / kTile;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const long long i0 = t * kTile;
        const int cnt = static_cast<int>(n - i0 < kTile ? n - i0 : kTile);
#pragma unroll
        for (int q = 0; q < PPT; ++q) {
            const int l = q * kGenTile + threadIdx.x;  // point of the tile
            if (l < cnt) {
                double r[DIMS > 0 ? DIMS : CHILI_MAX_DIMS];
                load_uniforms(seed, ctr0 + i0 + l, nullptr, dims, r);
                // AdaptiveMap::operator() (AdaptiveMap.cc:40-56) on the staged
                // edges, rounded as grid_map_checked
                double jac = 1.0;
                bool ok = true;
#pragma unroll
                for (int d = 0; d < dims; ++d) {
                    const double pos = __dmul_rn(r[d], fb);
                    if (!(pos >= 0.0 && pos < fb)) {
                        ok = false;
                        break;
                    }
                    const int idx = static_cast<int>(pos);
                    const double loc = __dsub_rn(pos, static_cast<double>(idx));
                    const double *e = gsh + d * (bins + 1);
                    const double left = e[idx];
                    const double size = __dsub_rn(e[idx + 1], left);
                    r[d] = __dadd_rn(left, __dmul_rn(loc, size));
                    jac = __dmul_rn(jac, __dmul_rn(size, fb));
                }
                const double w = ok ? camel(f, r, dims) * jac : CUDART_NAN;
#pragma unroll
                for (int d = 0; d < dims; ++d) xt[l * dims + d] = ok ? r[d] : CUDART_NAN;
                wt[l] = w;
            }
        }
        __syncthreads();
        // the tile's rows are contiguous in x_out: cnt * dims doubles from
        // i0 * dims, written as double2 where both ends allow it
        double *xo = x_out + i0 * dims;
        const int nx = cnt * dims;
        const bool vec = ((reinterpret_cast<uintptr_t>(xo) & 15) == 0) && ((nx & 1) == 0);
        if (vec) {
            const double2 *src = reinterpret_cast<const double2 *>(xt);
            double2 *dst = reinterpret_cast<double2 *>(xo);
            for (int k = threadIdx.x; k < (nx >> 1); k += blockDim.x) dst[k] = src[k];
        } else {
            for (int k = threadIdx.x; k < nx; k += blockDim.x) xo[k] = xt[k];
        }
        for (int k = threadIdx.x; k < cnt; k += blockDim.x) w_out[i0 + k] = wt[k];
        __syncthreads();
    }
}

// Ordered fold of k_vegas_iter's partials: stats into out6, histogram
// partials (when per block) into train[dims*bins].  The partials are read
// from L2 (__ldcg): in k_vegas_step other blocks of the same launch wrote
// them.
__device__ __forceinline__ void vegas_fold(const double *part, int nblocks, const double *hist_part,
                                           int per_block_hist, int nh, double *__restrict__ train,
                                           double *__restrict__ out6) {
    if (per_block_hist) {
        for (int k = threadIdx.x; k < nh; k += blockDim.x) {
            double s = 0;
            for (int b = 0; b < nblocks; ++b) s += __ldcg(hist_part + static_cast<size_t>(b) * nh + k);
            train[k] = s;
        }
    }
    if (threadIdx.x == 0) {
        double n = 0, mn = 1.7976931348623157e308, mx = 2.2250738585072014e-308, sum = 0, csum = 0, sum2 = 0,
               csum2 = 0, nf = 0;
        for (int b = 0; b < nblocks; ++b) {
            const double *p = part + b * 6;
            n += __ldcg(p);
            mn = std_min(mn, __ldcg(p + 1));
            mx = std_max(mx, __ldcg(p + 2));
            double y = __ldcg(p + 3) - csum, t = sum + y;  // Kahan
            csum = (t - sum) - y;
            sum = t;
            y = __ldcg(p + 4) - csum2;
            t = sum2 + y;
            csum2 = (t - sum2) - y;
            sum2 = t;
            nf += __ldcg(p + 5);
        }
        out6[0] = n; out6[1] = mn; out6[2] = mx; out6[3] = sum; out6[4] = sum2; out6[5] = nf;
    }
}

__global__ void k_vegas_finalize(const double *__restrict__ part, int nblocks, const double *__restrict__ hist_part,
                                 int per_block_hist, int nh, double *__restrict__ train, double *__restrict__ out6) {
    vegas_fold(part, nblocks, hist_part, per_block_hist, nh, train, out6);
}

// Ordered fold of the partials of blocks [b0, b1) (StatsData with Kahan sums,
// histogram bin by bin) into one partial: out6 and out_hist[nh].  The
// partials were written by other blocks of the same launch: read from L2.
__device__ __forceinline__ void vegas_fold_range(const double *part, const double *hist_part, int b0, int b1, int nh,
                                                 double *__restrict__ out_hist, double *__restrict__ out6) {
    for (int k = threadIdx.x; k < nh; k += blockDim.x) {
        double s = 0;
        for (int b = b0; b < b1; ++b) s += __ldcg(hist_part + static_cast<size_t>(b) * nh + k);
        out_hist[k] = s;
    }
    if (threadIdx.x == 0) {
        double n = 0, mn = 1.7976931348623157e308, mx = 2.2250738585072014e-308, sum = 0, csum = 0, sum2 = 0,
               csum2 = 0, nf = 0;
        for (int b = b0; b < b1; ++b) {
            const double *p = part + b * 6;
            n += __ldcg(p);
            mn = std_min(mn, __ldcg(p + 1));
            mx = std_max(mx, __ldcg(p + 2));
            double y = __ldcg(p + 3) - csum, t = sum + y;  // Kahan
            csum = (t - sum) - y;
            sum = t;
            y = __ldcg(p + 4) - csum2;
            t = sum2 + y;
            csum2 = (t - sum2) - y;
            sum2 = t;
            nf += __ldcg(p + 5);
        }
        out6[0] = n; out6[1] = mn; out6[2] = mx; out6[3] = sum; out6[4] = sum2; out6[5] = nf;
    }
}

// One whole Vegas::operator() (Vegas.cc:18-52) in one launch: the points of
// k_vegas_iter (histogram in shared memory, one partial per block); then,
// per group of kStepGroup consecutive blocks, the last of them to finish
// folds the group's partials in block order into a group partial; the last
// group to be folded folds the group partials in group order, writes the
// StatsData to out6 and the histogram to train, and runs
// AdaptiveMap::Adapt (AdaptiveMap.cc:67-125) dimension by dimension from g
// into g_new.  Arrival counters (arrive[0] for the groups, arrive[1 + group]
// within a group) are zero between launches and reset by the block that
// completes them; no block waits for another.  The fixed grouping keeps the
// sums deterministic.
constexpr int kStepGroup = 16;
template <int DIMS>
__global__ void k_vegas_step(const double *__restrict__ g, double *__restrict__ g_new, int dims_rt, int bins,
                             uint64_t seed, uint64_t ctr0, const double *__restrict__ u_in, long long n,
                             const IntegrandDesc *__restrict__ f, double *part, double *hist_part, double *gpart,
                             double *ghist, double *__restrict__ train, double *__restrict__ out6, double alpha,
                             int adapt, unsigned *__restrict__ arrive, int *__restrict__ status) {
    extern __shared__ double sh[];
    vegas_points<DIMS>(g, dims_rt, bins, seed, ctr0, u_in, n, f, part, hist_part, 1);
    const int dims = DIMS > 0 ? DIMS : dims_rt;
    const int nh = dims * bins;
    const int grp = blockIdx.x / kStepGroup, ngrp = (gridDim.x + kStepGroup - 1) / kStepGroup;
    const int b0 = grp * kStepGroup, b1 = min(b0 + kStepGroup, static_cast<int>(gridDim.x));
    __shared__ bool last;
    __threadfence();  // this block's partials visible before its arrival
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(arrive + 1 + grp, 1u) == static_cast<unsigned>(b1 - b0 - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    vegas_fold_range(part, hist_part, b0, b1, nh, ghist + static_cast<size_t>(grp) * nh, gpart + grp * 6);
    if (threadIdx.x == 0) arrive[1 + grp] = 0u;
    __threadfence();  // the group partial visible before the group's arrival
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(arrive, 1u) == static_cast<unsigned>(ngrp - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    vegas_fold_range(gpart, ghist, 0, ngrp, nh, train, out6);
    __syncthreads();  // train complete (and the points' shared histogram no longer needed)
    if (adapt) {
        // one warp per dimension (each with its own bins doubles of shared
        // memory), the dimensions in rounds of the block's warps
        if (threadIdx.x == 0) *status = 0;
        __syncthreads();
        const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
        for (int d = w; d < dims; d += nw) grid_adapt_impl<true>(g, g_new, dims, bins, alpha, train, 0, status, d, 0,
                                                                 sh + static_cast<size_t>(w) * bins);
    }
    if (threadIdx.x == 0) *arrive = 0u;
}

// ------------------------------------------------------------- channels
__global__ void k_fs_generate(const ChannelProgram *__restrict__ prog, const double *__restrict__ x,
                              double *__restrict__ mom, long long n) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const int nd = prog->ndims, ne = prog->n_ext;
    double r[CHILI_MAX_DIMS];
    for (int d = 0; d < nd; ++d) r[d] = x[i * nd + d];
    V4 m[CHILI_MAX_SLOTS];
    double m2[CHILI_MAX_SLOTS];
    fs_generate(prog, r, m, m2);
    for (int k = 0; k < ne; ++k) {
        double *o = mom + (i * ne + k) * 4;
        o[0] = m[k].e; o[1] = m[k].x; o[2] = m[k].y; o[3] = m[k].z;
    }
}

// x_out is also read first when x_in != 0: the uniform buffer then starts
// from the caller's contents (FSMapper::GenerateWeight writes only the
// entries its chain consumes, Channel.cc:40-61), else from zeros.
__global__ void k_fs_weight(const ChannelProgram *__restrict__ prog, const double *__restrict__ mom,
                            double *x_out, double *__restrict__ w, long long n, int x_in) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const int nd = prog->ndims, ne = prog->n_ext;
    V4 m[CHILI_MAX_SLOTS];
    for (int k = 0; k < ne; ++k) {
        const double *q = mom + (i * ne + k) * 4;
        m[k] = V4{q[0], q[1], q[2], q[3]};
    }
    double r[CHILI_MAX_DIMS];
    for (int d = 0; d < nd; ++d) r[d] = x_in ? x_out[i * nd + d] : 0.0;
    const double wt = fs_weight(prog, m, r);
    w[i] = wt;
    if (x_out)
        for (int d = 0; d < nd; ++d) x_out[i * nd + d] = r[d];
}

__global__ void k_select(const double *__restrict__ cp, int nch, const double *__restrict__ v,
                         int32_t *__restrict__ out, long long n) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    out[i] = select_channel(cp, nch, v[i]);
}

__global__ void k_mc_weight_batch(const ChannelProgram *__restrict__ progs, const double *__restrict__ grids,
                                  const double *__restrict__ alpha, int nch, int dims, int bins, int n_ext,
                                  const double *__restrict__ mom, const int32_t *__restrict__ ich,
                                  double *__restrict__ wgt, double *__restrict__ dens, double *__restrict__ x_ich,
                                  long long n, const PointProgram *__restrict__ pp) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    V4 m[CHILI_MAX_SLOTS];
    for (int k = 0; k < n_ext; ++k) {
        const double *q = mom + (i * n_ext + k) * 4;
        m[k] = V4{q[0], q[1], q[2], q[3]};
    }
    double x[CHILI_MAX_DIMS], xs[CHILI_MAX_DIMS];
    for (int d = 0; d < dims; ++d) xs[d] = 0.0;
    const int c = ich[i];
    const int cs = (c >= 0 && c < nch) ? c : -1;
    const double w = pp ? combined_weight_pp(pp, grids, alpha, dims, bins, cs, m, x, xs,
                                             dens ? dens + i * nch : nullptr, 1, edge_before_table(dims, bins))
                        : combined_weight(progs, grids, alpha, nch, dims, bins, cs, m, x, xs,
                                          dens ? dens + i * nch : nullptr, 1);
    wgt[i] = w;
    if (x_ich)
        for (int d = 0; d < dims; ++d) x_ich[i * dims + d] = xs[d];
}

// ------------------------------------------------------------- multichannel
__global__ void __launch_bounds__(kFwdBlock) k_mc_forward(
    const ChannelProgram *__restrict__ progs, const double *__restrict__ grids, const double *__restrict__ cp,
    int nch, int dims, int bins, uint64_t seed, uint64_t ctr0, const double *__restrict__ u_in, long long m,
    const IntegrandDesc *__restrict__ f, int n_ext, double *__restrict__ mom_soa, int32_t *__restrict__ ich_out,
    uint8_t *__restrict__ flag, int32_t *__restrict__ block_count, const long long *__restrict__ gate) {
    // gate (queued rounds): the count still needed; nothing to do once it is 0
    if (gate && *gate <= 0) {
        if (threadIdx.x == 0) block_count[blockIdx.x] = 0;
        return;
    }
    const long long k = blockIdx.x * static_cast<long long>(kFwdBlock) + threadIdx.x;
    int acc = 0;
    if (k < m) {
        double r[CHILI_MAX_DIMS + 1];
        if (u_in) {
            for (int j = 0; j <= dims; ++j) r[j] = __ldg(u_in + k * (dims + 1) + j);
        } else {
            load_uniforms(seed, ctr0 + k, nullptr, dims + 1, r);
        }
        const int c = select_channel(cp, nch, r[dims]);
        const double *g = grids + static_cast<size_t>(c) * dims * (bins + 1);
        double jac;
        V4 mom[CHILI_MAX_SLOTS];
        double m2[CHILI_MAX_SLOTS];
        if (grid_map_checked(g, dims, bins, r, jac)) {
            fs_generate(progs + c, r, mom, m2);
        } else {
            for (int s = 0; s < n_ext; ++s) mom[s] = V4{CUDART_NAN, CUDART_NAN, CUDART_NAN, CUDART_NAN};
        }
        acc = preprocess(f, mom) ? 1 : 0;
        if (acc) {
            for (int s = 0; s < n_ext; ++s) {
                mom_soa[(4 * s + 0) * m + k] = mom[s].e;
                mom_soa[(4 * s + 1) * m + k] = mom[s].x;
                mom_soa[(4 * s + 2) * m + k] = mom[s].y;
                mom_soa[(4 * s + 3) * m + k] = mom[s].z;
            }
        }
        ich_out[k] = c;
        flag[k] = static_cast<uint8_t>(acc);
    }
    const int cnt = __syncthreads_count(acc);
    if (threadIdx.x == 0) block_count[blockIdx.x] = cnt;
}

// One block of 1024 threads: exclusive scan of the per-block accepted counts
// and the cut at the `needed`-th accepted point.  remaining (queued rounds,
// may be NULL): the device's count still needed; when it is 0 the round is
// empty (cut 0, nothing accepted), and with cut_at_remaining it replaces
// `needed`.

__global__ void __launch_bounds__(1024) k_mc_scan(const int32_t *__restrict__ block_count, int nb,
                                                  const uint8_t *__restrict__ flag, long long m, long long needed,
                                                  const long long *__restrict__ remaining, int cut_at_remaining,
                                                  long long *__restrict__ block_off, RoundCtl *__restrict__ ctl) {
    mc_scan_body(block_count, nb, flag, m, needed, remaining, cut_at_remaining, block_off, ctl);
}


__global__ void __launch_bounds__(kFwdBlock) k_mc_compact(const uint8_t *__restrict__ flag,
                                                          const long long *__restrict__ block_off,
                                                          const RoundCtl *__restrict__ ctl, long long m,
                                                          int32_t *__restrict__ list) {
    mc_compact_block(flag, block_off, ctl, m, list, blockIdx.x);
}

// The expensive pass: combined weight and integrand of every PreProcess-
// accepted point list[0..n) of the chunk, written as per-point records so
// that the exact cut (the `needed`-th point whose value is not NaN, in
// counter order) can be taken afterwards and only that prefix accumulated:
//   rec_val, rec_wgt   value f*w and weight (both 0 for a NaN retry)
//   rec_ok             0 for a NaN retry (MultiChannel.hh:230-236), else 1
//   rec_slot[j*n+i]    histogram slot of dimension j in the chosen channel's
//                      histogram (Integrand.hh:91-95), -1 when it would lie
//                      before the histogram
//   rec_dens[c*n+i]    channel c's density, for the alpha-training terms
__global__ void __launch_bounds__(kWgtBlock) k_mc_weight(
    const ChannelProgram *__restrict__ progs, const double *__restrict__ grids, const double *__restrict__ alpha,
    int nch, int dims, int bins, int n_ext, const double *__restrict__ mom_soa, long long m,
    const int32_t *__restrict__ ich_arr, const int32_t *__restrict__ list, const RoundCtl *__restrict__ ctl,
    const IntegrandDesc *__restrict__ f, int should_opt, double *__restrict__ rec_val, double *__restrict__ rec_wgt,
    uint8_t *__restrict__ rec_ok, int32_t *__restrict__ rec_slot, double *__restrict__ rec_dens,
    const PointProgram *__restrict__ pp) {
    // records are laid out with stride m (the chunk size, known on the host);
    // only the first ctl->n_acc entries are written
    const long long n = ctl->n_acc;
    const long long i = blockIdx.x * static_cast<long long>(kWgtBlock) + threadIdx.x;
    if (i >= n || i >= m) return;
    const long long k = list[i];
    const int c_sel = ich_arr[k];
    V4 mom[CHILI_MAX_SLOTS];
    for (int s = 0; s < n_ext; ++s)
        mom[s] = V4{mom_soa[(4 * s + 0) * m + k], mom_soa[(4 * s + 1) * m + k], mom_soa[(4 * s + 2) * m + k],
                    mom_soa[(4 * s + 3) * m + k]};
    double x[CHILI_MAX_DIMS], xs[CHILI_MAX_DIMS];
    const int stride = static_cast<int>(m);
    double wgt = pp ? combined_weight_pp(pp, grids, alpha, dims, bins, c_sel, mom, x, xs, rec_dens + i, stride,
                                         edge_before_table(dims, bins))
                    : combined_weight(progs, grids, alpha, nch, dims, bins, c_sel, mom, x, xs, rec_dens + i, stride);
    const double fv = eval_momenta(f, mom, n_ext);
    double val = wgt == 0 ? 0 : fv * wgt;
    uint8_t ok = 1;
    if (isnan(val)) {
        val = wgt = 0;
        ok = 0;
    }
    rec_val[i] = val;
    rec_wgt[i] = wgt;
    rec_ok[i] = ok;
    if (should_opt) {
        const double *g = grids + static_cast<size_t>(c_sel) * dims * (bins + 1);
        const int base = c_sel * dims * bins;
        for (int j = 0; j < dims; ++j) {
            const int b = find_bin(g + j * (bins + 1), bins, xs[j]);
            const int s = j * bins + b;
            rec_slot[j * m + i] = s >= 0 ? base + s : -1;
        }
    }
}

// Per-256-entry counts of a byte flag array (input of k_mc_scan).
__global__ void __launch_bounds__(kFwdBlock) k_block_count(const uint8_t *__restrict__ flag,
                                                           const RoundCtl *__restrict__ ctl,
                                                           int32_t *__restrict__ block_count) {
    const long long n = ctl->n_acc;
    const long long k = blockIdx.x * static_cast<long long>(kFwdBlock) + threadIdx.x;
    const int cnt = __syncthreads_count(k < n ? flag[k] : 0);
    if (threadIdx.x == 0) block_count[blockIdx.x] = cnt;
}

// Turns the cut over the record list (ctl_list: cut = records included,
// n_acc = non-NaN among them) into the round record: counters consumed,
// PreProcess-accepted points among them, NaN retries among those.
// iter (queued rounds, may be NULL; k_iter_init): the count still needed
// replaces `needed` and is brought down by this round, which also adds to
// the chunk's totals; a round queued after the count reached 0 is empty.
__global__ void k_cut_finalize(const RoundCtl *__restrict__ ctl_list, const RoundCtl *__restrict__ ctl_pre,
                               const int32_t *__restrict__ list, long long m, long long needed,
                               long long *__restrict__ iter, RoundCtl *__restrict__ ctl) {
    if (iter) {
        needed = iter[0];
        if (needed <= 0) {
            *ctl = RoundCtl{0, 0, 0, 0};
            return;
        }
    }
    const long long n_pre = ctl_pre->n_acc;
    const long long ok = n_pre > 0 ? ctl_list->n_acc : 0;
    const bool enough = ok >= needed;
    const long long L = enough ? ctl_list->cut : n_pre;  // records included
    RoundCtl r;
    r.cut = (enough && L > 0) ? static_cast<long long>(list[L - 1]) + 1 : m;
    r.n_acc = L;
    r.nan_round = L - ok;
    r.pad = 0;
    *ctl = r;
    if (iter) {
        iter[0] = needed - (r.n_acc - r.nan_round);
        iter[1] += r.cut;
        iter[2] += r.n_acc;
        iter[3] += r.nan_round;
        iter[4] += n_pre;
    }
}

// Queued rounds' state: the count still needed, then the totals of counters
// consumed, PreProcess-accepted points, NaN retries and weighted points.
constexpr int kIterCtl = 5;
__global__ void k_iter_init(long long *__restrict__ iter, long long needed) {
    iter[0] = needed;
    for (int j = 1; j < kIterCtl; ++j) iter[j] = 0;
}

// Ordered-prefix accumulation of the records [0, ctl->n_acc): StatsData
// partials, histogram adds (hist non-null; else k_mc_hist does them; the
// out-of-range slots are counted here either way), alpha-training terms
// val^2 w / dens_j (MultiChannel.hh:167-180).  Dynamic shared memory:
// (kWgtBlock/32) * nch.
__global__ void __launch_bounds__(kWgtBlock) k_mc_accum(
    const RoundCtl *__restrict__ ctl, long long n_rec, int nch, int dims, int hist_size,
    const double *__restrict__ rec_val,
    const double *__restrict__ rec_wgt, const uint8_t *__restrict__ rec_ok, const int32_t *__restrict__ rec_slot,
    const double *__restrict__ rec_dens, int should_opt, int guard, double *__restrict__ hist,
    double *__restrict__ part) {
    extern __shared__ double atr_s[];  // (kWgtBlock/32) * nch
    const long long n_list = ctl->n_acc;
    const long long i = blockIdx.x * static_cast<long long>(kWgtBlock) + threadIdx.x;
    const bool active = i < n_list && i < n_rec;
    const double val = active ? rec_val[i] : 0.0;
    const double wgt = active ? rec_wgt[i] : 0.0;
    double cnt = active ? 1.0 : 0.0;
    double nan_cnt = (active && !rec_ok[i]) ? 1.0 : 0.0;
    double dropped = 0;
    const double val2 = val * val;
    if (active && should_opt) {
        for (int j = 0; j < dims; ++j) {
            const int s = rec_slot[j * n_rec + i];
            if (s >= 0 && s < hist_size) {
                if (hist) atomicAdd(hist + s, val2);
            } else {
                dropped += 1;
            }
        }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double nonfin = 0;
    if (should_opt) {
        for (int j = 0; j < nch; ++j) {
            double term = active ? val2 * wgt / rec_dens[j * n_rec + i] : 0.0;
            if (guard && !isfinite(term)) {
                nonfin += 1;
                term = 0.0;
            }
            term = warp_sum(term);
            if (lane == 0) atr_s[w * nch + j] = term;
        }
    }
    double sum = warp_sum(val), sum2 = warp_sum(val * val);
    double mn = warp_min(active ? val : 1.7976931348623157e308);
    double mx = warp_max(active ? val : 2.2250738585072014e-308);
    cnt = warp_sum(cnt);
    double nf = warp_sum((active && val != 0) ? 1.0 : 0.0);
    nan_cnt = warp_sum(nan_cnt);
    nonfin = warp_sum(nonfin);
    dropped = warp_sum(dropped);
    double wm = warp_max(active ? val : 0.0);
    __shared__ double ws[kWgtBlock / 32][kPartFixed];
    if (lane == 0) {
        ws[w][0] = cnt; ws[w][1] = mn; ws[w][2] = mx; ws[w][3] = sum; ws[w][4] = sum2;
        ws[w][5] = nf; ws[w][6] = nan_cnt; ws[w][7] = nonfin; ws[w][8] = wm; ws[w][9] = dropped;
    }
    __syncthreads();
    const int stride = kPartFixed + nch;
    double *P = part + static_cast<size_t>(blockIdx.x) * stride;
    if (threadIdx.x == 0) {
        double a[kPartFixed];
        for (int q = 0; q < kPartFixed; ++q) a[q] = ws[0][q];
        for (int v = 1; v < kWgtBlock / 32; ++v) {
            a[0] += ws[v][0]; a[1] = std_min(a[1], ws[v][1]); a[2] = std_max(a[2], ws[v][2]);
            a[3] += ws[v][3]; a[4] += ws[v][4]; a[5] += ws[v][5]; a[6] += ws[v][6]; a[7] += ws[v][7];
            a[8] = std_max(a[8], ws[v][8]); a[9] += ws[v][9];
        }
        for (int q = 0; q < kPartFixed; ++q) P[q] = a[q];
    }
    if (should_opt) {
        for (int j = threadIdx.x; j < nch; j += kWgtBlock) {
            double s = 0;
            for (int v = 0; v < kWgtBlock / 32; ++v) s += atr_s[v * nch + j];
            P[kPartFixed + j] = s;
        }
    }
}

// The histogram adds of the records [0, ctl->n_acc) (val^2 into the bin of
// each dimension of the record's channel, MultiChannel.hh:167-180), staged
// in shared memory: every block sums its records' adds into a private copy
// of the whole histogram (hist_size doubles of dynamic shared memory) with
// shared-memory atomics, then adds its nonzero bins to the global histogram
// -- one global atomic per (block, bin) instead of one per (record, dim).
// The bins' sums agree with k_mc_accum's direct adds up to the order of
// addition.
__global__ void __launch_bounds__(1024) k_mc_hist(const RoundCtl *__restrict__ ctl, long long n_rec, int dims,
                                                  int hist_size, const double *__restrict__ rec_val,
                                                  const int32_t *__restrict__ rec_slot, double *__restrict__ hist) {
    extern __shared__ double sh[];
    for (int k = threadIdx.x; k < hist_size; k += blockDim.x) sh[k] = 0.0;
    __syncthreads();
    const long long n = ctl->n_acc < n_rec ? ctl->n_acc : n_rec;
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n; i += stride) {
        const double v = rec_val[i];
        const double v2 = v * v;
        for (int j = 0; j < dims; ++j) {
            const int s = rec_slot[j * n_rec + i];
            if (s >= 0 && s < hist_size) atomicAdd(sh + s, v2);
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < hist_size; k += blockDim.x) {
        const double v = sh[k];
        if (v != 0.0) atomicAdd(hist + k, v);
    }
}

// Ordered tree fold of k_mc_weight's partials: block f reduces field f
// (kPartFixed statistics fields, then one alpha-training sum per channel)
// over the round's blocks into round_res[f].
__global__ void __launch_bounds__(256) k_mc_reduce(const double *__restrict__ part, int nch,
                                                   const RoundCtl *__restrict__ ctl, double *__restrict__ round_res) {
    const long long n_list = ctl->n_acc;
    const long long nb = (n_list + kWgtBlock - 1) / kWgtBlock;
    const int stride = kPartFixed + nch;
    const int fld = blockIdx.x;
    // 0 sum-like, 1 min, 2 max
    const int op = (fld == 1) ? 1 : ((fld == 2 || fld == 8) ? 2 : 0);
    const double ident = op == 1 ? 1.7976931348623157e308 : (op == 2 ? (fld == 2 ? 2.2250738585072014e-308 : 0.0) : 0.0);
    double v = ident;
    for (long long b = threadIdx.x; b < nb; b += blockDim.x) {
        const double p = part[b * stride + fld];
        v = op == 0 ? v + p : (op == 1 ? std_min(v, p) : std_max(v, p));
    }
    __shared__ double red[256];
    red[threadIdx.x] = v;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            const double a = red[threadIdx.x], c = red[threadIdx.x + s];
            red[threadIdx.x] = op == 0 ? a + c : (op == 1 ? std_min(a, c) : std_max(a, c));
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) round_res[fld] = red[0];
}

// Merge one round into the iteration accumulator; PreProcess rejections
// before the cut count as zero-valued calls (MultiChannel.hh:219-223).
__global__ void k_mc_accumulate(const double *__restrict__ round_res, int nch, RoundCtl *__restrict__ ctl,
                                IterAcc *__restrict__ acc) {
    for (int j = threadIdx.x; j < nch; j += blockDim.x) acc->atrain[j] += round_res[kPartFixed + j];
    if (threadIdx.x != 0) return;
    const long long rej = ctl->cut - ctl->n_acc;
    double mn = std_min(acc->st[1], round_res[1]);
    double mx = std_max(acc->st[2], round_res[2]);
    if (rej > 0) {
        mn = std_min(mn, 0.0);
        mx = std_max(mx, 0.0);
    }
    acc->st[0] += round_res[0] + static_cast<double>(rej);
    acc->st[1] = mn;
    acc->st[2] = mx;
    acc->st[3] += round_res[3];
    acc->st[4] += round_res[4];
    acc->st[5] += round_res[5];
    acc->nan_count += round_res[6];
    acc->nonfinite += round_res[7];
    acc->wmax = std_max(acc->wmax, round_res[8]);
    acc->dropped += round_res[9];
    acc->rejected_pre += static_cast<double>(rej);
    ctl->nan_round = static_cast<long long>(round_res[6]);
}

// MultiChannel::Adapt and MaxDifference (MultiChannel.cc:109-154), then the
// cumulative table of std::discrete_distribution (libstdc++ _M_initialize:
// normalise by the accumulated sum, partial_sum, last entry forced to 1).
// mode 0: only rebuild cp from alpha.
__global__ void k_alpha_update(double *__restrict__ alpha, double *__restrict__ best, double *__restrict__ min_diff,
                               double *__restrict__ cp, const double *__restrict__ train, int nch, double beta,
                               double min_alpha, int mode) {
    if (threadIdx.x != 0) return;
    alpha_update(alpha, best, min_diff, cp, train, nch, beta, min_alpha, mode);
}

// Event generation: MultiChannel::GeneratePoint + GenerateWeight for n points.
__global__ void k_generate(const ChannelProgram *__restrict__ progs, const double *__restrict__ grids,
                           const double *__restrict__ alpha, const double *__restrict__ cp, int nch, int dims,
                           int bins, int n_ext, uint64_t seed, uint64_t ctr0, long long n,
                           const IntegrandDesc *__restrict__ f, double *__restrict__ mom_out,
                           double *__restrict__ wgt_out, int32_t *__restrict__ ch_out,
                           const PointProgram *__restrict__ pp) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    double r[CHILI_MAX_DIMS + 1];
    load_uniforms(seed, ctr0 + i, nullptr, dims + 1, r);
    const int c = select_channel(cp, nch, r[dims]);
    double jac;
    V4 mom[CHILI_MAX_SLOTS];
    double m2[CHILI_MAX_SLOTS];
    double w = 0;
    if (grid_map_checked(grids + static_cast<size_t>(c) * dims * (bins + 1), dims, bins, r, jac)) {
        fs_generate(progs + c, r, mom, m2);
        double x[CHILI_MAX_DIMS], xs[CHILI_MAX_DIMS];
        const double wt = pp ? combined_weight_pp(pp, grids, alpha, dims, bins, c, mom, x, xs, nullptr, 0,
                                                  edge_before_table(dims, bins))
                             : combined_weight(progs, grids, alpha, nch, dims, bins, c, mom, x, xs, nullptr, 0);
        const double fv = eval_momenta(f, mom, n_ext);
        w = wt == 0 ? 0 : fv * wt;
        if (!isfinite(w)) w = 0;
    } else {
        for (int s = 0; s < n_ext; ++s) mom[s] = V4{CUDART_NAN, CUDART_NAN, CUDART_NAN, CUDART_NAN};
    }
    if (mom_out)
        for (int s = 0; s < n_ext; ++s) {
            double *o = mom_out + (i * n_ext + s) * 4;
            o[0] = mom[s].e; o[1] = mom[s].x; o[2] = mom[s].y; o[3] = mom[s].z;
        }
    if (wgt_out) wgt_out[i] = w;
    if (ch_out) ch_out[i] = c;
}

// Interface::Evaluate (nanobind.hh:23-50): uniforms through one channel's
// FSMapper, no grid.
__global__ void k_evaluate_batch(const ChannelProgram *__restrict__ prog, const double *__restrict__ u,
                                 double *__restrict__ out, long long n, const IntegrandDesc *__restrict__ f) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const int nd = prog->ndims, ne = prog->n_ext;
    double r[CHILI_MAX_DIMS];
    for (int d = 0; d < nd; ++d) r[d] = u[i * nd + d];
    V4 mom[CHILI_MAX_SLOTS];
    double m2[CHILI_MAX_SLOTS];
    fs_generate(prog, r, mom, m2);
    if (!preprocess(f, mom)) {
        out[i] = 0;
        return;
    }
    const double w = fs_weight(prog, mom, r);
    out[i] = w == 0 ? 0 : eval_momenta(f, mom, ne) * w;
}

// ------------------------------------------------------------- unweighting
// Hit-or-miss flag of every listed point i < n_pre (point k = list[i], value
// rec_val[i]): keep when r * w_max < |v|, r the accept-stream uniform of
// counter ctr0 + k.  keep[i] for all i < m (0 beyond the list); per block:
// sum of values, largest value, overweight count.
__global__ void __launch_bounds__(kFwdBlock) k_unw_flag(const int32_t *__restrict__ list,
                                                         const RoundCtl *__restrict__ ctl_pre,
                                                         const double *__restrict__ rec_val, uint64_t seed,
                                                         uint64_t ctr0, double w_max, long long m,
                                                         uint8_t *__restrict__ keep, double *__restrict__ part) {
    const long long i = blockIdx.x * static_cast<long long>(kFwdBlock) + threadIdx.x;
    const long long n_pre = ctl_pre->n_acc;
    double v = 0.0, mx = -1.7976931348623157e308, over = 0.0;
    int kp = 0;
    if (i < m && i < n_pre) {
        const long long k = list[i];
        v = rec_val[i];
        double r, r_unused;
        uniform_pair(seed, ctr0 + static_cast<uint64_t>(k), kStreamAccept, 0u, r, r_unused);
        kp = r * w_max < fabs(v) ? 1 : 0;
        mx = v;
        over = (kp && fabs(v) > w_max) ? 1.0 : 0.0;
    }
    if (i < m) keep[i] = static_cast<uint8_t>(kp);
    double sum = warp_sum(v);
    mx = warp_max(mx);
    over = warp_sum(over);
    __shared__ double ws[kFwdBlock / 32][3];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        ws[w][0] = sum;
        ws[w][1] = mx;
        ws[w][2] = over;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = -1.7976931348623157e308, c = 0;
        for (int q = 0; q < kFwdBlock / 32; ++q) {
            a += ws[q][0];
            b = std_max(b, ws[q][1]);
            c += ws[q][2];
        }
        part[blockIdx.x * 3 + 0] = a;
        part[blockIdx.x * 3 + 1] = b;
        part[blockIdx.x * 3 + 2] = c;
    }
}

// Ordered fold of k_unw_flag's partials into out[3] (one block of 256:
// strided, then a fixed tree).
__global__ void __launch_bounds__(256) k_unw_reduce(const double *__restrict__ part, long long nb,
                                                    double *__restrict__ out) {
    __shared__ double s[3][256];
    const int t = threadIdx.x;
    double a = 0, b = -1.7976931348623157e308, c = 0;
    for (long long q = t; q < nb; q += 256) {
        a += part[q * 3 + 0];
        b = std_max(b, part[q * 3 + 1]);
        c += part[q * 3 + 2];
    }
    s[0][t] = a;
    s[1][t] = b;
    s[2][t] = c;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (t < w) {
            s[0][t] += s[0][t + w];
            s[1][t] = std_max(s[1][t], s[1][t + w]);
            s[2][t] += s[2][t + w];
        }
        __syncthreads();
    }
    if (t == 0) {
        out[0] = s[0][0];
        out[1] = s[1][0];
        out[2] = s[2][0];
    }
}

// Kept event j (j < ctl_keep->n_acc) -> output slot base + j (< max_events):
// momenta [event][leg][E, px, py, pz], weight sign(v) max(|v|, w_max),
// channel.
__global__ void __launch_bounds__(kFwdBlock) k_unw_write(
    const int32_t *__restrict__ kept, const RoundCtl *__restrict__ ctl_keep, const int32_t *__restrict__ list,
    const double *__restrict__ mom_soa, long long m, int n_ext, const int32_t *__restrict__ ich,
    const double *__restrict__ rec_val, double w_max, long long base, long long max_events,
    double *__restrict__ mom_out, double *__restrict__ wgt_out, int32_t *__restrict__ ch_out) {
    const long long j = blockIdx.x * static_cast<long long>(kFwdBlock) + threadIdx.x;
    if (j >= ctl_keep->n_acc || j >= m) return;
    const long long e = base + j;
    if (e >= max_events) return;
    const long long i = kept[j];
    const long long k = list[i];
    const double v = rec_val[i];
    if (mom_out)
        for (int s = 0; s < n_ext; ++s) {
            double *o = mom_out + (e * n_ext + s) * 4;
            for (int c = 0; c < 4; ++c) o[c] = mom_soa[(4 * s + c) * m + k];
        }
    if (wgt_out) wgt_out[e] = copysign(std_max(fabs(v), w_max), v);
    if (ch_out) ch_out[e] = ich[k];
}

}  // namespace chili_dev
