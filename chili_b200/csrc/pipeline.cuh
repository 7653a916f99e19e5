// pipeline.cuh -- the phased form of the all-channel weight pass.
//
// Integrand::GenerateWeight (include/Channel/Integrand.hh:112-123) evaluated
// for a list of points in four kernels with small per-thread state, instead of
// one thread running every channel's inverse mapping from start to end:
//   k_pp_nodes     gathers the point's external momenta and sums the compound
//                  currents (one thread per point)
//   k_pp_items     every t-channel entry, decay propagator weight and
//                  two-body decay weight (one thread per point and item)
//   k_pp_chains    every t-channel chain's weight and last uniform (one thread
//                  per point and chain)
//   k_pp_channel   every channel's density and VEGAS weight (one thread per
//                  point and channel; the channel's uniforms come from the
//                  memo slots through its position map and stay in registers:
//                  DIMS is a compile-time constant)
//   k_pp_combine   per point, the combined weight in channel order, the
//                  integrand and the records of k_mc_weight.
// Intermediate values live in SoA buffers [slot][point] of one tile of points
// (stride m), so every access of a warp is coalesced and a tile's buffers
// stay in L2.
#pragma once

#include "phase_dev.cuh"

namespace chili_dev {



__global__ void __launch_bounds__(256) k_pp_nodes(const PointProgram *__restrict__ pp, const double *__restrict__ mom_soa,
                                                  long long mc, const int32_t *__restrict__ list,
                                                  const int32_t *__restrict__ ich_arr,
                                                  const long long *__restrict__ n_list, long long base,
                                                  double *__restrict__ node_soa, int32_t *__restrict__ ich_tile,
                                                  long long m) {
    pp_nodes_block(pp, mom_soa, mc, list, ich_arr, n_list, base, node_soa, ich_tile, m, blockIdx.x);
}


template <int KIND>
__global__ void __launch_bounds__(256, KIND == 2 ? 4 : 1) k_pp_items(const PointProgram *__restrict__ pp,
                                                  const double *__restrict__ node_soa,
                                                  const long long *__restrict__ n_list, long long base, long long m,
                                                  double *__restrict__ memo) {
    pp_items_block<KIND>(pp, node_soa, n_list, base, m, memo, blockIdx.x, blockIdx.y);
}

// Fills the (smin, smax)-only propagator terms of the point program with the
// device's own pow/atan, so that the shortcut in k_pp_items reproduces the
// full evaluation bit for bit.
__global__ void k_pp_prepare(PointProgram *__restrict__ pp) {
    const int k = threadIdx.x + blockIdx.x * blockDim.x;
    if (k < pp->n_dws) pp_prepare_entry(pp, k);
}


__global__ void __launch_bounds__(256) k_pp_chains(const PointProgram *__restrict__ pp,
                                                   const double *__restrict__ node_soa,
                                                   const long long *__restrict__ n_list, long long base, long long m,
                                                   double *__restrict__ memo, uint8_t *__restrict__ cfail) {
    pp_chains_block(pp, node_soa, n_list, base, m, memo, cfail, blockIdx.x, blockIdx.y);
}


// k_pp_channel with channel c's edge, hint, width and monotone tables staged
// in shared memory (blockIdx.x = c, kTabPoints points per block): the bin
// searches' scattered reads hit shared memory instead of L1, where the tables
// of all channels do not fit. The same per-point function and arithmetic as
// k_pp_channel.
constexpr int kTabPoints = 1024;
constexpr int kTabThreads = 256;

// Shared-memory bytes of one channel's tables.
__host__ __device__ inline size_t channel_tab_bytes(int dims, int bins) {
    const size_t H = static_cast<size_t>(kHintPerBin) * bins;
    return 8 * static_cast<size_t>(dims) * (2 * bins + 1) + 4 * dims * H + dims;
}

template <int DIMS>
__global__ void __launch_bounds__(kTabThreads) k_pp_channel_tab(
    const PointProgram *__restrict__ pp, const double *__restrict__ grids, const uint32_t *__restrict__ hints,
    const uint8_t *__restrict__ sorted, const double *__restrict__ widths, int bins, const double *__restrict__ memo,
    const uint8_t *__restrict__ cfail, const int32_t *__restrict__ ich_tile, const long long *__restrict__ n_list,
    long long base, long long m, long long mr, int should_opt, double *__restrict__ dcv, double *__restrict__ vwv,
    int32_t *__restrict__ rec_slot, double *__restrict__ rec_dens) {
    extern __shared__ double tab[];
    const int c = blockIdx.x;
    const int H = kHintPerBin * bins;
    const int ne = DIMS * (bins + 1), nw = DIMS * bins, nh = DIMS * H;
    double *se = tab;
    double *sw = se + ne;
    uint32_t *sh = reinterpret_cast<uint32_t *>(sw + nw);
    uint8_t *ss = reinterpret_cast<uint8_t *>(sh + nh);
    const double *ge = grids + static_cast<size_t>(c) * ne;
    const double *gw = widths + static_cast<size_t>(c) * nw;
    const uint32_t *gh = hints + static_cast<size_t>(c) * nh;
    for (int k = threadIdx.x; k < ne; k += kTabThreads) se[k] = __ldg(ge + k);
    for (int k = threadIdx.x; k < nw; k += kTabThreads) sw[k] = __ldg(gw + k);
    for (int k = threadIdx.x; k < nh; k += kTabThreads) sh[k] = __ldg(gh + k);
    if (threadIdx.x < DIMS) ss[threadIdx.x] = __ldg(sorted + c * DIMS + threadIdx.x);
    __syncthreads();
    const long long n = *n_list;
#pragma unroll 1
    for (int j = 0; j < kTabPoints / kTabThreads; ++j) {
        const long long i = blockIdx.y * static_cast<long long>(kTabPoints) + j * kTabThreads + threadIdx.x;
        const long long r = base + i;
        if (i < m && r < n)
            pp_channel_point<DIMS, true, true>(pp, se, sh, ss, sw, bins, memo, cfail, ich_tile, m, mr, should_opt,
                                               dcv, vwv, rec_slot, rec_dens, i, r, c);
    }
}

// The combine step fused into k_pp_channel: the last of a point block's
// nch channel blocks to finish (an arrival counter per point block, reset by
// that block for the next launch) runs k_pp_combine's per-point work on the
// block's 128 points, while their densities are still in L2.
struct PPCombine {
    const double *alpha;
    const double *node_soa;
    const IntegrandDesc *f;
    double *rec_val, *rec_wgt;
    uint8_t *rec_ok;
    unsigned *arrivals;  // one per point block of the tile, zero between launches
};



// One thread per (point, channel = blockIdx.x): channel c's density, the
// product of its items in the reference's order (Channel.cc:40-61), and its
// VEGAS weight on the uniforms the position map selects.  When c's chain
// fails, its last uniform is the one the shared buffer still holds: the last
// uniform of the latest earlier channel whose chain did not fail (zero if
// none).  Writes dcv/vwv (tile-local, stride m), the density record and, for
// the point's own channel, the histogram slots.
// HINTS false (batched tasks): the plain bin search and widths from the
// edges, no hint tables.
// FUSE: the combine step runs in the last channel block of each point block.
template <int DIMS, bool HINTS = true, bool FUSE = false>
__global__ void __launch_bounds__(128) k_pp_channel(
    const PointProgram *__restrict__ pp, const double *__restrict__ grids, const uint32_t *__restrict__ hints,
    const uint8_t *__restrict__ sorted, const double *__restrict__ widths, int bins, const double *__restrict__ memo,
    const uint8_t *__restrict__ cfail, const int32_t *__restrict__ ich_tile, const long long *__restrict__ n_list,
    long long base, long long m, long long mr, int should_opt, double *__restrict__ dcv, double *__restrict__ vwv,
    int32_t *__restrict__ rec_slot, double *__restrict__ rec_dens, PPCombine comb = PPCombine{}) {
    const long long i = blockIdx.y * 128ll + threadIdx.x;  // tile-local point
    const long long r = base + i;                          // record index
    const bool valid = i < m && r < *n_list;
    if (valid) pp_channel_point<DIMS, HINTS>(pp, grids, hints, sorted, widths, bins, memo, cfail, ich_tile, m, mr,
                                             should_opt, dcv, vwv, rec_slot, rec_dens, i, r, blockIdx.x);
    if constexpr (FUSE) {
        __shared__ bool last;
        __threadfence();  // this block's densities visible before its arrival
        __syncthreads();
        if (threadIdx.x == 0) last = atomicAdd(comb.arrivals + blockIdx.y, 1u) == gridDim.x - 1;
        __syncthreads();
        if (!last) return;
        __threadfence();
        if (valid)
            pp_combine_point(pp, comb.alpha, dcv, vwv, comb.node_soa, m, i, r, comb.f, comb.rec_val, comb.rec_wgt,
                             comb.rec_ok, true);
        if (threadIdx.x == 0) comb.arrivals[blockIdx.y] = 0u;
    }
}

// Per point: 1 / sum_c alpha_c / dens_c / vw_c in channel order
// (Integrand.hh:118-122), the integrand and the value records.
__global__ void __launch_bounds__(256) k_pp_combine(const PointProgram *__restrict__ pp,
                                                    const double *__restrict__ alpha,
                                                    const double *__restrict__ dcv, const double *__restrict__ vwv,
                                                    const double *__restrict__ node_soa,
                                                    const long long *__restrict__ n_list, long long base, long long m,
                                                    const IntegrandDesc *__restrict__ f, double *__restrict__ rec_val,
                                                    double *__restrict__ rec_wgt, uint8_t *__restrict__ rec_ok) {
    const long long i = blockIdx.x * 256ll + threadIdx.x;
    const long long r = base + i;
    if (i >= m || r >= *n_list) return;
    pp_combine_point(pp, alpha, dcv, vwv, node_soa, m, i, r, f, rec_val, rec_wgt, rec_ok, false);
}

}  // namespace chili_dev
