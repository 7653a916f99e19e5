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

#include "channel_program.h"
#include "common.cuh"
#include "fsmapper.cuh"
#include "grid.cuh"
#include "integrands.cuh"

namespace chili_dev {

__device__ __forceinline__ V4 load_v4(const double *__restrict__ soa, int node, long long m, long long i) {
    return V4{soa[(4 * node + 0) * m + i], soa[(4 * node + 1) * m + i], soa[(4 * node + 2) * m + i],
              soa[(4 * node + 3) * m + i]};
}
__device__ __forceinline__ void store_v4(double *__restrict__ soa, int node, long long m, long long i, V4 v) {
    soa[(4 * node + 0) * m + i] = v.e;
    soa[(4 * node + 1) * m + i] = v.x;
    soa[(4 * node + 2) * m + i] = v.y;
    soa[(4 * node + 3) * m + i] = v.z;
}

// Nodes of point i = list[i]: externals copied from the chunk's momenta
// (mom_soa, stride mc), compounds summed as the reference's tmp_mom.
__global__ void __launch_bounds__(256) k_pp_nodes(const PointProgram *__restrict__ pp, const double *__restrict__ mom_soa,
                                                  long long mc, const int32_t *__restrict__ list,
                                                  const int32_t *__restrict__ ich_arr,
                                                  const long long *__restrict__ n_list, long long base,
                                                  double *__restrict__ node_soa, int32_t *__restrict__ ich_tile,
                                                  long long m) {
    const long long i = blockIdx.x * 256ll + threadIdx.x;  // tile-local point
    if (i >= m || base + i >= *n_list) return;
    const long long k = list[base + i];
    ich_tile[i] = ich_arr[k];
    const int ne = pp->n_ext, nn = pp->n_nodes;
    for (int s = 0; s < ne; ++s) store_v4(node_soa, s, m, i, load_v4(mom_soa, s, mc, k));
    for (int s = ne; s < nn; ++s)
        store_v4(node_soa, s, m, i, load_v4(node_soa, pp->node_a[s], m, i) + load_v4(node_soa, pp->node_b[s], m, i));
}

// One thread per (point, item): items 0..n_tents-1 are t-channel entries
// (Channel.cc:160-186), then decay weights (Channel.cc:83-113), then two-body
// decays (Channel.cc:222-237).
// KIND selects the item type (0 t-entries, 1 decay weights, 2 two-body
// decays), so that each type gets its own register allocation; the two-body
// decays (80 registers unbounded) are held to 64 for four resident blocks
// per SM (2.3% faster items on the 2->4 workload than three).
template <int KIND>
__global__ void __launch_bounds__(256, KIND == 2 ? 4 : 1) k_pp_items(const PointProgram *__restrict__ pp,
                                                  const double *__restrict__ node_soa,
                                                  const long long *__restrict__ n_list, long long base, long long m,
                                                  double *__restrict__ memo) {
    const long long i = blockIdx.y * 256ll + threadIdx.x;  // tile-local point
    if (i >= m || base + i >= *n_list) return;
    // consecutive blocks: items of the same points (L2 reuse)
    int item = blockIdx.x + (KIND >= 1 ? pp->n_tents : 0) + (KIND >= 2 ? pp->n_dws : 0);
    const double sqrts = pp->sqrts, ptmax = pp->ptmax;
    if (KIND == 0 && item < pp->n_tents) {
        const int t = item;
        const double ptmin = pp->tent_ptmin[t];
        const V4 q = load_v4(node_soa, pp->tent_node[t], m, i);
        const double pt = sqrt(pt2(q));
        const double f2 = 2 * ptmin + pt;
        double *o = memo + static_cast<long long>(pp->memo_tent + 5 * t) * m + i;
        o[0] = pt * ptmax / 2 / ptmin / (2 * ptmin + ptmax) * (f2 * f2);
        o[2 * m] = pt * (ptmax + 2 * ptmin) / (ptmax * (pt + 2 * ptmin));
        double etamax = sqrts / 2 / pt;
        etamax = log(etamax + sqrt(etamax * etamax - 1));
        etamax = isnan(etamax) ? 99 : etamax;
        etamax = std_min(etamax, pp->tent_etacut[t]);
        o[m] = 2 * etamax * 2 * kPi;
        o[3 * m] = (rapidity(q) / etamax + 1) / 2;
        o[4 * m] = phi_0_2pi(q) / 2 / kPi;
        return;
    }
    item -= pp->n_tents;
    if (KIND == 1 && item < pp->n_dws) {
        const int k = item;
        const V4 a = load_v4(node_soa, pp->dw_c1[k], m, i), b = load_v4(node_soa, pp->dw_c2[k], m, i);
        const double r = sqrt(fabs(mass2(a))) + sqrt(fabs(mass2(b)));
        const double smin = std_max(std_max(r * r, pp->dw_smin2[k]), pp->dw_cut[k]);
        const double s = mass2(load_v4(node_soa, pp->dw_node[k], m, i));
        double u, w;
        if (smin == pp->dw_smin_c[k]) {  // the usual case: smin-only terms precomputed
            w = pp->dw_massless[k] ? massless_prop_weight_c(0.99, pp->dw_t1[k], pp->dw_t2[k], s, u)
                                   : massive_prop_weight_c(pp->dw_mass[k], pp->dw_width[k], pp->dw_t1[k],
                                                           pp->dw_t2[k], s, u);
        } else {
            w = pp->dw_massless[k] ? massless_prop_weight(0.99, smin, pp->dw_smax[k], s, u)
                                   : massive_prop_weight(pp->dw_mass[k], pp->dw_width[k], smin, pp->dw_smax[k], s, u);
        }
        double *o = memo + static_cast<long long>(pp->memo_dw + 2 * k) * m + i;
        o[0] = w;
        o[m] = u;
        return;
    }
    item -= pp->n_dws;
    if (KIND == 2 && item < pp->n_sws) {
        const int k = item;
        double r1, r2;
        const double w = schannel_weight(load_v4(node_soa, pp->sw_a[k], m, i), load_v4(node_soa, pp->sw_b[k], m, i),
                                         r1, r2);
        double *o = memo + static_cast<long long>(pp->memo_sw + 3 * k) * m + i;
        o[0] = w;
        o[m] = r1;
        o[2 * m] = r2;
    }
}

// Fills the (smin, smax)-only propagator terms of the point program with the
// device's own pow/atan, so that the shortcut in k_pp_items reproduces the
// full evaluation bit for bit.
__global__ void k_pp_prepare(PointProgram *__restrict__ pp) {
    const int k = threadIdx.x + blockIdx.x * blockDim.x;
    if (k < pp->n_dws) pp_prepare_entry(pp, k);
}

// One thread per (point, chain): WgtTChan's weight and last uniform
// (Channel.cc:160-202), with the entries' factors taken from the memo.
__global__ void __launch_bounds__(256) k_pp_chains(const PointProgram *__restrict__ pp,
                                                   const double *__restrict__ node_soa,
                                                   const long long *__restrict__ n_list, long long base, long long m,
                                                   double *__restrict__ memo, uint8_t *__restrict__ cfail) {
    const long long i = blockIdx.y * 256ll + threadIdx.x;  // tile-local point
    if (i >= m || base + i >= *n_list) return;
    const int c = blockIdx.x;  // consecutive blocks: chains of the same points
    const double sqrts = pp->sqrts;
    double wt = kTwoPi;
    V4 psum{0., 0., 0., 0.};
    const int len = pp->chain_len[c];
    for (int e = 0; e < len; ++e) {
        const int t = pp->chain_tent[c][e];
        const double *tm = memo + static_cast<long long>(pp->memo_tent + 5 * t) * m + i;
        wt *= pp->inv16pi3;
        wt *= tm[0];
        wt *= tm[m];
        psum = psum + load_v4(node_soa, pp->tent_node[t], m, i);
    }
    const V4 q = load_v4(node_soa, pp->chain_last[c], m, i);
    const double mjets2 = mass2(psum);
    const double yjets = rapidity(psum);
    const double ptj2 = pt2(psum);
    const double qt = sqrt(mass2(q) + ptj2);
    const double mt = sqrt(mjets2 + ptj2);
    const double yv = rapidity(q);
    const double ymin = -log(sqrts / qt * (1 - mt / sqrts * exp(-yjets)));
    const double ymax = log(sqrts / qt * (1 - mt / sqrts * exp(yjets)));
    const double dely = ymax - ymin;
    double *o = memo + static_cast<long long>(pp->memo_chain + 2 * c) * m + i;
    if (isnan(ymax) || isnan(ymin)) {
        o[0] = 0;
        o[m] = 0;
        cfail[c * m + i] = 1;
    } else {
        o[0] = wt * (dely / sqrts / sqrts);
        o[m] = (yv - ymin) / dely;
        cfail[c * m + i] = 0;
    }
}

// Pair Breit-Wigner / t-channel integrand reading the externals from the
// node buffer (same arithmetic as eval_momenta).
__device__ __forceinline__ double eval_momenta_soa(const IntegrandDesc *__restrict__ f,
                                                   const double *__restrict__ node_soa, long long m, long long i,
                                                   int n_ext) {
    if (f->kind != CHILI_FUNC_PROPAGATOR && f->kind != CHILI_FUNC_PROPAGATOR_TOP2) return 1.0;
    const bool top2 = f->kind == CHILI_FUNC_PROPAGATOR_TOP2;
    const double mm = f->p[0], g = f->p[1], mt = f->p[2];
    const double m2 = mm * mm, mw2 = mm * mm * g * g, mt2 = mt * mt;
    double sum = 0, big1 = 0, big2 = 0;
    for (int a = 2; a < n_ext; ++a) {
        const V4 pa = load_v4(node_soa, a, m, i);
        for (int b = a + 1; b < n_ext; ++b) {
            const double d = mass2(pa + load_v4(node_soa, b, m, i)) - m2;
            const double bw = 1.0 / (d * d + mw2);
            sum += bw;
            if (bw > big1) {
                big2 = big1;
                big1 = bw;
            } else if (bw > big2) {
                big2 = bw;
            }
        }
    }
    const V4 p0 = load_v4(node_soa, 0, m, i);
    double tprod = 1;
    for (int b = 2; b < n_ext; ++b) tprod *= 1.0 / (fabs(mass2(p0 + load_v4(node_soa, b, m, i))) + mt2);
    return (top2 ? big1 * big2 : sum) * tprod;
}

// One thread per (point, channel = blockIdx.x): channel c's density, the
// product of its items in the reference's order (Channel.cc:40-61), and its
// VEGAS weight on the uniforms the position map selects.  When c's chain
// fails, its last uniform is the one the shared buffer still holds: the last
// uniform of the latest earlier channel whose chain did not fail (zero if
// none).  Writes dcv/vwv (tile-local, stride m), the density record and, for
// the point's own channel, the histogram slots.
// HINTS false (batched tasks): the plain bin search and widths from the
// edges, no hint tables.
template <int DIMS, bool HINTS = true>
__global__ void __launch_bounds__(128) k_pp_channel(
    const PointProgram *__restrict__ pp, const double *__restrict__ grids, const uint32_t *__restrict__ hints,
    const uint8_t *__restrict__ sorted, const double *__restrict__ widths, int bins, const double *__restrict__ memo,
    const uint8_t *__restrict__ cfail, const int32_t *__restrict__ ich_tile, const long long *__restrict__ n_list,
    long long base, long long m, long long mr, int should_opt, double *__restrict__ dcv, double *__restrict__ vwv,
    int32_t *__restrict__ rec_slot, double *__restrict__ rec_dens) {
    const long long i = blockIdx.y * 128ll + threadIdx.x;  // tile-local point
    const long long r = base + i;                          // record index
    if (i >= m || r >= *n_list) return;
    const int c = blockIdx.x;  // consecutive blocks: channels of the same points
    const PPChannel &C = pp->ch[c];
    const bool fail = cfail[C.chain * m + i] != 0;
    double wdec = 1;
    for (int k = 0; k < C.n_dec; ++k) {
        wdec *= memo[static_cast<long long>(pp->memo_dw + 2 * C.dw[k]) * m + i];
        wdec /= kTwoPi;
    }
    const double wt = memo[static_cast<long long>(pp->memo_chain + 2 * C.chain) * m + i];
    double ws = 1;
    for (int k = 0; k < C.n_sd; ++k) ws *= memo[static_cast<long long>(pp->memo_sw + 3 * C.sw[k]) * m + i];
    const double dc = wdec * wt * ws;
    double x[DIMS];
    if (!fail) {
        const int16_t *pos = pp->pos_src[c];
#pragma unroll
        for (int p = 0; p < DIMS; ++p) x[p] = memo[static_cast<long long>(pos[p]) * m + i];
    } else {
        const int16_t *pos = pp->pos_src_fail[c];
#pragma unroll
        for (int p = 0; p < DIMS - 1; ++p) x[p] = memo[static_cast<long long>(pos[p]) * m + i];
        double stale = 0.0;
        for (int q = c - 1; q >= 0; --q) {
            if (!cfail[pp->ch[q].chain * m + i]) {
                stale = memo[static_cast<long long>(pp->pos_src[q][DIMS - 1]) * m + i];
                break;
            }
        }
        x[DIMS - 1] = stale;
    }
    const int H = kHintPerBin * bins;
    const double fb = static_cast<double>(bins);
    const double before = edge_before_table(DIMS, bins);
    const double *g = grids + static_cast<size_t>(c) * DIMS * (bins + 1);
    const uint32_t *hc = HINTS ? hints + static_cast<size_t>(c) * DIMS * H : nullptr;
    const double *wc = HINTS ? widths + static_cast<size_t>(c) * DIMS * bins : nullptr;
    const uint8_t *sc = HINTS ? sorted + c * DIMS : nullptr;
    const bool chosen = should_opt && c == ich_tile[i];
    double vw = 1.0;
#pragma unroll
    for (int p = 0; p < DIMS; ++p) {
        int b;
        double wdt;
        if constexpr (HINTS) {
            b = find_bin_hinted(g + p * (bins + 1), hc + p * H, __ldg(sc + p) != 0, bins, H, x[p]);
            wdt = bin_width_t(g, wc, bins, p, b, before);
        } else {
            b = find_bin(g + p * (bins + 1), bins, x[p]);
            wdt = bin_width(g, bins, p, b, before);
        }
        vw = __dmul_rn(vw, __dmul_rn(wdt, fb));
        if (chosen) {
            const int s = p * bins + b;
            rec_slot[p * mr + r] = s >= 0 ? c * DIMS * bins + s : -1;
        }
    }
    dcv[static_cast<long long>(c) * m + i] = dc;
    vwv[static_cast<long long>(c) * m + i] = vw;
    if (rec_dens) rec_dens[static_cast<long long>(c) * mr + r] = dc;
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
    double acc = 0.0;
    const int nch = pp->nch;
    for (int c = 0; c < nch; ++c)
        acc += __ldg(alpha + c) / dcv[static_cast<long long>(c) * m + i] / vwv[static_cast<long long>(c) * m + i];
    double wgt = 1.0 / acc;
    const double fv = eval_momenta_soa(f, node_soa, m, i, pp->n_ext);
    double val = wgt == 0 ? 0 : fv * wgt;
    uint8_t ok = 1;
    if (isnan(val)) {
        val = wgt = 0;
        ok = 0;
    }
    rec_val[r] = val;
    rec_wgt[r] = wgt;
    rec_ok[r] = ok;
}

}  // namespace chili_dev
