// phase_dev.cuh -- device functions of the phased weight pass and of the
// ordered compaction, with explicit block coordinates, shared by the
// kernels of one launch per step (pipeline.cuh, kernels.cuh) and by the
// grouped launches of the batched integrands (batch.cu), where one launch
// covers the pieces of many tasks.
#pragma once

#include "channel_program.h"
#include "common.cuh"
#include "fsmapper.cuh"
#include "grid.cuh"
#include "integrands.cuh"
#include "mc_device.cuh"

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
__device__ __forceinline__ void pp_nodes_block(const PointProgram *__restrict__ pp, const double *__restrict__ mom_soa,
                                               long long mc, const int32_t *__restrict__ list,
                                               const int32_t *__restrict__ ich_arr,
                                               const long long *__restrict__ n_list, long long base,
                                               double *__restrict__ node_soa, int32_t *__restrict__ ich_tile,
                                               long long m, long long bx) {
    const long long i = bx * 256ll + threadIdx.x;  // tile-local point
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
// Block (bx = item of this kind, by = point block).
template <int KIND>
__device__ __forceinline__ void pp_items_block(const PointProgram *__restrict__ pp,
                                               const double *__restrict__ node_soa,
                                               const long long *__restrict__ n_list, long long base, long long m,
                                               double *__restrict__ memo, int bx, long long by) {
    const long long i = by * 256ll + threadIdx.x;  // tile-local point
    if (i >= m || base + i >= *n_list) return;
    // consecutive blocks: items of the same points (L2 reuse)
    int item = bx + (KIND >= 1 ? pp->n_tents : 0) + (KIND >= 2 ? pp->n_dws : 0);
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

// One thread per (point, chain): WgtTChan's weight and last uniform
// (Channel.cc:160-202), with the entries' factors taken from the memo.
__device__ __forceinline__ void pp_chains_block(const PointProgram *__restrict__ pp,
                                                const double *__restrict__ node_soa,
                                                const long long *__restrict__ n_list, long long base, long long m,
                                                double *__restrict__ memo, uint8_t *__restrict__ cfail, int bx,
                                                long long by) {
    const long long i = by * 256ll + threadIdx.x;  // tile-local point
    if (i >= m || base + i >= *n_list) return;
    const int c = bx;  // consecutive blocks: chains of the same points
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

__device__ __forceinline__ void pp_combine_point(const PointProgram *__restrict__ pp, const double *__restrict__ alpha,
                                                 const double *dcv, const double *vwv,
                                                 const double *__restrict__ node_soa, long long m, long long i,
                                                 long long r, const IntegrandDesc *__restrict__ f,
                                                 double *__restrict__ rec_val, double *__restrict__ rec_wgt,
                                                 uint8_t *__restrict__ rec_ok, bool coherent) {
    double acc = 0.0;
    const int nch = pp->nch;
    for (int c = 0; c < nch; ++c) {
        const long long q = static_cast<long long>(c) * m + i;
        // written by other blocks of this launch: read from L2, past L1
        const double d = coherent ? __ldcg(dcv + q) : dcv[q];
        const double v = coherent ? __ldcg(vwv + q) : vwv[q];
        acc += __ldg(alpha + c) / d / v;
    }
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

// Channel c's density and VEGAS weight at tile point i (record r).
// TAB: grids / hints / sorted / widths are channel c's own tables staged in
// shared memory (plain loads), instead of the tables of every channel in
// global memory.
template <int DIMS, bool HINTS, bool TAB = false>
__device__ __forceinline__ void pp_channel_point(
    const PointProgram *__restrict__ pp, const double *__restrict__ grids, const uint32_t *__restrict__ hints,
    const uint8_t *__restrict__ sorted, const double *__restrict__ widths, int bins, const double *__restrict__ memo,
    const uint8_t *__restrict__ cfail, const int32_t *__restrict__ ich_tile, long long m, long long mr,
    int should_opt, double *__restrict__ dcv, double *__restrict__ vwv, int32_t *__restrict__ rec_slot,
    double *__restrict__ rec_dens, long long i, long long r, int c) {
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
    const double *g = TAB ? grids : grids + static_cast<size_t>(c) * DIMS * (bins + 1);
    const uint32_t *hc = HINTS ? (TAB ? hints : hints + static_cast<size_t>(c) * DIMS * H) : nullptr;
    const double *wc = HINTS ? (TAB ? widths : widths + static_cast<size_t>(c) * DIMS * bins) : nullptr;
    const uint8_t *sc = HINTS ? (TAB ? sorted : sorted + c * DIMS) : nullptr;
    const bool chosen = should_opt && c == ich_tile[i];
    double vw = 1.0;
#pragma unroll
    for (int p = 0; p < DIMS; ++p) {
        int b;
        double wdt;
        if constexpr (HINTS) {
            b = find_bin_hinted<!TAB>(g + p * (bins + 1), hc + p * H, tab_ld<!TAB>(sc + p) != 0, bins, H, x[p]);
            wdt = bin_width_t<!TAB>(g, wc, bins, p, b, before);
        } else {
            b = find_bin<!TAB>(g + p * (bins + 1), bins, x[p]);
            wdt = bin_width<!TAB>(g, bins, p, b, before);
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

// (The body as a device function, so that a grouped launch can run it for
// one piece of work per block.)
__device__ __forceinline__ void mc_scan_body(const int32_t *__restrict__ block_count, int nb,
                                             const uint8_t *__restrict__ flag, long long m, long long needed,
                                             const long long *__restrict__ remaining, int cut_at_remaining,
                                             long long *__restrict__ block_off, RoundCtl *__restrict__ ctl) {
    if (remaining) {
        const long long rem = *remaining;
        if (rem <= 0) {
            if (threadIdx.x == 0) {
                ctl->cut = 0;
                ctl->n_acc = 0;
            }
            return;
        }
        if (cut_at_remaining) needed = rem;
    }
    __shared__ long long wsum[32];
    __shared__ long long running_s;
    __shared__ int cut_block_s;
    __shared__ long long cut_off_s;
    if (threadIdx.x == 0) {
        running_s = 0;
        cut_block_s = -1;
        cut_off_s = 0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int base = 0; base < nb; base += 1024) {
        const int i = base + threadIdx.x;
        const long long c = i < nb ? block_count[i] : 0;
        long long incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) wsum[w] = incl;
        __syncthreads();
        if (w == 0) {
            long long v = wsum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const long long t = __shfl_up_sync(0xffffffffu, v, o);
                if (lane >= o) v += t;
            }
            wsum[lane] = v;  // inclusive warp totals
        }
        __syncthreads();
        const long long warp_excl = w > 0 ? wsum[w - 1] : 0;
        const long long off = running_s + warp_excl + incl - c;
        if (i < nb) {
            block_off[i] = off;
            if (off < needed && needed <= off + c) {
                cut_block_s = i;
                cut_off_s = off;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) running_s += wsum[31];
        __syncthreads();
    }
    const long long total = running_s;
    if (cut_block_s < 0) {
        if (threadIdx.x == 0) {
            ctl->cut = m;
            ctl->n_acc = total;
        }
        return;
    }
    // position of the r-th accepted point inside the cut block
    const long long r = needed - cut_off_s;
    const long long k = static_cast<long long>(cut_block_s) * kFwdBlock + threadIdx.x;
    int f = 0;
    if (threadIdx.x < kFwdBlock && k < m) f = flag[k] ? 1 : 0;
    long long incl = f;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    __syncthreads();
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    long long pre = 0;
    for (int q = 0; q < w; ++q) pre += wsum[q];
    incl += pre;
    if (threadIdx.x < kFwdBlock && f && incl == r) {
        ctl->cut = k + 1;
        ctl->n_acc = needed;
    }
}

// Block bx of the ordered compaction of the accepted points.
__device__ __forceinline__ void mc_compact_block(const uint8_t *__restrict__ flag,
                                                 const long long *__restrict__ block_off,
                                                 const RoundCtl *__restrict__ ctl, long long m,
                                                 int32_t *__restrict__ list, long long bx) {
    const long long k = bx * static_cast<long long>(kFwdBlock) + threadIdx.x;
    const long long cut = ctl->cut;
    const int a = (k < m && k < cut) ? flag[k] : 0;
    const unsigned ballot = __ballot_sync(0xffffffffu, a);
    __shared__ int wc[kFwdBlock / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) wc[w] = __popc(ballot);
    __syncthreads();
    int pre = 0;
    for (int q = 0; q < w; ++q) pre += wc[q];
    if (a) {
        const long long pos = block_off[bx] + pre + __popc(ballot & ((1u << lane) - 1u));
        list[pos] = static_cast<int32_t>(k);
    }
}

}  // namespace chili_dev
