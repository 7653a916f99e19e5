// batch.cu -- many independent integrations in one persistent launch per
// iteration (include/chili_gpu.h, "batched integrands"; no counterpart in
// the reference, which integrates one Integrand per MultiChannel/Vegas
// object).
//
// A task is either a camel function integrated by plain VEGAS
// (Vegas::operator(), Vegas.cc:18-52: ncalls points, f*J, per-bin (f J)^2
// histogram, AdaptiveMap::Adapt) or a multichannel FSMapper integrand with
// the combined weight of all its channels (Integrand::GenerateWeight,
// Integrand.hh:112-123), its channel histograms and alpha training
// (MultiChannel.hh:167-194).  A multichannel task's iteration keeps the
// reference's retry loop (MultiChannel.hh:214-248): points are drawn until
// ncalls of them pass PreProcess with a finite value, and the rejected ones
// enter StatsData as zero-valued calls (option batch_retry; with it off, the
// default, a fixed budget of ncalls drawn points).  The retry loop runs in
// rounds: round 0 draws the task's planned count (ncalls at first, then the
// points the previous iterations needed, plus a margin) and cuts the task at
// its ncalls-th accepted point; a task still short of ncalls after a round
// (too few accepted points, or NaN values) draws again from the counter after
// the last one counted, in further rounds sized on the device.
//
// Work units are tiles of blockDim * points_per_thread points of one task;
// a persistent grid (resident blocks of every SM) pulls units from an atomic
// counter, so tasks of 1e4 and 1e6 points share the machine without one
// launch per task. Per unit one StatsData partial; per task an ordered fold
// of its partials (deterministic), then the channel-weight update and a
// batched grid adaptation over every (task, channel, dimension). The
// iteration (resets, evaluation, folds, adaptation, iteration counter) is
// captured once in a CUDA graph and replayed (with the retry loop: the first
// round and the final part as two graphs, further rounds launched directly
// between them); block size and points per thread are chosen by timing the
// candidates on the first call.
#include <cuda_runtime.h>
#include <math_constants.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "channel_program.h"
#include "context.h"
#include "phase_dev.cuh"

using namespace chili_dev;

namespace {

// Channels per multichannel task (the per-thread channel densities live in
// local memory).
constexpr int kBatchMaxCh = 64;
// Parallel branches of the phased multichannel task chains in the graph.
constexpr int kPhBranches = 8;
// Grouped mode: waves on up to this many streams (option
// "batch_wave_streams"), so that one wave's tail overlaps the next one's start.
constexpr int kMaxWaveStreams = 4;

struct BatchTask {
    int32_t kind, dims, bins, nch;
    long long ncalls;
    long long draw;            // points a round may draw (phased tasks; ncalls with a fixed budget)
    int32_t retry;             // 1: the reference's retry loop (rounds, RetryState)
    int32_t pad_;
    long long unit0, units;    // first work unit, number of units
    long long grid_off;        // doubles: nch * dims * (bins+1)
    long long hist_off;        // doubles: nch * dims * bins
    long long hint_off;        // bin-search hints (uint32): nch * dims * kHintPerBin * bins
    long long width_off;       // bin widths (doubles): nch * dims * bins
    long long sorted_off;      // monotone flags (bytes): nch * dims
    int32_t ch_off;            // first ChannelProgram / channel-weight slot
    int32_t desc;              // IntegrandDesc index
    int32_t pp;                // PointProgram index, -1: per-channel weights
    int32_t phased;            // 1: weighted by the phased pass, outside k_batch_eval
    double grid_alpha, beta, min_alpha;
    double before;             // edge_before_table(dims, bins)
    uint64_t key;              // Philox key of the task
};

// Retry loop of one multichannel task in the current iteration (reset by
// k_rt_begin, advanced by k_rt_end after every round).
struct RetryState {
    long long need;       // accepted points with a finite value still wanted
    long long ctr0;       // counter offset of the next round (points counted so far)
    long long lim;        // points the next round draws (at most the task's draw)
    long long rounds;
    // this round, summed over the task's pieces (their RoundCtl lives in the
    // wave's arena, which a later wave on the same stream reuses)
    unsigned long long counted_round;   // points before the pieces' cuts
    unsigned long long accepted_round;  // accepted points before the cuts
    unsigned long long nan_round;       // of those, NaN values
    unsigned long long nan_total;       // NaN values of the iteration
    double acc[6];        // StatsData of the rounds so far
};

// Work unit u of the iteration: unit `unit` of task `task`.  Units are
// handed out interleaved over the tasks (ordered by their position within
// their task), so that the blocks running at one time work on many tasks and
// their histogram and training adds spread over many addresses.
struct UnitRef {
    int32_t task, unit;
};

struct BatchDev {
    const BatchTask *tasks;
    int ntasks;
    const UnitRef *umap;  // [nunits]
    long long nunits;
    const ChannelProgram *progs;
    const PointProgram *pps;
    const IntegrandDesc *descs;
    double *grids, *grids_new, *hist, *atrain;  // atrain per channel slot
    uint32_t *hints;                            // bin-search tables of the grids (BatchTask offsets)
    double *widths;
    uint8_t *sorted;
    double *alpha, *best, *mindiff, *cp;        // per channel slot; mindiff per task
    double *part;                              // [nunits][6], task-contiguous
    double *stats;                             // [iter slot][ntasks][6]
    int stat_slots;
    unsigned long long *next_unit;
    unsigned long long *iter;
    RetryState *retry;  // [ntasks]
    int *rflag;         // after a round: 1 some task needs another round, 2 counter space exhausted
    int ppt;
};

// One iteration's evaluation: persistent blocks pull units.  Per unit one
// StatsData partial; histogram adds go straight to global memory, the
// channel-training terms are summed per warp, then per block in shared
// memory, and reach global memory once per unit and channel.
__global__ void __launch_bounds__(256) k_batch_eval(BatchDev B) {
    __shared__ long long s_unit;
    __shared__ double ws[8][6];
    __shared__ double s_atr[kBatchMaxCh];
    const uint64_t iter = *B.iter;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    if (t < kBatchMaxCh) s_atr[t] = 0.0;
    for (;;) {
        if (t == 0) s_unit = static_cast<long long>(atomicAdd(B.next_unit, 1ull));
        __syncthreads();
        const long long u = s_unit;
        __syncthreads();
        if (u >= B.nunits) break;
        const UnitRef ur = B.umap[u];
        const BatchTask T = B.tasks[ur.task];
        const IntegrandDesc *f = B.descs + T.desc;
        const long long tile = static_cast<long long>(blockDim.x) * B.ppt;
        const long long p0 = ur.unit * tile;
        const int D = T.dims, bins = T.bins;
        const size_t gsz = static_cast<size_t>(D) * (bins + 1);
        double cnt = 0, sum = 0, sum2 = 0, mn = 1.7976931348623157e308, mx = 2.2250738585072014e-308, nf = 0;
        for (int q = 0; q < B.ppt; ++q) {
            const long long i = p0 + static_cast<long long>(q) * blockDim.x + t;
            const bool active = i < T.ncalls;
            const uint64_t ctr = (iter << 32) + static_cast<uint64_t>(i);
            double val = 0;
            if (T.kind == CHILI_TASK_CAMEL) {
                if (active) {
                    double r[CHILI_MAX_DIMS];
                    load_uniforms(T.key, ctr, nullptr, D, r);
                    const double *g = B.grids + T.grid_off;
                    double jac;
                    if (grid_map_checked(g, D, bins, r, jac)) val = camel(f, r, D) * jac;
                    else val = CUDART_NAN;
                    const double v2 = val * val;
                    double *H = B.hist + T.hist_off;
                    for (int j = 0; j < D; ++j) {
                        const int s = j * bins + find_bin(g + j * (bins + 1), bins, r[j]);
                        if (s >= 0) atomicAdd(H + s, v2);
                    }
                }
            } else {
                // the task is the block's: every lane reaches the reductions
                double dens[kBatchMaxCh];
                double vw = 0;  // val^2 * weight of a point that trains, else 0
                if (active) {
                    double r[CHILI_MAX_DIMS + 1];
                    load_uniforms(T.key, ctr, nullptr, D + 1, r);
                    const double *cp = B.cp + T.ch_off;
                    const int c = select_channel(cp, T.nch, r[D]);
                    const double *grids = B.grids + T.grid_off;
                    double jac;
                    if (grid_map_checked(grids + c * gsz, D, bins, r, jac)) {
                        const ChannelProgram *progs = B.progs + T.ch_off;
                        V4 mom[CHILI_MAX_SLOTS];
                        double m2[CHILI_MAX_SLOTS];
                        fs_generate(progs + c, r, mom, m2);
                        if (preprocess(f, mom)) {
                            double x[CHILI_MAX_DIMS], xs[CHILI_MAX_DIMS];
                            const double *al = B.alpha + T.ch_off;
                            const double wgt =
                                T.pp >= 0 ? combined_weight_pp(B.pps + T.pp, grids, al, D, bins, c, mom, x, xs, dens,
                                                               1, T.before)
                                          : combined_weight(progs, grids, al, T.nch, D, bins, c, mom, x, xs, dens, 1);
                            const double fv = eval_momenta(f, mom, progs[0].n_ext);
                            val = wgt == 0 ? 0 : fv * wgt;
                            if (isnan(val)) val = 0;  // a retry in the reference; a call of value 0 here
                            if (val != 0) {
                                // AddTrainData (MultiChannel.hh:167-180)
                                const double v2 = val * val;
                                double *H = B.hist + T.hist_off + static_cast<size_t>(c) * D * bins;
                                const double *g = grids + c * gsz;
                                for (int j = 0; j < D; ++j) {
                                    const int s = j * bins + find_bin(g + j * (bins + 1), bins, xs[j]);
                                    if (s >= 0) atomicAdd(H + s, v2);
                                }
                                vw = v2 * wgt;
                            }
                        }
                    }
                }
                const unsigned any = __ballot_sync(0xffffffffu, vw != 0);
                if (any) {
                    for (int k = 0; k < T.nch; ++k) {
                        double term = vw != 0 ? vw / dens[k] : 0.0;
                        if (!isfinite(term)) term = 0.0;  // non-finite terms dropped
                        term = warp_sum(term);
                        if (lane == 0 && term != 0) atomicAdd(s_atr + k, term);
                    }
                }
            }
            if (active) {
                cnt += 1;
                sum += val;
                sum2 += val * val;
                mn = std_min(mn, val);
                mx = std_max(mx, val);
                nf += (val != 0);
            }
        }
        cnt = warp_sum(cnt);
        sum = warp_sum(sum);
        sum2 = warp_sum(sum2);
        mn = warp_min(mn);
        mx = warp_max(mx);
        nf = warp_sum(nf);
        if (lane == 0) {
            ws[w][0] = cnt; ws[w][1] = mn; ws[w][2] = mx; ws[w][3] = sum; ws[w][4] = sum2; ws[w][5] = nf;
        }
        __syncthreads();
        if (t == 0) {
            double a[6] = {ws[0][0], ws[0][1], ws[0][2], ws[0][3], ws[0][4], ws[0][5]};
            for (int k = 1; k < static_cast<int>(blockDim.x >> 5); ++k) {
                a[0] += ws[k][0]; a[1] = std_min(a[1], ws[k][1]); a[2] = std_max(a[2], ws[k][2]);
                a[3] += ws[k][3]; a[4] += ws[k][4]; a[5] += ws[k][5];
            }
            double *o = B.part + (T.unit0 + ur.unit) * 6;
            for (int k = 0; k < 6; ++k) o[k] = a[k];
        }
        if (T.kind != CHILI_TASK_CAMEL && t < T.nch) {
            if (s_atr[t] != 0) atomicAdd(B.atrain + T.ch_off + t, s_atr[t]);
            s_atr[t] = 0.0;
        }
    }
}

// Phased multichannel tasks (the shared-entry weight pass of the single
// iterations, pipeline.cuh, one tile of up to ph_tile points of one task at a
// time): step 1, the points p0 .. p0+mm-1 of task ti as k_batch_eval draws
// them (Philox key of the task, counters (iteration << 32) + point), the
// channel, VEGAS map, FSMapper and PreProcess; accepted points' external
// momenta to mom_soa [slot][component][ms], per block of kFwdBlock points
// the accepted count.  ctr_off: the retry round's counter offset (the points
// the task's earlier rounds of this iteration counted).
__device__ __forceinline__ void bt_forward_block(const BatchDev &B, int ti, long long p0, long long mm,
                                                 double *__restrict__ mom_soa, long long ms,
                                                 int32_t *__restrict__ ich_out, uint8_t *__restrict__ flag,
                                                 int32_t *__restrict__ block_count, long long bx,
                                                 long long ctr_off = 0) {
    const BatchTask T = B.tasks[ti];
    const long long k = bx * static_cast<long long>(kFwdBlock) + threadIdx.x;
    int acc = 0;
    if (k < mm) {
        const int D = T.dims, bins = T.bins;
        const uint64_t ctr = (*B.iter << 32) + static_cast<uint64_t>(ctr_off + p0 + k);
        double r[CHILI_MAX_DIMS + 1];
        load_uniforms(T.key, ctr, nullptr, D + 1, r);
        const int c = select_channel(B.cp + T.ch_off, T.nch, r[D]);
        const double *g = B.grids + T.grid_off + static_cast<size_t>(c) * D * (bins + 1);
        double jac;
        if (grid_map_checked(g, D, bins, r, jac)) {
            V4 mom[CHILI_MAX_SLOTS];
            double m2[CHILI_MAX_SLOTS];
            const ChannelProgram *prog = B.progs + T.ch_off + c;
            fs_generate(prog, r, mom, m2);
            if (preprocess(B.descs + T.desc, mom)) {
                acc = 1;
                for (int s = 0; s < prog->n_ext; ++s) {
                    mom_soa[(4 * s + 0) * ms + k] = mom[s].e;
                    mom_soa[(4 * s + 1) * ms + k] = mom[s].x;
                    mom_soa[(4 * s + 2) * ms + k] = mom[s].y;
                    mom_soa[(4 * s + 3) * ms + k] = mom[s].z;
                }
            }
        }
        ich_out[k] = c;
        flag[k] = static_cast<uint8_t>(acc);
    }
    const int cnt = __syncthreads_count(acc);
    if (threadIdx.x == 0) block_count[bx] = cnt;
}

__global__ void __launch_bounds__(kFwdBlock) k_bt_forward(BatchDev B, int ti, long long p0, long long mm,
                                                          double *__restrict__ mom_soa, long long ms,
                                                          int32_t *__restrict__ ich_out, uint8_t *__restrict__ flag,
                                                          int32_t *__restrict__ block_count) {
    bt_forward_block(B, ti, p0, mm, mom_soa, ms, ich_out, flag, block_count, blockIdx.x);
}

// Step 3 (after compact_launch and pp_pass_launch): block b of the tile is
// work unit p0/kFwdBlock + b of the task; its accepted points are the records
// block_off[b] .. + block_count[b] (the list keeps point order), the others
// are calls of value 0.  StatsData partial of the unit, AddTrainData
// (MultiChannel.hh:167-180) histogram adds and channel-training terms, as
// k_batch_eval does per point (NaN values count as 0).  ctl (retry rounds):
// only the points before the round's cut are calls and only the first n_acc
// accepted points are records; R: the round's NaN values are counted (they
// do not count towards ncalls, MultiChannel.hh:229-235).
__device__ __forceinline__ void bt_accum_block(const BatchDev &B, int ti, long long p0, long long mm,
                                               const int32_t *__restrict__ block_count,
                                               const long long *__restrict__ block_off,
                                               const double *__restrict__ rec_val,
                                               const double *__restrict__ rec_wgt,
                                               const uint8_t *__restrict__ rec_ok,
                                               const int32_t *__restrict__ rec_slot,
                                               const double *__restrict__ rec_dens, long long mr, long long bx,
                                               const RoundCtl *__restrict__ ctl = nullptr,
                                               RetryState *__restrict__ R = nullptr) {
    __shared__ double ws[kFwdBlock / 32][6];
    __shared__ double s_atr[kBatchMaxCh];
    const BatchTask T = B.tasks[ti];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    if (t < kBatchMaxCh) s_atr[t] = 0.0;
    __syncthreads();
    const long long k0 = bx * static_cast<long long>(kFwdBlock);
    const long long upto = ctl ? (ctl->cut < mm ? ctl->cut : mm) : mm;  // points counted in this piece
    const long long active = upto - k0 <= 0 ? 0 : (upto - k0 < kFwdBlock ? upto - k0 : kFwdBlock);
    int nrec = block_count[bx];
    if (ctl) {
        // a block past the cut has no records; where the whole piece lies
        // past it (the task had its ncalls before the piece) the scan wrote
        // no offsets, so block_off is not read
        if (active == 0) {
            nrec = 0;
        } else {
            const long long left = ctl->n_acc - block_off[bx];
            nrec = left <= 0 ? 0 : (left < nrec ? static_cast<int>(left) : nrec);
        }
    }
    const long long r = block_off[bx] + t;
    if (R) {
        const int nan_recs = __syncthreads_count(t < nrec && !rec_ok[r]);
        if (t == 0 && nan_recs) atomicAdd(&R->nan_round, static_cast<unsigned long long>(nan_recs));
    }
    double val = 0, vw = 0;
    if (t < nrec) {
        val = rec_ok[r] ? rec_val[r] : 0.0;
        if (isnan(val)) val = 0;
        if (val != 0) {
            const double v2 = val * val;
            double *H = B.hist + T.hist_off;
            for (int j = 0; j < T.dims; ++j) {
                const int s = rec_slot[j * mr + r];
                if (s >= 0) atomicAdd(H + s, v2);
            }
            vw = v2 * rec_wgt[r];
        }
    }
    const unsigned any = __ballot_sync(0xffffffffu, vw != 0);
    if (any) {
        for (int c = 0; c < T.nch; ++c) {
            double term = 0.0;
            if (vw != 0) {  // only the records' own lanes read their densities
                term = vw / rec_dens[c * mr + r];
                if (!isfinite(term)) term = 0.0;  // non-finite terms dropped
            }
            term = warp_sum(term);
            if (lane == 0 && term != 0) atomicAdd(s_atr + c, term);
        }
    }
    // StatsData over the unit's active points: the records, and value-0
    // calls for the rest (they enter min and max as 0)
    double cnt = t < nrec ? 1 : 0, sum = val, sum2 = val * val, nf = val != 0 ? 1 : 0;
    double mn = t < nrec ? val : 1.7976931348623157e308, mx = t < nrec ? val : 2.2250738585072014e-308;
    cnt = warp_sum(cnt);
    sum = warp_sum(sum);
    sum2 = warp_sum(sum2);
    nf = warp_sum(nf);
    mn = warp_min(mn);
    mx = warp_max(mx);
    if (lane == 0) {
        ws[w][0] = cnt; ws[w][1] = mn; ws[w][2] = mx; ws[w][3] = sum; ws[w][4] = sum2; ws[w][5] = nf;
    }
    __syncthreads();
    if (t == 0) {
        double a[6] = {ws[0][0], ws[0][1], ws[0][2], ws[0][3], ws[0][4], ws[0][5]};
        for (int q = 1; q < kFwdBlock / 32; ++q) {
            a[0] += ws[q][0]; a[1] = std_min(a[1], ws[q][1]); a[2] = std_max(a[2], ws[q][2]);
            a[3] += ws[q][3]; a[4] += ws[q][4]; a[5] += ws[q][5];
        }
        if (nrec < active) {  // rejected points: calls of value 0
            a[0] += static_cast<double>(active - nrec);
            a[1] = std_min(a[1], 0.0);
            a[2] = std_max(a[2], 0.0);
        }
        double *o = B.part + (T.unit0 + p0 / kFwdBlock + bx) * 6;
        for (int q = 0; q < 6; ++q) o[q] = a[q];
    }
    if (t < T.nch && s_atr[t] != 0) atomicAdd(B.atrain + T.ch_off + t, s_atr[t]);
}

__global__ void __launch_bounds__(kFwdBlock) k_bt_accum(BatchDev B, int ti, long long p0, long long mm,
                                                        const int32_t *__restrict__ block_count,
                                                        const long long *__restrict__ block_off,
                                                        const double *__restrict__ rec_val,
                                                        const double *__restrict__ rec_wgt,
                                                        const uint8_t *__restrict__ rec_ok,
                                                        const int32_t *__restrict__ rec_slot,
                                                        const double *__restrict__ rec_dens, long long mr) {
    bt_accum_block(B, ti, p0, mm, block_count, block_off, rec_val, rec_wgt, rec_ok, rec_slot, rec_dens, mr,
                   blockIdx.x);
}

// ----------------------------------------------- grouped phased weight pass
// The phased multichannel tasks of an iteration run in waves: a wave is a
// list of pieces (points [p0, p0 + mm) of one task, with buffers of their
// own carved out of one arena, stride ms = mm rounded up to kFwdBlock), and
// each step of the pass is ONE launch over all pieces of the wave: the
// blocks of a step are numbered piece after piece (prefix[step][k] is the
// first block of piece k) and each block finds its piece by binary search.
// The per-piece work is exactly the per-task chain's (the same device
// functions), so the results do not depend on the grouping.
struct Piece {
    int32_t ti, nb;                    // task; blocks of kFwdBlock points
    int32_t n_items[3], n_chains, nch, dims, bins;
    long long p0, mm, ms;
    const PointProgram *pp;
    const double *grids, *alpha;
    const uint32_t *hints;  // the task's bin-search tables (rows of its grids)
    const double *widths;
    const uint8_t *sorted;
    const IntegrandDesc *f;
    double *mom;
    int32_t *ich;
    uint8_t *flag;
    int32_t *bcount;
    long long *boff;
    RoundCtl *ctl;
    int32_t *list;
    double *node, *memo, *dcv, *vwv;
    uint8_t *cfail;
    int32_t *ich_tile;
    double *val, *wgt;
    uint8_t *ok;
    int32_t *slot;
    double *dens;
};
enum { GS_FWD, GS_COMPACT, GS_NODES, GS_ITEM0, GS_ITEM1, GS_ITEM2, GS_CHAINS, GS_CHANNEL, GS_COMBINE, GS_ACCUM,
       kGroupSteps };

struct WaveDev {
    const Piece *pieces;
    int n;
    const long long *prefix;  // [kGroupSteps][n + 1]
    int ch_pts;               // points per block of the channel step (a multiple of 128)
};

// The piece k in [lo, hi) of a step whose blocks [prefix[k], prefix[k+1])
// hold block b.
__device__ __forceinline__ int find_piece(const long long *__restrict__ pre, int lo, int hi, long long b) {
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(pre + mid) <= b) lo = mid;
        else hi = mid;
    }
    return lo;
}

#define CHILI_PIECE(step)                                                        \
    const long long *pre_ = W.prefix + static_cast<size_t>(step) * (W.n + 1);    \
    const long long b_ = blockIdx.x + blk0;                                      \
    const int k_ = find_piece(pre_, lo, hi, b_);                                 \
    const Piece &P = W.pieces[k_];                                               \
    const long long lb = b_ - pre_[k_];

// Points of piece P that the task's current retry round draws: the round's
// limit R.lim (from the task's first point), none once the task has its
// ncalls.
__device__ __forceinline__ long long round_points(const RetryState &R, const Piece &P) {
    if (R.need <= 0) return 0;
    const long long m = R.lim - P.p0;
    return m <= 0 ? 0 : (m < P.mm ? m : P.mm);
}

__global__ void __launch_bounds__(kFwdBlock) k_g_forward(BatchDev B, WaveDev W, int lo, int hi, long long blk0) {
    CHILI_PIECE(GS_FWD)
    if (B.tasks[P.ti].retry) {
        const RetryState &R = B.retry[P.ti];
        bt_forward_block(B, P.ti, P.p0, round_points(R, P), P.mom, P.ms, P.ich, P.flag, P.bcount, lb, R.ctr0);
    } else {
        bt_forward_block(B, P.ti, P.p0, P.mm, P.mom, P.ms, P.ich, P.flag, P.bcount, lb);
    }
}

// Per piece, the ordered offsets of its accepted points.  Retry rounds: the
// piece is cut at the point that brings its task to ncalls accepted points,
// counting the accepted points of the task's earlier pieces (adjacent in the
// wave, in counter order) first.
__global__ void __launch_bounds__(1024) k_g_scan(BatchDev B, WaveDev W) {
    const Piece &P = W.pieces[blockIdx.x];
    if (!B.tasks[P.ti].retry) {
        mc_scan_body(P.bcount, P.nb, P.flag, P.mm, P.mm + 1, nullptr, 0, P.boff, P.ctl);
        return;
    }
    const RetryState &R = B.retry[P.ti];  // need, lim, ctr0: fixed during the round
    __shared__ unsigned long long before_s;
    __shared__ long long rem_s;
    if (threadIdx.x == 0) before_s = 0;
    __syncthreads();
    for (int j = static_cast<int>(blockIdx.x) - 1; j >= 0 && W.pieces[j].ti == P.ti; --j) {
        const Piece &Q = W.pieces[j];
        unsigned long long c = 0;
        for (int b = threadIdx.x; b < Q.nb; b += blockDim.x) c += static_cast<unsigned long long>(Q.bcount[b]);
        if (c) atomicAdd(&before_s, c);
    }
    __syncthreads();
    if (threadIdx.x == 0) rem_s = R.need - static_cast<long long>(before_s);
    __syncthreads();
    mc_scan_body(P.bcount, P.nb, P.flag, round_points(R, P), 0, &rem_s, 1, P.boff, P.ctl);
    __syncthreads();
    if (threadIdx.x == 0) {
        RetryState &Rw = B.retry[P.ti];
        atomicAdd(&Rw.counted_round, static_cast<unsigned long long>(P.ctl->cut));
        atomicAdd(&Rw.accepted_round, static_cast<unsigned long long>(P.ctl->n_acc));
    }
}

__global__ void __launch_bounds__(kFwdBlock) k_g_compact(WaveDev W, int lo, int hi, long long blk0) {
    CHILI_PIECE(GS_COMPACT)
    mc_compact_block(P.flag, P.boff, P.ctl, P.mm, P.list, lb);
}

__global__ void __launch_bounds__(256) k_g_nodes(WaveDev W, int lo, int hi, long long blk0) {
    CHILI_PIECE(GS_NODES)
    pp_nodes_block(P.pp, P.mom, P.ms, P.list, P.ich, &P.ctl->n_acc, 0, P.node, P.ich_tile, P.ms, lb);
}

template <int KIND>
__global__ void __launch_bounds__(256, KIND == 2 ? 4 : 1) k_g_items(WaveDev W, int lo, int hi, long long blk0) {
    CHILI_PIECE(GS_ITEM0 + KIND)
    const int ni = P.n_items[KIND];
    pp_items_block<KIND>(P.pp, P.node, &P.ctl->n_acc, 0, P.ms, P.memo, static_cast<int>(lb % ni), lb / ni);
}

__global__ void __launch_bounds__(256) k_g_chains(WaveDev W, int lo, int hi, long long blk0) {
    CHILI_PIECE(GS_CHAINS)
    pp_chains_block(P.pp, P.node, &P.ctl->n_acc, 0, P.ms, P.memo, P.cfail, static_cast<int>(lb % P.n_chains),
                    lb / P.n_chains);
}

// Pieces [lo, hi) of the wave have DIMS dimensions. A block works on one
// channel c of one piece; TAB: the block first stages channel c's edges,
// bin widths, hint tables and monotone flags (dynamic shared memory) and runs
// the hinted bin search of the single-integrand path on them, instead of a
// plain binary search through L1 on the edges in global memory.
template <int DIMS, bool TAB>
__global__ void __launch_bounds__(128) k_g_channel(WaveDev W, int lo, int hi, long long blk0) {
    CHILI_PIECE(GS_CHANNEL)
    const int c = static_cast<int>(lb % P.nch);
    const long long i0 = (lb / P.nch) * W.ch_pts;  // W.ch_pts points per block: one table copy for all of them
    const long long n = P.ctl->n_acc;
    if constexpr (TAB) {
        extern __shared__ double se[];
        const int bins = P.bins, H = kHintPerBin * bins;
        const int ne = DIMS * (bins + 1), nw = DIMS * bins, nh = DIMS * H;
        double *sw = se + ne;
        uint32_t *sh = reinterpret_cast<uint32_t *>(sw + nw);
        uint8_t *ss = reinterpret_cast<uint8_t *>(sh + nh);
        const size_t row0 = static_cast<size_t>(c) * DIMS;
        const double *ge = P.grids + row0 * (bins + 1);
        const double *gw = P.widths + row0 * bins;
        const uint32_t *gh = P.hints + row0 * H;
        for (int k = threadIdx.x; k < ne; k += 128) se[k] = __ldg(ge + k);
        for (int k = threadIdx.x; k < nw; k += 128) sw[k] = __ldg(gw + k);
        for (int k = threadIdx.x; k < nh; k += 128) sh[k] = __ldg(gh + k);
        if (threadIdx.x < DIMS) ss[threadIdx.x] = __ldg(P.sorted + row0 + threadIdx.x);
        __syncthreads();
#pragma unroll 1
        for (int j = 0; j < W.ch_pts; j += 128) {
            const long long i = i0 + j + threadIdx.x;
            if (i < P.ms && i < n)
                pp_channel_point<DIMS, true, true>(P.pp, se, sh, ss, sw, bins, P.memo, P.cfail, P.ich_tile, P.ms,
                                                   P.ms, 1, P.dcv, P.vwv, P.slot, P.dens, i, i, c);
        }
    } else {
#pragma unroll 1
        for (int j = 0; j < W.ch_pts; j += 128) {
            const long long i = i0 + j + threadIdx.x;
            if (i < P.ms && i < n)
                pp_channel_point<DIMS, false>(P.pp, P.grids, nullptr, nullptr, nullptr, P.bins, P.memo, P.cfail,
                                              P.ich_tile, P.ms, P.ms, 1, P.dcv, P.vwv, P.slot, P.dens, i, i, c);
        }
    }
}

__global__ void __launch_bounds__(256) k_g_combine(WaveDev W, int lo, int hi, long long blk0) {
    CHILI_PIECE(GS_COMBINE)
    const long long i = lb * 256 + threadIdx.x;
    if (i < P.ms && i < P.ctl->n_acc)
        pp_combine_point(P.pp, P.alpha, P.dcv, P.vwv, P.node, P.ms, i, i, P.f, P.val, P.wgt, P.ok, false);
}

__global__ void __launch_bounds__(kFwdBlock) k_g_accum(BatchDev B, WaveDev W, int lo, int hi, long long blk0) {
    CHILI_PIECE(GS_ACCUM)
    const bool retry = B.tasks[P.ti].retry != 0;
    bt_accum_block(B, P.ti, P.p0, P.mm, P.bcount, P.boff, P.val, P.wgt, P.ok, P.slot, P.dens, P.ms, lb,
                   retry ? P.ctl : nullptr, retry ? B.retry + P.ti : nullptr);
}
#undef CHILI_PIECE

// The PointPrograms' (smin, smax) terms.
__global__ void k_batch_pp_prepare(PointProgram *__restrict__ pps) {
    PointProgram *pp = pps + blockIdx.x;
    for (int k = threadIdx.x; k < pp->n_dws; k += blockDim.x) pp_prepare_entry(pp, k);
}

// Per task (one block of kFoldThreads each): fold of its unit partials into
// the StatsData of this iteration (thread t takes units t, t + kFoldThreads,
// ... in order, then a fixed tree: deterministic); multichannel tasks then
// update their channel weights (MultiChannel::Adapt + MaxDifference,
// MultiChannel.hh:100-140) when adapting.
constexpr int kFoldThreads = 128;

__global__ void __launch_bounds__(kFoldThreads) k_batch_finalize(BatchDev B, int adapt) {
    __shared__ double sh[6][kFoldThreads];
    const int ti = blockIdx.x, t = threadIdx.x;
    const BatchTask T = B.tasks[ti];
    double a[6] = {0, 1.7976931348623157e308, 2.2250738585072014e-308, 0, 0, 0};
    for (long long u = T.unit0 + t; u < T.unit0 + T.units; u += kFoldThreads) {
        const double *p = B.part + u * 6;
        a[0] += p[0];
        a[1] = std_min(a[1], p[1]);
        a[2] = std_max(a[2], p[2]);
        a[3] += p[3];
        a[4] += p[4];
        a[5] += p[5];
    }
    for (int k = 0; k < 6; ++k) sh[k][t] = a[k];
    __syncthreads();
    for (int w = kFoldThreads / 2; w > 0; w >>= 1) {
        if (t < w) {
            sh[0][t] += sh[0][t + w];
            sh[1][t] = std_min(sh[1][t], sh[1][t + w]);
            sh[2][t] = std_max(sh[2][t], sh[2][t + w]);
            sh[3][t] += sh[3][t + w];
            sh[4][t] += sh[4][t + w];
            sh[5][t] += sh[5][t + w];
        }
        __syncthreads();
    }
    if (t == 0) {
        const uint64_t slot = *B.iter % static_cast<uint64_t>(B.stat_slots);
        double *o = B.stats + (slot * B.ntasks + ti) * 6;
        // retry tasks: the StatsData that k_rt_end folded round by round
        for (int k = 0; k < 6; ++k) o[k] = T.retry ? B.retry[ti].acc[k] : sh[k][0];
        if (adapt && T.kind == CHILI_TASK_MULTICHANNEL)
            alpha_update(B.alpha + T.ch_off, B.best + T.ch_off, B.mindiff + ti, B.cp + T.ch_off,
                         B.atrain + T.ch_off, T.nch, T.beta, T.min_alpha, 1);
    }
}

// Retry loop: the state of every retry task at the start of an iteration
// (one thread per task).
__global__ void k_rt_begin(BatchDev B) {
    const int ti = blockIdx.x * blockDim.x + threadIdx.x;
    if (ti >= B.ntasks) return;
    const BatchTask &T = B.tasks[ti];
    if (!T.retry) return;
    RetryState &R = B.retry[ti];
    R.need = T.ncalls;
    R.ctr0 = 0;
    R.lim = T.draw;
    R.rounds = 0;
    R.counted_round = 0;
    R.accepted_round = 0;
    R.nan_round = 0;
    R.nan_total = 0;
    const double e[6] = {0, 1.7976931348623157e308, 2.2250738585072014e-308, 0, 0, 0};
    for (int k = 0; k < 6; ++k) R.acc[k] = e[k];
}

// After a round (one block of kFoldThreads per task): the round's unit
// partials folded in unit order into the task's StatsData, the accepted
// points with a finite value subtracted from need, the counter offset moved
// past the points counted; a task still short of ncalls flags another round,
// sized from this round's rate of accepted points per point drawn.
__global__ void __launch_bounds__(kFoldThreads) k_rt_end(BatchDev B) {
    __shared__ double sh[6][kFoldThreads];
    const int ti = blockIdx.x, t = threadIdx.x;
    const BatchTask T = B.tasks[ti];
    if (!T.retry) return;
    RetryState &R = B.retry[ti];
    if (R.need <= 0) return;  // finished in an earlier round: this round drew nothing for it
    double a[6] = {0, 1.7976931348623157e308, 2.2250738585072014e-308, 0, 0, 0};
    for (long long u = T.unit0 + t; u < T.unit0 + T.units; u += kFoldThreads) {
        const double *p = B.part + u * 6;
        a[0] += p[0];
        a[1] = std_min(a[1], p[1]);
        a[2] = std_max(a[2], p[2]);
        a[3] += p[3];
        a[4] += p[4];
        a[5] += p[5];
    }
    for (int k = 0; k < 6; ++k) sh[k][t] = a[k];
    __syncthreads();
    for (int w = kFoldThreads / 2; w > 0; w >>= 1) {
        if (t < w) {
            sh[0][t] += sh[0][t + w];
            sh[1][t] = std_min(sh[1][t], sh[1][t + w]);
            sh[2][t] = std_max(sh[2][t], sh[2][t + w]);
            sh[3][t] += sh[3][t + w];
            sh[4][t] += sh[4][t + w];
            sh[5][t] += sh[5][t + w];
        }
        __syncthreads();
    }
    if (t != 0) return;
    R.acc[0] += sh[0][0];
    R.acc[1] = std_min(R.acc[1], sh[1][0]);
    R.acc[2] = std_max(R.acc[2], sh[2][0]);
    R.acc[3] += sh[3][0];
    R.acc[4] += sh[4][0];
    R.acc[5] += sh[5][0];
    const long long counted = static_cast<long long>(R.counted_round);
    const long long valid = static_cast<long long>(R.accepted_round) - static_cast<long long>(R.nan_round);
    R.need -= valid;
    R.ctr0 += counted;
    R.nan_total += R.nan_round;
    R.counted_round = 0;
    R.accepted_round = 0;
    R.nan_round = 0;
    R.rounds += 1;
    if (R.need <= 0) return;
    if (R.ctr0 + T.draw >= (1ll << 32)) {  // counters (iteration << 32) + point
        R.need = 0;
        atomicMax(B.rflag, 2);
        return;
    }
    // the next round: the points this round's rate predicts, 1/4 more and two
    // blocks' worth besides, at most the task's draw (the pieces cover no more)
    long long lim = T.draw;
    if (valid > 0 && counted > 0) {
        const double want = static_cast<double>(R.need) * static_cast<double>(counted) / static_cast<double>(valid);
        const double l = 1.25 * want + 2.0 * kFwdBlock;
        if (l < static_cast<double>(T.draw)) lim = static_cast<long long>(l);
    }
    R.lim = lim;
    atomicMax(B.rflag, 1);
}

// Grid adaptation of every (task, channel, dimension): one block each.
struct AdaptJob {
    int32_t task, ch, dim, pad;
};

__global__ void k_batch_adapt(BatchDev B, const AdaptJob *__restrict__ jobs, int njobs, int *status) {
    extern __shared__ double tmp[];
    const int j = blockIdx.x;
    if (j >= njobs) return;
    const AdaptJob J = jobs[j];
    const BatchTask T = B.tasks[J.task];
    // plain VEGAS adapts every grid; MultiChannel::Train skips channels
    // that received no training data
    grid_adapt_block(B.grids + T.grid_off, B.grids_new + T.grid_off, T.dims, T.bins, T.grid_alpha,
                     B.hist + T.hist_off, T.kind == CHILI_TASK_MULTICHANNEL ? 1 : 0, status, J.dim, J.ch, tmp);
}

__global__ void k_batch_commit(BatchDev B, const AdaptJob *__restrict__ jobs, int njobs) {
    // copy the adapted edges back (grids_new -> grids), one block per job
    const int j = blockIdx.x;
    if (j >= njobs) return;
    const AdaptJob J = jobs[j];
    const BatchTask T = B.tasks[J.task];
    const size_t row = static_cast<size_t>(J.ch) * T.dims + J.dim;
    const size_t off = T.grid_off + row * (T.bins + 1);
    for (int k = threadIdx.x; k <= T.bins; k += blockDim.x) B.grids[off + k] = B.grids_new[off + k];
    __syncthreads();
    // the row's bin-search tables for the next iteration's channel step
    build_hint_row(B.grids + off, T.bins, B.hints + T.hint_off + row * (kHintPerBin * T.bins),
                   B.sorted + T.sorted_off + row, B.widths + T.width_off + row * T.bins);
}

// The bin-search tables of every (task, channel, dimension) row, one block
// per row (after the grids are set).
__global__ void k_batch_hints(BatchDev B, const AdaptJob *__restrict__ jobs, int njobs) {
    const int j = blockIdx.x;
    if (j >= njobs) return;
    const AdaptJob J = jobs[j];
    const BatchTask T = B.tasks[J.task];
    const size_t row = static_cast<size_t>(J.ch) * T.dims + J.dim;
    build_hint_row(B.grids + T.grid_off + row * (T.bins + 1), T.bins,
                   B.hints + T.hint_off + row * (kHintPerBin * T.bins), B.sorted + T.sorted_off + row,
                   B.widths + T.width_off + row * T.bins);
}

__global__ void k_batch_next(BatchDev B) {
    if (threadIdx.x == 0) {
        *B.next_unit = 0;
        *B.iter += 1;
    }
}

}  // namespace

struct BatchState {
    std::vector<BatchTask> tasks;
    std::vector<UnitRef> umap;
    std::vector<AdaptJob> jobs;
    int max_bins = 2, nslots = 0;
    long long total_points = 0, nunits = 0;
    DevBuf d_tasks, d_umap, d_pps, d_progs, d_descs, d_grids, d_grids_new, d_hist, d_atrain, d_alpha, d_best, d_mindiff,
        d_cp, d_part, d_stats, d_counters, d_jobs, d_status, d_hints, d_widths, d_sorted;
    int block = 0, ppt = 0, grid_blocks = 0;
    long long n_pulled = 0;  // units k_batch_eval pulls (the tasks that are not phased)
    // phased multichannel tasks: host copies of the point programs (launch
    // sizes) and the tile size (ph_tile points)
    std::vector<PointProgram> pps_host;
    long long ph_tile = 0;
    struct PhBufs {
        DevBuf mom, ich, flag, list, bcount, boff, ctl, node, memo, cfail, dcv, vwv, ich_tile, val, wgt, ok, slot, dens;
    };
    // the task chains run as kPhBranches parallel branches of the graph,
    // each with its own stream (at capture) and tile buffers
    std::vector<PhBufs> ph;
    std::vector<cudaStream_t> ph_streams;
    std::vector<cudaEvent_t> ph_events;
    // grouped mode (option "batch_grouped", the default): the phased tasks in
    // waves of pieces, one launch per step and wave (see Piece)
    bool grouped = false;
    struct WaveHost {
        int first = 0, n = 0;                        // pieces [first, first + n)
        int sidx = 0;                                // stream (and arena) of the wave
        long long prefix_off = 0;                    // into d_prefix
        std::vector<long long> blocks;               // per step: total blocks
        std::vector<std::array<int, 4>> dgroups;     // (dims, k0, k1, bins): pieces [k0, k1) of one dimension, their most bins
    };
    std::vector<Piece> pieces;
    std::vector<WaveHost> waves;
    std::vector<long long> prefix_host;
    DevBuf d_pieces, d_prefix;
    DevBuf d_arena[kMaxWaveStreams];  // wave w uses arena w % nstreams and stream w % nstreams
    int wave_streams = 2;
    int ch_pts = 2048;  // points per block of the channel step (option "batch_channel_points" at planning)
    bool tuned = false;
    cudaGraphExec_t graph = nullptr;
    unsigned long long graph_launches = 0;  // kernels of one replay
    // retry tasks (option batch_retry): the final graph, per-task loop state,
    // the round flag; the waves of a further round (the pieces of the tasks
    // still short of ncalls) and their device copies
    bool has_retry = false;
    cudaGraphExec_t graph_fin = nullptr;
    unsigned long long fin_launches = 0;
    DevBuf d_retry, d_rflag, d_top_pieces, d_top_prefix;
    std::vector<WaveHost> top_waves;
    std::vector<Piece> top_pieces;
    std::vector<long long> top_prefix;
    unsigned long long retry_rounds = 0;  // further rounds run by the last batch_iterate call
    int graph_adapt = -1;
    double last_ms = 0;
    size_t hist_doubles = 0;
    int nslots_alloc = 0;
};

namespace {

int need_batch(chili_ctx *ctx) {
    if (!ctx->batch) return fail(ctx, CHILI_ERR_STATE, "no batch set (chili_gpu_batch_set)");
    return CHILI_OK;
}

BatchDev batch_dev(chili_ctx *ctx) {
    BatchState &S = *ctx->batch;
    BatchDev B{};
    B.tasks = S.d_tasks.as<BatchTask>();
    B.ntasks = static_cast<int>(S.tasks.size());
    B.umap = S.d_umap.as<UnitRef>();
    B.nunits = S.n_pulled;
    B.progs = S.d_progs.as<ChannelProgram>();
    B.pps = S.d_pps.as<PointProgram>();
    B.descs = S.d_descs.as<IntegrandDesc>();
    B.grids = S.d_grids.as<double>();
    B.grids_new = S.d_grids_new.as<double>();
    B.hints = S.d_hints.as<uint32_t>();
    B.widths = S.d_widths.as<double>();
    B.sorted = S.d_sorted.as<uint8_t>();
    B.hist = S.d_hist.as<double>();
    B.atrain = S.d_atrain.as<double>();
    B.alpha = S.d_alpha.as<double>();
    B.best = S.d_best.as<double>();
    B.mindiff = S.d_mindiff.as<double>();
    B.cp = S.d_cp.as<double>();
    B.part = S.d_part.as<double>();
    B.stats = S.d_stats.as<double>();
    B.stat_slots = S.nslots_alloc;
    B.next_unit = S.d_counters.as<unsigned long long>();
    B.iter = S.d_counters.as<unsigned long long>() + 1;
    B.retry = S.d_retry.as<RetryState>();
    B.rflag = S.d_rflag.as<int>();
    B.ppt = S.ppt;
    return B;
}

// Work-unit layout for a block size and points per thread: units of each
// task, interleaved over the tasks in the order of (unit + 1/2) / units.
int layout_units(chili_ctx *ctx, int block, int ppt) {
    BatchState &S = *ctx->batch;
    long long u = 0;
    const long long tile = static_cast<long long>(block) * ppt;
    for (auto &T : S.tasks) {
        // a phased task's units are the kFwdBlock-point blocks of its tiles
        const long long tt = T.phased ? kFwdBlock : tile;
        T.unit0 = u;
        T.units = ((T.phased ? T.draw : T.ncalls) + tt - 1) / tt;
        u += T.units;
    }
    S.nunits = u;
    {
        std::vector<std::pair<double, UnitRef>> order;
        order.reserve(static_cast<size_t>(u));
        for (size_t k = 0; k < S.tasks.size(); ++k)
            for (long long j = 0; j < S.tasks[k].units && !S.tasks[k].phased; ++j)
                order.push_back({(j + 0.5) / static_cast<double>(S.tasks[k].units),
                                 UnitRef{static_cast<int32_t>(k), static_cast<int32_t>(j)}});
        S.umap.resize(order.size());
        S.n_pulled = static_cast<long long>(order.size());
        std::stable_sort(order.begin(), order.end(),
                         [](const auto &a, const auto &b) { return a.first < b.first; });
        for (size_t k = 0; k < order.size(); ++k) S.umap[k] = order[k].second;
    }
    CK(S.d_tasks.ensure(sizeof(BatchTask) * S.tasks.size()));
    CK(cudaMemcpyAsync(S.d_tasks.p, S.tasks.data(), sizeof(BatchTask) * S.tasks.size(), cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(S.d_umap.ensure(sizeof(UnitRef) * std::max<size_t>(S.umap.size(), 1)));
    CK(cudaMemcpyAsync(S.d_umap.p, S.umap.data(), sizeof(UnitRef) * S.umap.size(), cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(S.d_part.ensure(sizeof(double) * 6 * u));
    CK(cudaStreamSynchronize(ctx->stream));
    S.block = block;
    S.ppt = ppt;
    int per_sm = 1, sms = 148;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_eval, block, 0);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    S.grid_blocks = std::max(1, per_sm) * sms;
    return CHILI_OK;
}

// The kernels of one phased task, tile by tile, on ctx->stream with the
// buffers b.
int enqueue_phased_task(chili_ctx *ctx, const BatchDev &B, int ti, BatchState::PhBufs &b) {
    BatchState &S = *ctx->batch;
    const BatchTask &T = S.tasks[static_cast<size_t>(ti)];
    const long long ms = S.ph_tile;
    RoundCtl *ctl = b.ctl.as<RoundCtl>();
    const long long *n_list =
        reinterpret_cast<const long long *>(reinterpret_cast<const char *>(ctl) + offsetof(RoundCtl, n_acc));
    for (long long p0 = 0; p0 < T.ncalls; p0 += ms) {
        const long long mm = std::min(ms, T.ncalls - p0);
        const unsigned nb = static_cast<unsigned>((mm + kFwdBlock - 1) / kFwdBlock);
        k_bt_forward<<<nb, kFwdBlock, 0, ctx->stream>>>(B, ti, p0, mm, b.mom.as<double>(), ms, b.ich.as<int32_t>(),
                                                       b.flag.as<uint8_t>(), b.bcount.as<int32_t>());
        LAUNCHED();
        if (int rc = compact_launch(ctx, b.bcount.as<int32_t>(), static_cast<int>(nb), b.flag.as<uint8_t>(), mm,
                                    b.boff.as<long long>(), ctl, b.list.as<int32_t>()))
            return rc;
        PPPass a{};
        a.pp = S.d_pps.as<PointProgram>() + T.pp;
        a.pp_host = &S.pps_host[static_cast<size_t>(T.pp)];
        a.mom_soa = b.mom.as<double>();
        a.mc = ms;
        a.list = b.list.as<int32_t>();
        a.ich = b.ich.as<int32_t>();
        a.n_list = n_list;
        a.T = mm;
        a.mr = ms;
        a.bins = T.bins;
        a.grids = B.grids + T.grid_off;
        a.node_soa = b.node.as<double>();
        a.memo = b.memo.as<double>();
        a.dcv = b.dcv.as<double>();
        a.vwv = b.vwv.as<double>();
        a.cfail = b.cfail.as<uint8_t>();
        a.ich_tile = b.ich_tile.as<int32_t>();
        a.rec_slot = b.slot.as<int32_t>();
        a.rec_dens = b.dens.as<double>();
        a.alpha = B.alpha + T.ch_off;
        a.f = B.descs + T.desc;
        a.rec_val = b.val.as<double>();
        a.rec_wgt = b.wgt.as<double>();
        a.rec_ok = b.ok.as<uint8_t>();
        if (int rc = pp_pass_launch(ctx, a)) return rc;
        k_bt_accum<<<nb, kFwdBlock, 0, ctx->stream>>>(B, ti, p0, mm, b.bcount.as<int32_t>(), b.boff.as<long long>(),
                                                     b.val.as<double>(), b.wgt.as<double>(), b.ok.as<uint8_t>(),
                                                     b.slot.as<int32_t>(), b.dens.as<double>(), ms);
        LAUNCHED();
    }
    return CHILI_OK;
}

// The phased tasks' waves, one after another on ctx->stream: one launch per
// step and wave.
int enqueue_waves(chili_ctx *ctx, const BatchDev &B, const std::vector<BatchState::WaveHost> &waves,
                  const Piece *d_pieces, const long long *d_prefix, const std::vector<long long> &prefix_host) {
    BatchState &S = *ctx->batch;
    const cudaStream_t caller = ctx->stream;
    for (size_t wi = 0; wi < waves.size(); ++wi) {
        const auto &w = waves[wi];
        ctx->stream = S.ph_streams[static_cast<size_t>(w.sidx)];  // the wave's arena belongs to this stream
        const WaveDev W{d_pieces + w.first, w.n, d_prefix + w.prefix_off, S.ch_pts};
        const long long *pre = prefix_host.data() + w.prefix_off;
        auto blocks = [&](int step) { return static_cast<unsigned>(w.blocks[static_cast<size_t>(step)]); };
        k_g_forward<<<blocks(GS_FWD), kFwdBlock, 0, ctx->stream>>>(B, W, 0, w.n, 0);
        LAUNCHED();
        k_g_scan<<<static_cast<unsigned>(w.n), 1024, 0, ctx->stream>>>(B, W);
        LAUNCHED();
        k_g_compact<<<blocks(GS_COMPACT), kFwdBlock, 0, ctx->stream>>>(W, 0, w.n, 0);
        LAUNCHED();
        k_g_nodes<<<blocks(GS_NODES), 256, 0, ctx->stream>>>(W, 0, w.n, 0);
        LAUNCHED();
        if (blocks(GS_ITEM0)) {
            k_g_items<0><<<blocks(GS_ITEM0), 256, 0, ctx->stream>>>(W, 0, w.n, 0);
            LAUNCHED();
        }
        if (blocks(GS_ITEM1)) {
            k_g_items<1><<<blocks(GS_ITEM1), 256, 0, ctx->stream>>>(W, 0, w.n, 0);
            LAUNCHED();
        }
        if (blocks(GS_ITEM2)) {
            k_g_items<2><<<blocks(GS_ITEM2), 256, 0, ctx->stream>>>(W, 0, w.n, 0);
            LAUNCHED();
        }
        if (blocks(GS_CHAINS)) {
            k_g_chains<<<blocks(GS_CHAINS), 256, 0, ctx->stream>>>(W, 0, w.n, 0);
            LAUNCHED();
        }
        const long long *pc = pre + static_cast<size_t>(GS_CHANNEL) * (w.n + 1);
        for (const auto &g : w.dgroups) {
            const long long b0 = pc[g[1]], nbk = pc[g[2]] - b0;
            if (nbk <= 0) continue;
            // one channel's edges, widths, hints and flags in shared memory
            // when they fit the default 48 KB
            const size_t tab = sizeof(double) * static_cast<size_t>(g[0]) * (2 * g[3] + 1) +
                               sizeof(uint32_t) * static_cast<size_t>(g[0]) * kHintPerBin * g[3] + g[0];
            const bool use_tab = ctx->channel_tables && tab <= 48 * 1024;
            switch (g[0]) {
#define CHILI_GCH(D)                                                                                        \
    case D:                                                                                                 \
        if (use_tab)                                                                                        \
            k_g_channel<D, true><<<static_cast<unsigned>(nbk), 128, tab, ctx->stream>>>(W, g[1], g[2], b0); \
        else                                                                                                \
            k_g_channel<D, false><<<static_cast<unsigned>(nbk), 128, 0, ctx->stream>>>(W, g[1], g[2], b0);  \
        break;
                CHILI_GCH(1) CHILI_GCH(4) CHILI_GCH(7) CHILI_GCH(10) CHILI_GCH(13) CHILI_GCH(16) CHILI_GCH(19)
                CHILI_GCH(22)
#undef CHILI_GCH
                default: return fail(ctx, CHILI_ERR_STATE, "no phased weight kernel for this dimension");
            }
            LAUNCHED();
        }
        k_g_combine<<<blocks(GS_COMBINE), 256, 0, ctx->stream>>>(W, 0, w.n, 0);
        LAUNCHED();
        k_g_accum<<<blocks(GS_ACCUM), kFwdBlock, 0, ctx->stream>>>(B, W, 0, w.n, 0);
        LAUNCHED();
    }
    ctx->stream = caller;
    return CHILI_OK;
}

// A retry round after the first, launched directly: the waves cut down to
// the pieces of the tasks still short of ncalls (read back from the device),
// each kept on its wave's stream and buffers, then the round's bookkeeping.
int run_retry_round(chili_ctx *ctx) {
    BatchState &S = *ctx->batch;
    BatchDev B = batch_dev(ctx);
    const cudaStream_t main = ctx->stream;
    const int ns = S.wave_streams;
    std::vector<RetryState> R(S.tasks.size());
    CK(cudaMemcpyAsync(R.data(), S.d_retry.p, sizeof(RetryState) * R.size(), cudaMemcpyDeviceToHost, main));
    CK(cudaStreamSynchronize(main));
    // the filtered waves: a task's pieces stay together and in order
    S.top_waves.clear();
    S.top_pieces.clear();
    S.top_prefix.clear();
    for (const auto &w : S.waves) {
        std::vector<int> keep;
        for (int k = 0; k < w.n; ++k) {
            const int ti = S.pieces[static_cast<size_t>(w.first + k)].ti;
            if (S.tasks[static_cast<size_t>(ti)].retry && R[static_cast<size_t>(ti)].need > 0) keep.push_back(k);
        }
        if (keep.empty()) continue;
        BatchState::WaveHost fw;
        fw.sidx = w.sidx;
        fw.first = static_cast<int>(S.top_pieces.size());
        fw.n = static_cast<int>(keep.size());
        fw.prefix_off = static_cast<long long>(S.top_prefix.size());
        for (int st = 0; st < kGroupSteps; ++st) {
            const long long *po = S.prefix_host.data() + w.prefix_off + static_cast<size_t>(st) * (w.n + 1);
            long long acc = 0;
            S.top_prefix.push_back(0);
            for (int k : keep) {
                acc += po[k + 1] - po[k];
                S.top_prefix.push_back(acc);
            }
            fw.blocks.push_back(acc);
        }
        for (size_t j = 0; j < keep.size(); ++j) {
            const Piece &P = S.pieces[static_cast<size_t>(w.first + keep[j])];
            S.top_pieces.push_back(P);
            const int kj = static_cast<int>(j);
            if (fw.dgroups.empty() || fw.dgroups.back()[0] != P.dims) {
                fw.dgroups.push_back({P.dims, kj, kj + 1, P.bins});
            } else {
                fw.dgroups.back()[2] = kj + 1;
                fw.dgroups.back()[3] = std::max(fw.dgroups.back()[3], P.bins);
            }
        }
        S.top_waves.push_back(fw);
    }
    CK(S.d_top_pieces.ensure(sizeof(Piece) * std::max<size_t>(1, S.top_pieces.size())));
    CK(S.d_top_prefix.ensure(sizeof(long long) * std::max<size_t>(1, S.top_prefix.size())));
    CK(cudaMemcpyAsync(S.d_top_pieces.p, S.top_pieces.data(), sizeof(Piece) * S.top_pieces.size(),
                       cudaMemcpyHostToDevice, main));
    CK(cudaMemcpyAsync(S.d_top_prefix.p, S.top_prefix.data(), sizeof(long long) * S.top_prefix.size(),
                       cudaMemcpyHostToDevice, main));
    CK(cudaMemsetAsync(S.d_rflag.p, 0, sizeof(int), main));
    CK(cudaEventRecord(S.ph_events[ns], main));
    for (int j = 0; j < ns; ++j) CK(cudaStreamWaitEvent(S.ph_streams[j], S.ph_events[ns], 0));
    const int rc = enqueue_waves(ctx, B, S.top_waves, S.d_top_pieces.as<Piece>(), S.d_top_prefix.as<long long>(),
                                 S.top_prefix);
    ctx->stream = main;
    if (rc) return rc;
    for (int j = 0; j < ns; ++j) {
        CK(cudaEventRecord(S.ph_events[j], S.ph_streams[j]));
        CK(cudaStreamWaitEvent(main, S.ph_events[j], 0));
    }
    k_rt_end<<<static_cast<unsigned>(S.tasks.size()), kFoldThreads, 0, main>>>(B);
    LAUNCHED();
    return CHILI_OK;
}

// The iteration's folds, channel-weight update, grid adaptation and counter
// (captured into its own graph when retry rounds may run before it).
int enqueue_final(chili_ctx *ctx, bool adapt);

// The iteration as a stream of launches (captured into the graph); with
// retry tasks only its first round (the final part is a graph of its own).
int enqueue_iteration(chili_ctx *ctx, bool adapt) {
    BatchState &S = *ctx->batch;
    CK(cudaMemsetAsync(S.d_hist.p, 0, sizeof(double) * S.hist_doubles, ctx->stream));
    CK(cudaMemsetAsync(S.d_atrain.p, 0, S.d_atrain.cap, ctx->stream));
    BatchDev B = batch_dev(ctx);
    const cudaStream_t main = ctx->stream;
    if (S.has_retry) {
        CK(cudaMemsetAsync(S.d_rflag.p, 0, sizeof(int), main));
        k_rt_begin<<<static_cast<unsigned>((S.tasks.size() + 127) / 128), 128, 0, main>>>(B);
        LAUNCHED();
    }
    if (S.grouped && !S.waves.empty()) {
        // the waves on their streams beside the camel tasks' evaluation
        const int ns = S.wave_streams;
        CK(cudaEventRecord(S.ph_events[ns], main));
        for (int j = 0; j < ns; ++j) CK(cudaStreamWaitEvent(S.ph_streams[j], S.ph_events[ns], 0));
        k_batch_eval<<<S.grid_blocks, S.block, 0, ctx->stream>>>(B);
        LAUNCHED();
        const int rc = enqueue_waves(ctx, B, S.waves, S.d_pieces.as<Piece>(), S.d_prefix.as<long long>(), S.prefix_host);
        ctx->stream = main;
        if (rc) return rc;
        for (int j = 0; j < ns; ++j) {
            CK(cudaEventRecord(S.ph_events[j], S.ph_streams[j]));
            CK(cudaStreamWaitEvent(main, S.ph_events[j], 0));
        }
        if (S.has_retry) {
            k_rt_end<<<static_cast<unsigned>(S.tasks.size()), kFoldThreads, 0, main>>>(B);
            LAUNCHED();
            return CHILI_OK;
        }
    } else {
    if (!S.ph.empty()) CK(cudaEventRecord(S.ph_events[kPhBranches], main));
    k_batch_eval<<<S.grid_blocks, S.block, 0, ctx->stream>>>(B);
    LAUNCHED();
    }
    if (!S.grouped && !S.ph.empty()) {
        // fork (before the camel tasks' evaluation, which runs beside the
        // branches): each branch runs its phased tasks on its own stream and
        // buffers; join before the folds
        // tasks by decreasing points, each to the branch with the fewest
        // points so far (longest-processing-time order)
        std::vector<int> order;
        for (size_t ti = 0; ti < S.tasks.size(); ++ti)
            if (S.tasks[ti].phased) order.push_back(static_cast<int>(ti));
        std::stable_sort(order.begin(), order.end(),
                         [&](int a, int b) { return S.tasks[a].ncalls > S.tasks[b].ncalls; });
        std::vector<long long> load(kPhBranches, 0);
        std::vector<bool> used(kPhBranches, false);
        for (int ti : order) {
            const int br = static_cast<int>(std::min_element(load.begin(), load.end()) - load.begin());
            load[br] += S.tasks[ti].ncalls;
            if (!used[br]) CK(cudaStreamWaitEvent(S.ph_streams[br], S.ph_events[kPhBranches], 0));
            used[br] = true;
            ctx->stream = S.ph_streams[br];  // the launchers below enqueue on ctx->stream
            const int rc = enqueue_phased_task(ctx, B, ti, S.ph[br]);
            ctx->stream = main;
            if (rc) return rc;
        }
        for (int br = 0; br < kPhBranches; ++br) {
            if (!used[br]) continue;
            CK(cudaEventRecord(S.ph_events[br], S.ph_streams[br]));
            CK(cudaStreamWaitEvent(main, S.ph_events[br], 0));
        }
    }
    return enqueue_final(ctx, adapt);
}

int enqueue_final(chili_ctx *ctx, bool adapt) {
    BatchState &S = *ctx->batch;
    BatchDev B = batch_dev(ctx);
    k_batch_finalize<<<static_cast<unsigned>(S.tasks.size()), kFoldThreads, 0, ctx->stream>>>(B, adapt ? 1 : 0);
    LAUNCHED();
    if (adapt && !S.jobs.empty()) {
        k_batch_adapt<<<static_cast<unsigned>(S.jobs.size()), 32, sizeof(double) * S.max_bins, ctx->stream>>>(
            B, S.d_jobs.as<AdaptJob>(), static_cast<int>(S.jobs.size()), S.d_status.as<int>());
        LAUNCHED();
        k_batch_commit<<<static_cast<unsigned>(S.jobs.size()), 128, 0, ctx->stream>>>(
            B, S.d_jobs.as<AdaptJob>(), static_cast<int>(S.jobs.size()));
        LAUNCHED();
    }
    k_batch_next<<<1, 32, 0, ctx->stream>>>(B);
    LAUNCHED();
    return CHILI_OK;
}

// Block size and points per thread: the fastest evaluation pass among the
// candidates (the evaluation accumulates into buffers that every iteration
// resets; the iteration counter is not advanced).
int autotune(chili_ctx *ctx) {
    BatchState &S = *ctx->batch;
    const int cand[][2] = {{128, 1}, {128, 2}, {256, 1}, {256, 2}, {256, 4}, {128, 4}};
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    float best = 1e30f;
    int bb = 128, bp = 1;
    for (const auto &c : cand) {
        if (int rc = layout_units(ctx, c[0], c[1])) return rc;
        BatchDev B = batch_dev(ctx);
        for (int rep = 0; rep < 2; ++rep) {  // first pass warms up
            CK(cudaMemsetAsync(S.d_counters.p, 0, sizeof(unsigned long long), ctx->stream));
            CK(cudaEventRecord(e0, ctx->stream));
            k_batch_eval<<<S.grid_blocks, S.block, 0, ctx->stream>>>(B);
            LAUNCHED();
            CK(cudaEventRecord(e1, ctx->stream));
            CK(cudaEventSynchronize(e1));
        }
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) {
            best = ms;
            bb = c[0];
            bp = c[1];
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CK(cudaMemsetAsync(S.d_counters.p, 0, sizeof(unsigned long long), ctx->stream));
    return layout_units(ctx, bb, bp);
}

void drop_graphs(BatchState &S) {
    for (cudaGraphExec_t *g : {&S.graph, &S.graph_fin}) {
        if (*g) cudaGraphExecDestroy(*g);
        *g = nullptr;
    }
}

template <class Enqueue>
int capture_one(chili_ctx *ctx, Enqueue enqueue, cudaGraphExec_t *out, unsigned long long *n_launches) {
    const unsigned long long launches = ctx->launches;  // replays are counted, not the capture
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue();
    *n_launches = ctx->launches - launches;
    ctx->launches = launches;
    cudaGraph_t captured = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &captured);
    if (rc) {
        if (captured) cudaGraphDestroy(captured);
        return rc;
    }
    if (e != cudaSuccess) return fail(ctx, CHILI_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    const cudaError_t ei = cudaGraphInstantiate(out, captured, 0);
    cudaGraphDestroy(captured);
    if (ei != cudaSuccess) return fail(ctx, CHILI_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
    return CHILI_OK;
}

// The iteration's graphs: one, or with retry tasks two (the first round;
// the final part; further rounds are launched directly between them).
int capture(chili_ctx *ctx, bool adapt) {
    BatchState &S = *ctx->batch;
    drop_graphs(S);
    if (int rc = capture_one(ctx, [&] { return enqueue_iteration(ctx, adapt); }, &S.graph, &S.graph_launches))
        return rc;
    if (S.has_retry)
        if (int rc = capture_one(ctx, [&] { return enqueue_final(ctx, adapt); }, &S.graph_fin, &S.fin_launches))
            return rc;
    S.graph_adapt = adapt ? 1 : 0;
    return CHILI_OK;
}

int plan_waves(chili_ctx *ctx, const std::vector<PointProgram> &pps);

// Two CUDA events released with their owner (batch_iterate's timing events,
// on its error returns too).
struct EventPair {
    cudaEvent_t a = nullptr, b = nullptr;
    ~EventPair() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};

// Rounds of the retry loop per iteration beyond the first, at most (and at
// most the context's option max_rounds).
constexpr int kMaxRetryRounds = 4096;

// First-round draw of a retry task: ncalls, 1.2 times the points beyond
// them that an iteration had to draw (rejected and NaN points) plus four
// standard deviations of that count, and a margin of ncalls/32 and two
// blocks for rejections that the iteration did not see.
long long retry_draw(long long ncalls, double extra) {
    const double d = static_cast<double>(ncalls) * (1.0 + 1.0 / 32) + 1.2 * extra + 4.0 * std::sqrt(extra) +
                     2.0 * kFwdBlock;
    return static_cast<long long>(std::min(d, static_cast<double>((1ll << 32) - 1)));
}

// Retry tasks whose iteration needed further rounds draw more in the first
// round from now on (the plan grows only).  Re-plans the waves and drops the
// graphs when a draw changed.
int replan_draws(chili_ctx *ctx) {
    BatchState &S = *ctx->batch;
    std::vector<RetryState> R(S.tasks.size());
    CK(cudaMemcpyAsync(R.data(), S.d_retry.p, sizeof(RetryState) * R.size(), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    bool changed = false;
    for (size_t k = 0; k < S.tasks.size(); ++k) {
        BatchTask &T = S.tasks[k];
        if (!T.retry || R[k].rounds <= 1) continue;
        const long long d = retry_draw(T.ncalls, static_cast<double>(R[k].ctr0 - T.ncalls));
        if (d > T.draw) {
            T.draw = d;
            changed = true;
        }
    }
    if (!changed) return CHILI_OK;
    drop_graphs(S);
    if (int rc = plan_waves(ctx, S.pps_host)) return rc;
    return layout_units(ctx, S.block, S.ppt);
}

// Grouped mode: the phased tasks cut into pieces of at most kPieceMax
// points, packed into waves of at most ctx->batch_wave points (pieces of one
// dimension together within a wave), each piece's buffers carved out of one
// arena that every wave reuses (the waves run one after another).
constexpr long long kPieceMax = 1ll << 20;

int plan_waves(chili_ctx *ctx, const std::vector<PointProgram> &pps) {
    BatchState &S = *ctx->batch;
    S.ch_pts = static_cast<int>(ctx->batch_ch_pts);
    // a piece never exceeds a wave (small waves, for tests, cut the tasks finer)
    const long long wave_max = std::max<long long>(ctx->batch_wave / kFwdBlock * kFwdBlock, kFwdBlock);
    const long long piece_max = std::min(kPieceMax, wave_max);
    // pieces, task by task (largest tasks first, so that waves fill evenly)
    std::vector<int> order;
    for (size_t ti = 0; ti < S.tasks.size(); ++ti)
        if (S.tasks[ti].phased) order.push_back(static_cast<int>(ti));
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return S.tasks[a].draw > S.tasks[b].draw; });
    // a task's pieces (of a round's draw), in counter order
    auto task_pieces = [&](int ti) {
        const BatchTask &T = S.tasks[static_cast<size_t>(ti)];
        std::vector<Piece> v;
        for (long long p0 = 0; p0 < T.draw; p0 += piece_max) {
            Piece P{};
            P.ti = ti;
            P.p0 = p0;
            P.mm = std::min(piece_max, T.draw - p0);
            P.ms = (P.mm + kFwdBlock - 1) / kFwdBlock * kFwdBlock;
            P.nb = static_cast<int32_t>(P.ms / kFwdBlock);
            v.push_back(P);
        }
        return v;
    };
    // waves: first fit in that order; the pieces of a retry task all in one
    // wave, adjacent (its cut counts the accepted points of its earlier
    // pieces), a wave grown to the task where the task is larger
    std::vector<std::vector<Piece>> waves;
    std::vector<long long> load;
    auto place = [&](const std::vector<Piece> &v, long long need) {
        size_t w = 0;
        while (w < waves.size() && load[w] > 0 && load[w] + need > wave_max) ++w;
        if (w == waves.size()) {
            waves.emplace_back();
            load.push_back(0);
        }
        for (const Piece &P : v) waves[w].push_back(P);
        load[w] += need;
    };
    for (int ti : order) {
        const std::vector<Piece> v = task_pieces(ti);
        if (S.tasks[static_cast<size_t>(ti)].retry) {
            long long tot = 0;
            for (const Piece &P : v) tot += P.ms;
            place(v, tot);
        } else {
            for (const Piece &P : v) place({P}, P.ms);
        }
    }
    // per piece: constants and buffer sizes
    auto sizes = [&](const Piece &P, const PointProgram &PP, size_t *out) {
        const size_t ms = static_cast<size_t>(P.ms), nb = static_cast<size_t>(P.nb);
        const size_t v[] = {sizeof(double) * 4 * PP.n_ext * ms, sizeof(int32_t) * ms, ms, sizeof(int32_t) * nb,
                            sizeof(long long) * nb, sizeof(RoundCtl), sizeof(int32_t) * ms,
                            sizeof(double) * 4 * PP.n_nodes * ms, sizeof(double) * std::max(1, PP.n_memo) * ms,
                            static_cast<size_t>(std::max(1, PP.n_chains)) * ms, sizeof(double) * PP.nch * ms,
                            sizeof(double) * PP.nch * ms, sizeof(int32_t) * ms, sizeof(double) * ms,
                            sizeof(double) * ms, ms, sizeof(int32_t) * PP.ndims * ms, sizeof(double) * PP.nch * ms};
        for (int q = 0; q < 18; ++q) out[q] = (v[q] + 255) / 256 * 256;
    };
    S.wave_streams = static_cast<int>(std::min<long long>(std::max<long long>(ctx->batch_wave_streams, 1),
                                                          kMaxWaveStreams));
    const int ns = S.wave_streams;
    size_t arena[kMaxWaveStreams] = {256, 256, 256, 256};
    for (size_t wi = 0; wi < waves.size(); ++wi) {
        size_t tot = 0;
        for (const Piece &P : waves[wi]) {
            size_t sz[18];
            sizes(P, pps[static_cast<size_t>(S.tasks[static_cast<size_t>(P.ti)].pp)], sz);
            for (size_t q : sz) tot += q;
        }
        arena[wi % ns] = std::max(arena[wi % ns], tot);
    }
    for (int j = 0; j < ns; ++j) CK(S.d_arena[j].ensure(arena[j]));
    S.pieces.clear();
    S.waves.clear();
    S.prefix_host.clear();
    for (size_t wi = 0; wi < waves.size(); ++wi) {
        auto &w = waves[wi];
        // pieces of one dimension together
        std::stable_sort(w.begin(), w.end(), [&](const Piece &a, const Piece &b) {
            return S.tasks[static_cast<size_t>(a.ti)].dims < S.tasks[static_cast<size_t>(b.ti)].dims;
        });
        BatchState::WaveHost wh;
        wh.sidx = static_cast<int>(wi % ns);
        wh.first = static_cast<int>(S.pieces.size());
        wh.n = static_cast<int>(w.size());
        wh.prefix_off = static_cast<long long>(S.prefix_host.size());
        std::vector<std::vector<long long>> pre(kGroupSteps, std::vector<long long>(w.size() + 1, 0));
        uint8_t *base = S.d_arena[wi % ns].as<uint8_t>();
        size_t off = 0;
        for (size_t k = 0; k < w.size(); ++k) {
            Piece &P = w[k];
            const BatchTask &T = S.tasks[static_cast<size_t>(P.ti)];
            const PointProgram &PP = pps[static_cast<size_t>(T.pp)];
            P.n_items[0] = PP.n_tents;
            P.n_items[1] = PP.n_dws;
            P.n_items[2] = PP.n_sws;
            P.n_chains = PP.n_chains;
            P.nch = PP.nch;
            P.dims = T.dims;
            P.bins = T.bins;
            P.pp = S.d_pps.as<PointProgram>() + T.pp;
            P.grids = S.d_grids.as<double>() + T.grid_off;
            P.hints = S.d_hints.as<uint32_t>() + T.hint_off;
            P.widths = S.d_widths.as<double>() + T.width_off;
            P.sorted = S.d_sorted.as<uint8_t>() + T.sorted_off;
            P.alpha = S.d_alpha.as<double>() + T.ch_off;
            P.f = S.d_descs.as<IntegrandDesc>() + T.desc;
            size_t sz[18];
            sizes(P, PP, sz);
            void *ptr[18];
            for (int q = 0; q < 18; ++q) {
                ptr[q] = base + off;
                off += sz[q];
            }
            P.mom = static_cast<double *>(ptr[0]);
            P.ich = static_cast<int32_t *>(ptr[1]);
            P.flag = static_cast<uint8_t *>(ptr[2]);
            P.bcount = static_cast<int32_t *>(ptr[3]);
            P.boff = static_cast<long long *>(ptr[4]);
            P.ctl = static_cast<RoundCtl *>(ptr[5]);
            P.list = static_cast<int32_t *>(ptr[6]);
            P.node = static_cast<double *>(ptr[7]);
            P.memo = static_cast<double *>(ptr[8]);
            P.cfail = static_cast<uint8_t *>(ptr[9]);
            P.dcv = static_cast<double *>(ptr[10]);
            P.vwv = static_cast<double *>(ptr[11]);
            P.ich_tile = static_cast<int32_t *>(ptr[12]);
            P.val = static_cast<double *>(ptr[13]);
            P.wgt = static_cast<double *>(ptr[14]);
            P.ok = static_cast<uint8_t *>(ptr[15]);
            P.slot = static_cast<int32_t *>(ptr[16]);
            P.dens = static_cast<double *>(ptr[17]);
            const long long gx = (P.ms + 255) / 256, gy = (P.ms + S.ch_pts - 1) / S.ch_pts;
            const long long nblk[kGroupSteps] = {P.nb, P.nb, gx, P.n_items[0] * gx, P.n_items[1] * gx,
                                                 P.n_items[2] * gx, P.n_chains * gx, P.nch * gy, gx, P.nb};
            for (int st = 0; st < kGroupSteps; ++st) pre[static_cast<size_t>(st)][k + 1] = pre[st][k] + nblk[st];
            if (wh.dgroups.empty() || wh.dgroups.back()[0] != P.dims) {
                wh.dgroups.push_back({P.dims, static_cast<int>(k), static_cast<int>(k) + 1, P.bins});
            } else {
                wh.dgroups.back()[2] = static_cast<int>(k) + 1;
                wh.dgroups.back()[3] = std::max(wh.dgroups.back()[3], P.bins);
            }
        }
        for (int st = 0; st < kGroupSteps; ++st) {
            wh.blocks.push_back(pre[static_cast<size_t>(st)][w.size()]);
            if (wh.blocks.back() > 0x7fffffffll) return fail(ctx, CHILI_ERR_LIMIT, "wave too large for one launch");
            S.prefix_host.insert(S.prefix_host.end(), pre[static_cast<size_t>(st)].begin(),
                                 pre[static_cast<size_t>(st)].end());
        }
        for (const Piece &P : w) S.pieces.push_back(P);
        S.waves.push_back(wh);
    }
    CK(S.d_pieces.ensure(sizeof(Piece) * std::max<size_t>(1, S.pieces.size())));
    CK(cudaMemcpyAsync(S.d_pieces.p, S.pieces.data(), sizeof(Piece) * S.pieces.size(), cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(S.d_prefix.ensure(sizeof(long long) * std::max<size_t>(1, S.prefix_host.size())));
    CK(cudaMemcpyAsync(S.d_prefix.p, S.prefix_host.data(), sizeof(long long) * S.prefix_host.size(),
                       cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));  // the host vectors are the copies' sources
    if (S.ph_streams.empty()) {  // the first plan (later ones re-plan the retry tasks' draws)
        for (int j = 0; j < ns; ++j) {
            cudaStream_t st;
            CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            S.ph_streams.push_back(st);
        }
        for (int k = 0; k <= ns; ++k) {
            cudaEvent_t e;
            CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            S.ph_events.push_back(e);
        }
    }
    return CHILI_OK;
}

}  // namespace

void batch_release(chili_ctx *ctx) {
    if (!ctx || !ctx->batch) return;
    BatchState &S = *ctx->batch;
    drop_graphs(S);
    S.d_retry.release();
    S.d_rflag.release();
    S.d_top_pieces.release();
    S.d_top_prefix.release();
    for (DevBuf *b : {&S.d_tasks, &S.d_umap, &S.d_pps, &S.d_progs, &S.d_descs, &S.d_grids, &S.d_grids_new, &S.d_hist,
                      &S.d_hints, &S.d_widths, &S.d_sorted,
                      &S.d_atrain, &S.d_alpha, &S.d_best, &S.d_mindiff, &S.d_cp, &S.d_part, &S.d_stats,
                      &S.d_counters, &S.d_jobs, &S.d_status, &S.d_pieces, &S.d_prefix, &S.d_arena[0],
                      &S.d_arena[1], &S.d_arena[2], &S.d_arena[3]})
        b->release();
    for (auto &b : S.ph)
        for (DevBuf *d : {&b.mom, &b.ich, &b.flag, &b.list, &b.bcount, &b.boff, &b.ctl, &b.node, &b.memo, &b.cfail,
                          &b.dcv, &b.vwv, &b.ich_tile, &b.val, &b.wgt, &b.ok, &b.slot, &b.dens})
            d->release();
    for (cudaStream_t st : S.ph_streams) cudaStreamDestroy(st);
    for (cudaEvent_t e : S.ph_events) cudaEventDestroy(e);
    delete ctx->batch;
    ctx->batch = nullptr;
}

extern "C" {

int chili_gpu_batch_set(chili_ctx *ctx, const chili_task *tasks, int ntasks) {
    if (!ctx || !tasks || ntasks < 1 || ntasks > (1 << 20)) return fail(ctx, CHILI_ERR_INVALID_ARG, "1..2^20 tasks");
    if (int rc = set_device(ctx)) return rc;
    batch_release(ctx);
    ctx->batch = new BatchState();
    BatchState &S = *ctx->batch;
    std::vector<ChannelProgram> progs;
    std::vector<PointProgram> pps;
    std::vector<IntegrandDesc> descs;
    std::vector<double> grids, alpha;
    long long goff = 0, hoff = 0, hnoff = 0, woff = 0, soff = 0;
    for (int k = 0; k < ntasks; ++k) {
        const chili_task &t = tasks[k];
        BatchTask T{};
        T.kind = t.kind;
        T.bins = t.bins;
        T.ncalls = static_cast<long long>(t.ncalls);
        T.draw = T.ncalls;
        T.grid_alpha = t.grid_alpha;
        T.beta = t.beta;
        T.min_alpha = t.min_alpha;
        T.key = 0;
        T.pp = -1;
        IntegrandDesc d{};
        if (t.bins < 2 || t.bins > CHILI_MAX_BINS || t.ncalls < 1 || t.ncalls >= (1ull << 32)) {
            batch_release(ctx);
            return fail(ctx, CHILI_ERR_INVALID_ARG, "task " + std::to_string(k) + ": bins in [2, max], ncalls in [1, 2^32)");
        }
        if (t.kind == CHILI_TASK_CAMEL) {
            if (t.dims < 1 || t.dims > CHILI_MAX_DIMS || t.nparams != 2 + 2 * t.dims || !t.params) {
                batch_release(ctx);
                return fail(ctx, CHILI_ERR_INVALID_ARG, "task " + std::to_string(k) + ": camel needs 2 + 2 dims params");
            }
            T.dims = t.dims;
            T.nch = 1;
            d.kind = CHILI_FUNC_CAMEL;
            d.nparams = t.nparams;
            for (int i = 0; i < t.nparams; ++i) d.p[i] = t.params[i];
            T.ch_off = static_cast<int32_t>(alpha.size());
            alpha.push_back(1.0);
        } else if (t.kind == CHILI_TASK_MULTICHANNEL) {
            std::vector<ChannelProgram> p;
            const std::string why = build_channel_programs(t.descs, t.nch, t.cuts, t.sqrts, t.n_ext, p);
            if (!why.empty()) {
                batch_release(ctx);
                return fail(ctx, CHILI_ERR_INVALID_ARG, "task " + std::to_string(k) + ": " + why);
            }
            const int need = t.fkind == CHILI_FUNC_UNIT ? 0 : 3;
            const bool fk_ok = t.fkind == CHILI_FUNC_UNIT || t.fkind == CHILI_FUNC_PROPAGATOR ||
                               t.fkind == CHILI_FUNC_PROPAGATOR_TOP2;
            const bool pre_ok = t.pre == CHILI_PRE_ACCEPT_ALL || t.pre == CHILI_PRE_FINITE ||
                                (t.pre == CHILI_PRE_CUTS && t.pre_cuts[0] > 0 && t.pre_cuts[1] >= 0 &&
                                 t.pre_cuts[2] >= 0 && t.pre_cuts[3] >= 0);
            if (!fk_ok || !pre_ok || t.nch > kBatchMaxCh || t.nparams < need ||
                t.nparams > CHILI_MAX_INTEGRAND_PARAMS || (t.nparams > 0 && !t.params)) {
                batch_release(ctx);
                return fail(ctx, CHILI_ERR_INVALID_ARG,
                            "task " + std::to_string(k) +
                                ": phase-space integrand kind and parameters, preprocess kind and cut values, "
                                "at most 64 channels");
            }
            T.dims = p[0].ndims;
            T.nch = t.nch;
            // the shared-entry form of the channel weights when the set fits
            pps.emplace_back();
            if (build_point_program(p, pps.back())) T.pp = static_cast<int32_t>(pps.size() - 1);
            else pps.pop_back();
            // weighted by the phased pass when its kernels cover the set
            T.phased = (T.pp >= 0 && ctx->batch_phased && pipeline_dims_ok(T.dims)) ? 1 : 0;
            T.ch_off = static_cast<int32_t>(alpha.size());
            for (int c = 0; c < t.nch; ++c) alpha.push_back(1.0 / t.nch);
            for (auto &q : p) progs.push_back(q);
            d.kind = t.fkind;
            d.nparams = t.nparams;
            for (int i = 0; i < t.nparams; ++i) d.p[i] = t.params[i];
            d.pre = t.pre;
            d.n_ext = t.n_ext;
            for (int i = 0; i < 4; ++i) d.cut[i] = t.pre == CHILI_PRE_CUTS ? t.pre_cuts[i] : 0.0;
        } else {
            batch_release(ctx);
            return fail(ctx, CHILI_ERR_INVALID_ARG, "task " + std::to_string(k) + ": unknown kind");
        }
        if (t.kind == CHILI_TASK_CAMEL) {
            // an unused program keeps programs and channel slots on one index
            progs.emplace_back();
            std::memset(&progs.back(), 0, sizeof(ChannelProgram));
        }
        T.desc = static_cast<int32_t>(descs.size());
        descs.push_back(d);
        T.before = edge_before_table(T.dims, T.bins);
        T.grid_off = goff;
        T.hist_off = hoff;
        T.hint_off = hnoff;
        T.width_off = woff;
        T.sorted_off = soff;
        hnoff += static_cast<long long>(T.nch) * T.dims * kHintPerBin * T.bins;
        woff += static_cast<long long>(T.nch) * T.dims * T.bins;
        soff += static_cast<long long>(T.nch) * T.dims;
        const long long per = static_cast<long long>(T.dims) * (T.bins + 1);
        for (int c = 0; c < T.nch; ++c)
            for (int dd = 0; dd < T.dims; ++dd)
                for (int b = 0; b <= T.bins; ++b) grids.push_back(static_cast<double>(b) / T.bins);
        goff += per * T.nch;
        hoff += static_cast<long long>(T.dims) * T.bins * T.nch;
        S.max_bins = std::max(S.max_bins, T.bins);
        for (int c = 0; c < T.nch; ++c)
            for (int dd = 0; dd < T.dims; ++dd) S.jobs.push_back(AdaptJob{k, c, dd, 0});
        S.tasks.push_back(T);
        S.total_points += T.ncalls;
    }
    const size_t nslot = alpha.size();
    S.hist_doubles = static_cast<size_t>(hoff);
    {
        // one tile of the phased tasks: up to 2^18 points; per branch,
        // buffers for the largest point program among them
        long long tile = 0;
        int ne = 1, nn = 1, nmemo = 1, nchain = 1, nch = 1, dims = 1;
        for (const auto &T : S.tasks) {
            if (!T.phased) continue;
            const PointProgram &P = pps[static_cast<size_t>(T.pp)];
            tile = std::max(tile, (T.ncalls + kFwdBlock - 1) / kFwdBlock * kFwdBlock);
            ne = std::max(ne, P.n_ext);
            nn = std::max(nn, P.n_nodes);
            nmemo = std::max(nmemo, P.n_memo);
            nchain = std::max(nchain, P.n_chains);
            nch = std::max(nch, P.nch);
            dims = std::max(dims, P.ndims);
        }
        S.ph_tile = std::min<long long>(tile, 1ll << 18);
        const size_t T = static_cast<size_t>(std::max<long long>(S.ph_tile, kFwdBlock));
        const size_t nb = T / kFwdBlock;
        S.grouped = ctx->batch_grouped && S.ph_tile > 0;  // waves planned once the device tables exist
        // the reference's retry loop: multichannel tasks weighted in the waves
        if (ctx->batch_retry) {
            for (auto &Tk : S.tasks) {
                if (Tk.kind != CHILI_TASK_MULTICHANNEL) continue;
                if (!Tk.phased || !S.grouped) {
                    batch_release(ctx);
                    return fail(ctx, CHILI_ERR_INVALID_ARG,
                                "the retry loop (option batch_retry) runs in the grouped phased pass: options "
                                "batch_grouped and batch_phased on, or batch_retry 0 for a fixed budget");
                }
                Tk.retry = 1;
                Tk.draw = retry_draw(Tk.ncalls, 0.0);
                S.has_retry = true;
            }
        }
        if (!S.grouped && S.ph_tile > 0) {
            S.ph.resize(kPhBranches);
            for (auto &b : S.ph) {
                CK(b.mom.ensure(sizeof(double) * 4 * ne * T));
                CK(b.ich.ensure(sizeof(int32_t) * T));
                CK(b.flag.ensure(T));
                CK(b.list.ensure(sizeof(int32_t) * T));
                CK(b.bcount.ensure(sizeof(int32_t) * nb));
                CK(b.boff.ensure(sizeof(long long) * nb));
                CK(b.ctl.ensure(sizeof(RoundCtl)));
                CK(b.node.ensure(sizeof(double) * 4 * nn * T));
                CK(b.memo.ensure(sizeof(double) * nmemo * T));
                CK(b.cfail.ensure(static_cast<size_t>(nchain) * T));
                CK(b.dcv.ensure(sizeof(double) * nch * T));
                CK(b.vwv.ensure(sizeof(double) * nch * T));
                CK(b.ich_tile.ensure(sizeof(int32_t) * T));
                CK(b.val.ensure(sizeof(double) * T));
                CK(b.wgt.ensure(sizeof(double) * T));
                CK(b.ok.ensure(T));
                CK(b.slot.ensure(sizeof(int32_t) * dims * T));
                CK(b.dens.ensure(sizeof(double) * nch * T));
            }
            for (int k = 0; k < kPhBranches; ++k) {
                cudaStream_t st;
                CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
                S.ph_streams.push_back(st);
            }
            for (int k = 0; k <= kPhBranches; ++k) {
                cudaEvent_t e;
                CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
                S.ph_events.push_back(e);
            }
        }
    }
    S.pps_host = pps;
    CK(S.d_progs.ensure(sizeof(ChannelProgram) * progs.size()));
    CK(cudaMemcpyAsync(S.d_progs.p, progs.data(), sizeof(ChannelProgram) * progs.size(), cudaMemcpyHostToDevice,
                       ctx->stream));
    if (!pps.empty()) {
        CK(S.d_pps.ensure(sizeof(PointProgram) * pps.size()));
        CK(cudaMemcpyAsync(S.d_pps.p, pps.data(), sizeof(PointProgram) * pps.size(), cudaMemcpyHostToDevice,
                           ctx->stream));
        k_batch_pp_prepare<<<static_cast<unsigned>(pps.size()), PP_MAX_DWS, 0, ctx->stream>>>(
            S.d_pps.as<PointProgram>());
        LAUNCHED();
    }
    CK(S.d_descs.ensure(sizeof(IntegrandDesc) * descs.size()));
    CK(cudaMemcpyAsync(S.d_descs.p, descs.data(), sizeof(IntegrandDesc) * descs.size(), cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(S.d_grids.ensure(sizeof(double) * grids.size()));
    CK(S.d_grids_new.ensure(sizeof(double) * grids.size()));
    CK(cudaMemcpyAsync(S.d_grids.p, grids.data(), sizeof(double) * grids.size(), cudaMemcpyHostToDevice, ctx->stream));
    CK(S.d_hints.ensure(sizeof(uint32_t) * std::max<long long>(hnoff, 1)));
    CK(S.d_widths.ensure(sizeof(double) * std::max<long long>(woff, 1)));
    CK(S.d_sorted.ensure(std::max<long long>(soff, 1)));
    CK(S.d_hist.ensure(sizeof(double) * std::max<size_t>(S.hist_doubles, 1)));
    CK(S.d_atrain.ensure(sizeof(double) * nslot));
    CK(S.d_alpha.ensure(sizeof(double) * nslot));
    CK(cudaMemcpyAsync(S.d_alpha.p, alpha.data(), sizeof(double) * nslot, cudaMemcpyHostToDevice, ctx->stream));
    std::vector<double> nanv(nslot, NAN), inf(ntasks, INFINITY);
    CK(S.d_best.ensure(sizeof(double) * nslot));
    CK(cudaMemcpyAsync(S.d_best.p, nanv.data(), sizeof(double) * nslot, cudaMemcpyHostToDevice, ctx->stream));
    CK(S.d_mindiff.ensure(sizeof(double) * ntasks));
    CK(cudaMemcpyAsync(S.d_mindiff.p, inf.data(), sizeof(double) * ntasks, cudaMemcpyHostToDevice, ctx->stream));
    CK(S.d_cp.ensure(sizeof(double) * nslot));
    // the channel-selection table of the initial weights, in the order of
    // operations of alpha_update
    std::vector<double> cp(nslot, 1.0);
    for (const auto &T : S.tasks) {
        if (T.nch < 2) continue;
        double sa = 0, c = 0;
        for (int i = 0; i < T.nch; ++i) sa += alpha[T.ch_off + i];
        for (int i = 0; i < T.nch; ++i) {
            const double p = alpha[T.ch_off + i] / sa;
            c = (i == 0) ? p : c + p;
            cp[T.ch_off + i] = c;
        }
        cp[T.ch_off + T.nch - 1] = 1.0;
    }
    CK(cudaMemcpyAsync(S.d_cp.p, cp.data(), sizeof(double) * nslot, cudaMemcpyHostToDevice, ctx->stream));
    CK(S.d_counters.ensure(sizeof(unsigned long long) * 2));
    CK(cudaMemsetAsync(S.d_counters.p, 0, sizeof(unsigned long long) * 2, ctx->stream));
    CK(S.d_jobs.ensure(sizeof(AdaptJob) * std::max<size_t>(S.jobs.size(), 1)));
    CK(cudaMemcpyAsync(S.d_jobs.p, S.jobs.data(), sizeof(AdaptJob) * S.jobs.size(), cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(S.d_status.ensure(sizeof(int)));
    CK(cudaMemsetAsync(S.d_status.p, 0, sizeof(int), ctx->stream));
    CK(S.d_retry.ensure(sizeof(RetryState) * S.tasks.size()));
    CK(cudaMemsetAsync(S.d_retry.p, 0, sizeof(RetryState) * S.tasks.size(), ctx->stream));
    CK(S.d_rflag.ensure(sizeof(int)));
    CK(cudaMemsetAsync(S.d_rflag.p, 0, sizeof(int), ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (S.grouped)
        if (int rc = plan_waves(ctx, pps)) return rc;
    if (int rc = layout_units(ctx, 256, 1)) return rc;
    // the bin-search tables of the initial grids (k_batch_commit keeps them
    // current after every adaptation)
    if (!S.jobs.empty()) {
        k_batch_hints<<<static_cast<unsigned>(S.jobs.size()), 128, 0, ctx->stream>>>(
            batch_dev(ctx), S.d_jobs.as<AdaptJob>(), static_cast<int>(S.jobs.size()));
        LAUNCHED();
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return CHILI_OK;
}

int chili_gpu_batch_iterate(chili_ctx *ctx, int iterations, uint64_t seed, int adapt, chili_stats *stats,
                            chili_batch_info *info) {
    if (!ctx || iterations < 1 || iterations > 100000) return fail(ctx, CHILI_ERR_INVALID_ARG, "iterations in [1, 1e5]");
    if (int rc = need_batch(ctx)) return rc;
    if (int rc = set_device(ctx)) return rc;
    BatchState &S = *ctx->batch;
    const int nt = static_cast<int>(S.tasks.size());
    // Philox key of task k: seed + k (the task's own stream)
    bool keys_changed = false;
    for (int k = 0; k < nt; ++k) {
        const uint64_t key = seed + static_cast<uint64_t>(k);
        keys_changed = keys_changed || S.tasks[k].key != key;
        S.tasks[k].key = key;
    }
    if (keys_changed) {
        CK(cudaMemcpyAsync(S.d_tasks.p, S.tasks.data(), sizeof(BatchTask) * nt, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    if (!S.tuned) {
        if (int rc = autotune(ctx)) return rc;
        S.tuned = true;
    }
    if (S.nslots_alloc < iterations) {
        CK(S.d_stats.ensure(sizeof(double) * 6 * static_cast<size_t>(iterations) * nt));
        S.nslots_alloc = iterations;
        drop_graphs(S);
    }
    if (!S.graph || S.graph_adapt != (adapt ? 1 : 0))
        if (int rc = capture(ctx, adapt != 0)) return rc;
    unsigned long long iter0 = 0;
    CK(cudaMemcpyAsync(&iter0, S.d_counters.as<unsigned long long>() + 1, sizeof(iter0), cudaMemcpyDeviceToHost,
                       ctx->stream));
    EventPair ev;  // destroyed on every return
    CK(cudaEventCreate(&ev.a));
    CK(cudaEventCreate(&ev.b));
    CK(cudaEventRecord(ev.a, ctx->stream));
    S.retry_rounds = 0;
    for (int it = 0; it < iterations; ++it) {
        if (!S.graph)  // dropped by a re-plan of the retry tasks' draws
            if (int rc = capture(ctx, adapt != 0)) return rc;
        CK(cudaGraphLaunch(S.graph, ctx->stream));
        ctx->launches += S.graph_launches;
        if (!S.has_retry) continue;
        // further rounds while a task is short of ncalls (one flag read per round)
        int flag = 0, rounds = 0;
        CK(cudaMemcpyAsync(&flag, S.d_rflag.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        const long long max_rounds = std::min<long long>(kMaxRetryRounds, ctx->max_rounds);
        while (flag == 1 && rounds < max_rounds) {
            if (int rc = run_retry_round(ctx)) return rc;
            ++rounds;
            CK(cudaMemcpyAsync(&flag, S.d_rflag.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
        }
        if (flag != 0) {
            // the first task still short of ncalls, for the message
            std::vector<RetryState> R(S.tasks.size());
            CK(cudaMemcpy(R.data(), S.d_retry.p, sizeof(RetryState) * R.size(), cudaMemcpyDeviceToHost));
            std::string who;
            for (size_t k = 0; k < R.size() && who.empty(); ++k)
                if (S.tasks[k].retry && R[k].need > 0)
                    who = ": task " + std::to_string(k) + " still needs " + std::to_string(R[k].need) + " of " +
                          std::to_string(S.tasks[k].ncalls) + " after " + std::to_string(R[k].ctr0) +
                          " points counted in " + std::to_string(R[k].rounds) + " rounds (" +
                          std::to_string(R[k].nan_total) + " NaN values)";
            // the reference's loop never ends on a task whose every point is
            // rejected or NaN; this one gives up like the single-integrand path
            return fail(ctx, flag == 2 ? CHILI_ERR_LIMIT : CHILI_ERR_TIMEOUT,
                        std::string(flag == 2 ? "retry loop: a task's counters ran out (2^32 per iteration)"
                                              : "retry loop: too many rounds") + who);
        }
        CK(cudaGraphLaunch(S.graph_fin, ctx->stream));
        ctx->launches += S.fin_launches;
        S.retry_rounds += static_cast<unsigned long long>(rounds);
        if (rounds > 0)
            if (int rc = replan_draws(ctx)) return rc;
    }
    CK(cudaEventRecord(ev.b, ctx->stream));
    CK(cudaEventSynchronize(ev.b));
    float ms = 0;
    cudaEventElapsedTime(&ms, ev.a, ev.b);
    S.last_ms = ms / iterations;
    if (stats) {
        std::vector<double> all(6 * static_cast<size_t>(S.nslots_alloc) * nt);
        CK(cudaMemcpy(all.data(), S.d_stats.p, sizeof(double) * all.size(), cudaMemcpyDeviceToHost));
        for (int it = 0; it < iterations; ++it) {
            const uint64_t slot = (iter0 + it) % static_cast<uint64_t>(S.nslots_alloc);
            for (int k = 0; k < nt; ++k) {
                const double *o = all.data() + (slot * nt + k) * 6;
                chili_stats &s = stats[static_cast<size_t>(it) * nt + k];
                s.n = o[0]; s.min = o[1]; s.max = o[2]; s.sum = o[3]; s.sum2 = o[4]; s.n_finite = o[5];
            }
        }
    }
    if (info) {
        info->block = static_cast<uint32_t>(S.block);
        info->points_per_thread = static_cast<uint32_t>(S.ppt);
        info->ms_per_iteration = S.last_ms;
        info->units = static_cast<uint64_t>(S.nunits);
        info->points = static_cast<uint64_t>(S.total_points);
        info->retry_rounds = S.retry_rounds;
    }
    return CHILI_OK;
}

int chili_gpu_batch_get_grid(chili_ctx *ctx, int task, double *edges, double *alpha) {
    if (!ctx) return fail(ctx, CHILI_ERR_INVALID_ARG, "NULL argument");
    if (int rc = need_batch(ctx)) return rc;
    BatchState &S = *ctx->batch;
    if (task < 0 || task >= static_cast<int>(S.tasks.size())) return fail(ctx, CHILI_ERR_INVALID_ARG, "task index");
    const BatchTask &T = S.tasks[task];
    const size_t n = static_cast<size_t>(T.nch) * T.dims * (T.bins + 1);
    if (edges) CK(cudaMemcpy(edges, S.d_grids.as<double>() + T.grid_off, sizeof(double) * n, cudaMemcpyDeviceToHost));
    if (alpha) CK(cudaMemcpy(alpha, S.d_alpha.as<double>() + T.ch_off, sizeof(double) * T.nch, cudaMemcpyDeviceToHost));
    return CHILI_OK;
}

}  // extern "C"
