// context.h -- the device context behind the C ABI and the host helpers
// shared by the translation units that implement it (chili_gpu.cu: VEGAS,
// FSMapper and multichannel entry points; flow.cu: the learned proposal).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <functional>
#include <initializer_list>
#include <string>
#include <vector>

#include "chili_gpu.h"
#include "channel_program.h"
#include "mc_device.cuh"

using namespace chili_dev;

// Text of the last error of any context on this host thread.
inline thread_local std::string g_last_error;


namespace {


// A growable device buffer.
struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap) return cudaSuccess;
        if (p) {
            cudaError_t e = cudaFree(p);
            if (e != cudaSuccess) return e;
            p = nullptr;
            cap = 0;
        }
        const size_t want = std::max<size_t>(bytes, 256);
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
};

constexpr int kStageSlots = 6;

}  // namespace

struct FlowState;
struct BatchState;
struct chili_ctx;
// Frees the learned proposal's state (flow.cu).
void flow_release(chili_ctx *ctx);
// Frees the batched integrands' state (batch.cu).
void batch_release(chili_ctx *ctx);
// Launches the last step of one tile of the phased weight pass (base = first
// listed point of the tile, T = tile capacity).
using TileFn = std::function<int(long long base, long long T)>;
// The phased weight pass (chili_gpu.cu) over listed points of a momenta
// buffer [slot][component][m]; rec_dens may be null.
// fused (optional): the standard combine step's outputs; when given (and the
// "pipeline_fuse" option is on) the combine runs inside the channel kernel
// and `combine` is not called.
struct PPFusedOut {
    double *rec_val, *rec_wgt;
    uint8_t *rec_ok;
};
int pipeline_run(chili_ctx *ctx, const double *mom_soa, long long m, const int32_t *list, const int32_t *ich,
                 const long long *n_list, long long n_pre, int bins, bool opt, int32_t *rec_slot, double *rec_dens,
                 const TileFn &combine, const PPFusedOut *fused = nullptr);

// One phased weight pass with explicit buffers and no host round trip (so
// that a graph can capture it; chili_gpu.cu): T launch points, of which the
// first *n_list are listed; tile-local buffers with stride T, records with
// stride mr; hints, sorted and widths may be null (plain bin search).
struct PPPass {
    const PointProgram *pp;       // device
    const PointProgram *pp_host;  // host copy: launch sizes
    const double *mom_soa;        // [slot][component][mc]
    long long mc;
    const int32_t *list, *ich;
    const long long *n_list;
    long long T, mr;
    int bins;
    const double *grids;
    const uint32_t *hints;
    const uint8_t *sorted;
    const double *widths;
    double *node_soa, *memo, *dcv, *vwv;
    uint8_t *cfail;
    int32_t *ich_tile, *rec_slot;
    double *rec_dens;
    const double *alpha;
    const IntegrandDesc *f;
    double *rec_val, *rec_wgt;
    uint8_t *rec_ok;
};
int pp_pass_launch(chili_ctx *ctx, const PPPass &a);
// The ordered list of flagged points of m (per-block counts of kFwdBlock
// points in block_count): offsets, ctl->n_acc and list (chili_gpu.cu).
int compact_launch(chili_ctx *ctx, const int32_t *block_count, int nb, const uint8_t *flag, long long m,
                   long long *block_off, RoundCtl *ctl, int32_t *list);
// Whether the phased weight kernels are built for this many dimensions.
bool pipeline_dims_ok(int d);

struct chili_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;      // uploads of host uniforms, overlapped with the forward pass
    std::vector<cudaEvent_t> copy_events;
    bool own_stream = false;
    std::string err;
    unsigned long long launches = 0;

    // grids
    int g_nch = 0, dims = 0, bins = 0;
    DevBuf edges, edges_tmp;
    // channels
    int nch = 0, n_ext = 0, ndims = 0;
    double sqrts = 0;
    DevBuf progs;
    DevBuf point_prog;         // PointProgram of the channel set, when it fits
    bool have_pp = false;      // the set fits the PointProgram limits
    bool use_pp = true;        // option "point_program"
    bool use_pipeline = true;  // option "pipeline": phased weight pass
    bool fuse_combine = false;  // option "pipeline_fuse": combine step inside the channel kernel (slower: off)
    long long gen_ppt = 2;       // option "vegas_gen_ppt": points per thread of chili_gpu_vegas_generate
    bool vegas_fused = true;     // option "vegas_fused": a whole adapting Vegas iteration in one launch
    bool hints_stale = false;    // the grids changed since the hint tables were built
    bool defer_train = false;  // option "defer_train": iterations collect training data, Train is the caller's
    bool batch_phased = true;  // option "batch_phased": batched multichannel tasks by the phased weight pass
    bool batch_grouped = true;  // option "batch_grouped": the phased tasks in waves, one launch per step and wave
    bool batch_retry = false;   // option "batch_retry": batched multichannel tasks keep the reference's retry loop
    long long batch_wave = 1ll << 24;  // option "batch_wave_points": points per wave of the grouped mode
    long long batch_ch_pts = 2048;  // option "batch_channel_points": points per block of the grouped channel step
    long long upload_slice = 1ll << 19;  // option "upload_slice": largest host-uniform slice (rows)
    bool pipe_sync = true;       // option "pipeline_sync": size the phased pass by the accepted count read back
    bool hist_shared = true;     // option "hist_shared": the iteration's histogram adds staged in shared memory
    bool channel_tables = true;  // option "channel_tables": k_pp_channel (and the batch's k_g_channel) with the
                                 // channel's tables in shared memory
    bool flow_streamed = false;  // option "flow_streamed": streamed-weight coupling kernels even at 2 x 128
    long long batch_wave_streams = 3;  // option "batch_wave_streams": streams the waves alternate over (1..4)
    long long pipe_tile = 1 << 22;  // option "pipeline_tile": points per tile
    long long max_rounds = 100000;  // option "max_rounds": chunks an iteration may take before CHILI_ERR_TIMEOUT
    PointProgram pp_host;      // host copy (sizes of the memo buffers)
    DevBuf node_soa, memo, cfail, dcv, vwv;
    DevBuf arrivals;  // per point block of a tile: the fused combine's arrival counters (zero between launches)
    DevBuf v_arrive;  // the fused Vegas iteration's arrival counter (zero between launches)
    DevBuf hints, sorted, widths;  // hinted bin search tables and bin widths of the grids
    DevBuf ich_tile;
    // channel weights: alpha[CH], best[CH], cp[CH], min_diff
    DevBuf alpha_buf;
    bool alpha_set = false;
    // integrand
    IntegrandDesc f_host{};
    DevBuf f_dev;
    bool f_set = false;
    // multichannel iteration scratch
    DevBuf mom_soa, ich, flag, list, block_count, block_off, part, hist, round_res, acc, ctl, status;
    // host-uniform rounds: the forward pass of the next round runs on its own
    // stream beside this round's weight pass, into the other set of buffers
    DevBuf mom_soa_alt, ich_alt, flag_alt, block_count_alt;
    cudaStream_t fwd_stream = nullptr;
    cudaEvent_t fwd_done[2] = {nullptr, nullptr}, round_done[2] = {nullptr, nullptr};
    RoundCtl *ctl_host = nullptr;  // pinned, two records: the round, the PreProcess count
    long long *iter_host = nullptr;  // pinned, the queued rounds' state (k_iter_init)
    DevBuf iter_ctl;                 // device copy of that state
    double accept_rate = 0.5, nan_rate = 0.0;
    DevBuf rec, ctl3;
    DevBuf unw;  // unweighting: keep flags, kept list, partials, round control
    // plain VEGAS scratch
    DevBuf v_part, v_hist, v_train, v_out;
    // staging of host buffers
    DevBuf stage[kStageSlots];
    int max_smem_optin = 0;
    int sms = 148;  // streaming multiprocessors of the device
    // option "kernel_timing": CUDA events around the iteration's kernels
    bool timing = false;
    struct Pending {
        int kernel;
        cudaEvent_t a, b;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> event_pool;
    double ktime_ms[32] = {0};
    unsigned long long klaunches[32] = {0};
    // channel descriptions as given (checkpoint.cu writes them back) and the
    // FSMapper ptmin list of every channel (Channel.hh:20-26)
    std::vector<std::vector<chili_particle_info>> ch_info;
    std::vector<std::vector<chili_decay>> ch_decays;
    std::vector<std::vector<double>> ch_ptmin;
    // MultiChannelSummary::best_weights as last loaded (written back unchanged)
    std::vector<double> summary_best;
    // learned proposal (flow.cu)
    FlowState *flow = nullptr;
    BatchState *batch = nullptr;
};

namespace {


// Kernel classes timed under the "kernel_timing" option.
const char *const kTimedKernels[] = {"k_mc_forward", "k_pp_nodes", "k_pp_items", "k_pp_chains", "k_pp_channel",
                                     "k_pp_combine", "k_mc_weight", "k_mc_accum", "k_vegas_iter", "k_flow_layer",
                                     "k_flow_layer_bwd", "k_flow_wgrad", "k_alpha_train", "k_flow_phys",
                                     "k_flow_batch", "k_vegas_generate", "k_vegas_step", "round_other",
                                     "iteration_end", "k_alpha_eval", nullptr};
// round_other: the small kernels of a multichannel round (offsets, compaction,
// the cut, the per-round folds); iteration_end: the channel-weight and grid
// adaptation after the last round.
enum { KT_FORWARD, KT_NODES, KT_ITEMS, KT_CHAINS, KT_CHANNEL, KT_COMBINE, KT_WEIGHT, KT_ACCUM, KT_VEGAS,
       KT_FLOW_LAYER, KT_FLOW_BWD, KT_FLOW_WGRAD, KT_ALPHA_TRAIN, KT_FLOW_PHYS, KT_FLOW_BATCH, KT_VEGAS_GEN,
       KT_VEGAS_STEP, KT_ROUND_OTHER, KT_ITER_END, KT_ALPHA_EVAL };

cudaEvent_t take_event(chili_ctx *ctx) {
    if (!ctx->event_pool.empty()) {
        cudaEvent_t e = ctx->event_pool.back();
        ctx->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Brackets one launch with events when timing is on.
struct KTimer {
    chili_ctx *ctx;
    int kernel;
    cudaEvent_t a = nullptr;
    KTimer(chili_ctx *c, int k) : ctx(c), kernel(k) {
        if (ctx->timing) {
            a = take_event(ctx);
            cudaEventRecord(a, ctx->stream);
        }
    }
    ~KTimer() {
        if (ctx->timing && a) {
            cudaEvent_t b = take_event(ctx);
            cudaEventRecord(b, ctx->stream);
            ctx->pending.push_back({kernel, a, b});
        }
    }
};

// Folds the recorded intervals into the totals (the stream must be idle).
void collect_times(chili_ctx *ctx) {
    for (auto &p : ctx->pending) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
            ctx->ktime_ms[p.kernel] += ms;
            ctx->klaunches[p.kernel] += 1;
        }
        ctx->event_pool.push_back(p.a);
        ctx->event_pool.push_back(p.b);
    }
    ctx->pending.clear();
    cudaGetLastError();
}

int fail(chili_ctx *ctx, int code, const std::string &msg) {
    if (ctx) ctx->err = msg;
    g_last_error = msg;
    return code;
}

#define CK(call)                                                                                  \
    do {                                                                                          \
        const cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                                    \
            return fail(ctx, CHILI_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define LAUNCHED()                                                                                     \
    do {                                                                                               \
        ++ctx->launches;                                                                               \
        const cudaError_t e_ = cudaGetLastError();                                                     \
        if (e_ != cudaSuccess) return fail(ctx, CHILI_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e_)); \
    } while (0)

bool is_device_ptr(const void *p) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Resolves a caller buffer to a device pointer: device buffers pass through,
// host buffers are staged in slot `slot` (copied in when `in`).
struct Arg {
    void *dev = nullptr;
    void *host = nullptr;
    size_t bytes = 0;
};

int resolve(chili_ctx *ctx, const void *p, size_t bytes, int slot, bool in, Arg &a) {
    a = Arg{};
    a.bytes = bytes;
    if (!p) return CHILI_OK;
    if (is_device_ptr(p)) {
        a.dev = const_cast<void *>(p);
        return CHILI_OK;
    }
    CK(ctx->stage[slot].ensure(bytes));
    a.dev = ctx->stage[slot].p;
    a.host = const_cast<void *>(p);
    if (in && bytes) CK(cudaMemcpyAsync(a.dev, p, bytes, cudaMemcpyHostToDevice, ctx->stream));
    return CHILI_OK;
}

int finish_out(chili_ctx *ctx, const Arg &a) {
    if (a.host && a.bytes) CK(cudaMemcpyAsync(a.host, a.dev, a.bytes, cudaMemcpyDeviceToHost, ctx->stream));
    return CHILI_OK;
}

int sync_if_host(chili_ctx *ctx, std::initializer_list<const Arg *> args) {
    for (const Arg *a : args)
        if (a->host) {
            CK(cudaStreamSynchronize(ctx->stream));
            return CHILI_OK;
        }
    return CHILI_OK;
}

unsigned grid_for(long long n, int block) { return static_cast<unsigned>((n + block - 1) / block); }

double *alpha_ptr(chili_ctx *ctx) { return ctx->alpha_buf.as<double>(); }
double *best_ptr(chili_ctx *ctx) { return ctx->alpha_buf.as<double>() + CHILI_MAX_CHANNELS; }
double *cp_ptr(chili_ctx *ctx) { return ctx->alpha_buf.as<double>() + 2 * CHILI_MAX_CHANNELS; }
double *mindiff_ptr(chili_ctx *ctx) { return ctx->alpha_buf.as<double>() + 3 * CHILI_MAX_CHANNELS; }
const PointProgram *pp_ptr(chili_ctx *ctx) {
    return (ctx->have_pp && ctx->use_pp) ? ctx->point_prog.as<PointProgram>() : nullptr;
}
double *acc_train_ptr(chili_ctx *ctx) {
    return reinterpret_cast<double *>(static_cast<char *>(ctx->acc.p) + offsetof(IterAcc, atrain));
}

int need_grids(chili_ctx *ctx) {
    if (!ctx->edges.p || ctx->g_nch <= 0) return fail(ctx, CHILI_ERR_STATE, "no grids set");
    return CHILI_OK;
}
int need_channels(chili_ctx *ctx) {
    if (!ctx->progs.p || ctx->nch <= 0) return fail(ctx, CHILI_ERR_STATE, "no channels set");
    return CHILI_OK;
}

int set_device(chili_ctx *ctx) {
    CK(cudaSetDevice(ctx->device));
    return CHILI_OK;
}

}  // namespace
