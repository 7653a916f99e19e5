// chili_gpu.cu -- implementation of the C ABI declared in include/chili_gpu.h.
//
// One context = one device, one stream, one grid set, one channel set, one
// integrand.  Host-side work is limited to argument checks, staging of host
// buffers, kernel launches and, in a multichannel iteration, reading a 32-byte
// round record to decide whether another round of points is needed.
#include <cuda_runtime.h>
#include <math_constants.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "chili_gpu.h"
#include "channel_program.h"
#include "kernels.cuh"
#include "pipeline.cuh"
#include "context.h"

using namespace chili_dev;

bool pipeline_dims_ok(int d) {
    switch (d) {
    case 1: case 4: case 7: case 10: case 13: case 16: case 19: case 22: return true;
    default: return false;
    }
}

namespace {

int rebuild_hints(chili_ctx *ctx);

// Largest table (one channel's edges, widths, hints) staged in shared memory
// by k_pp_channel_tab; larger channel tables take k_pp_channel.
constexpr size_t kMaxChannelTab = 112 * 1024;

template <int D>
void launch_channel(chili_ctx *ctx, long long base, long long T, long long mr, int bins, int opt,
                    const long long *n_list, int32_t *rec_slot, double *rec_dens, const PPCombine *fuse) {
    const dim3 grid(ctx->nch, static_cast<unsigned>((T + 127) / 128));
    if (fuse) {
        k_pp_channel<D, true, true><<<grid, 128, 0, ctx->stream>>>(
            ctx->point_prog.as<PointProgram>(), ctx->edges.as<double>(), ctx->hints.as<uint32_t>(),
            ctx->sorted.as<uint8_t>(), ctx->widths.as<double>(), bins, ctx->memo.as<double>(),
            ctx->cfail.as<uint8_t>(), ctx->ich_tile.as<int32_t>(), n_list, base, T, mr, opt, ctx->dcv.as<double>(),
            ctx->vwv.as<double>(), rec_slot, rec_dens, *fuse);
        return;
    }
    const size_t tab = channel_tab_bytes(D, bins);
    if (ctx->channel_tables && tab <= kMaxChannelTab) {
        static size_t attr = 0;  // dynamic shared memory granted so far
        if (tab > attr) {
            cudaFuncSetAttribute(k_pp_channel_tab<D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kMaxChannelTab));
            attr = kMaxChannelTab;
        }
        const dim3 gt(ctx->nch, static_cast<unsigned>((T + kTabPoints - 1) / kTabPoints));
        k_pp_channel_tab<D><<<gt, kTabThreads, tab, ctx->stream>>>(
            ctx->point_prog.as<PointProgram>(), ctx->edges.as<double>(), ctx->hints.as<uint32_t>(),
            ctx->sorted.as<uint8_t>(), ctx->widths.as<double>(), bins, ctx->memo.as<double>(),
            ctx->cfail.as<uint8_t>(), ctx->ich_tile.as<int32_t>(), n_list, base, T, mr, opt, ctx->dcv.as<double>(),
            ctx->vwv.as<double>(), rec_slot, rec_dens);
        return;
    }
    k_pp_channel<D><<<grid, 128, 0, ctx->stream>>>(
        ctx->point_prog.as<PointProgram>(), ctx->edges.as<double>(), ctx->hints.as<uint32_t>(),
        ctx->sorted.as<uint8_t>(), ctx->widths.as<double>(), bins, ctx->memo.as<double>(),
        ctx->cfail.as<uint8_t>(), ctx->ich_tile.as<int32_t>(), n_list, base, T, mr, opt, ctx->dcv.as<double>(),
        ctx->vwv.as<double>(), rec_slot, rec_dens);
}

}  // namespace

// The phased weight pass (pipeline.cuh) over the n_pre listed points of a
// momenta buffer of m points (list: their indices, ich: their channels,
// n_list: the device-side count), in tiles of at most ctx->pipe_tile points
// (option "pipeline_tile"; the default 2^22 makes one tile of a chunk, whose
// intermediates go through HBM: tiles small enough for their buffers to stay
// in L2 were measured slower, every launch's tail growing with the launch
// count); `combine` launches the last step of
// each tile (it reads the per-channel densities ctx->dcv, ctx->vwv and the
// nodes ctx->node_soa of the tile).
int pipeline_run(chili_ctx *ctx, const double *mom_soa, long long m, const int32_t *list, const int32_t *ich,
                 const long long *n_list, long long n_pre, int bins, bool opt, int32_t *rec_slot, double *rec_dens,
                 const TileFn &combine, const PPFusedOut *fused) {
    if (ctx->hints_stale)
        if (int rc = rebuild_hints(ctx)) return rc;
    const PointProgram &P = ctx->pp_host;
    const PointProgram *pp = ctx->point_prog.as<PointProgram>();
    // gridDim.y (point blocks of 128) stays below 65536
    const long long T = std::min<long long>(std::min<long long>(ctx->pipe_tile, 65535ll * 128),
                                            std::max<long long>(n_pre, 1));
    // buffers for a whole number of 2^16 points: the accepted count of a
    // chunk varies from call to call, and a buffer that grew by a few points
    // each time would be reallocated (a device synchronisation) each time
    const long long Ta = (T + 65535) / 65536 * 65536;
    CK(ctx->node_soa.ensure(sizeof(double) * 4 * P.n_nodes * Ta));
    CK(ctx->memo.ensure(sizeof(double) * std::max(1, P.n_memo) * Ta));
    CK(ctx->cfail.ensure(static_cast<size_t>(std::max(1, P.n_chains)) * Ta));
    CK(ctx->dcv.ensure(sizeof(double) * ctx->nch * Ta));
    CK(ctx->ich_tile.ensure(sizeof(int32_t) * Ta));
    CK(ctx->vwv.ensure(sizeof(double) * ctx->nch * Ta));
    PPCombine comb{};
    const bool fuse = fused && ctx->fuse_combine;
    if (fuse) {
        const size_t nblk = static_cast<size_t>((Ta + 127) / 128);
        if (ctx->arrivals.cap < sizeof(unsigned) * nblk) {
            CK(ctx->arrivals.ensure(sizeof(unsigned) * nblk));
            CK(cudaMemsetAsync(ctx->arrivals.p, 0, ctx->arrivals.cap, ctx->stream));
        }
        comb = PPCombine{alpha_ptr(ctx), ctx->node_soa.as<double>(), ctx->f_dev.as<IntegrandDesc>(), fused->rec_val,
                         fused->rec_wgt, fused->rec_ok, ctx->arrivals.as<unsigned>()};
    }
    const unsigned gx = static_cast<unsigned>((T + 255) / 256);
    const int n_items = P.n_tents + P.n_dws + P.n_sws;
    const int o = opt ? 1 : 0;
    for (long long base = 0; base < n_pre; base += T) {
        { KTimer kt_(ctx, KT_NODES);
        k_pp_nodes<<<gx, 256, 0, ctx->stream>>>(pp, mom_soa, m, list, ich, n_list, base, ctx->node_soa.as<double>(),
                                                 ctx->ich_tile.as<int32_t>(), T); }
        LAUNCHED();
        if (n_items > 0) {
            KTimer kt_(ctx, KT_ITEMS);
            if (P.n_tents > 0) {
                k_pp_items<0><<<dim3(P.n_tents, gx), 256, 0, ctx->stream>>>(pp, ctx->node_soa.as<double>(), n_list,
                                                                             base, T, ctx->memo.as<double>());
                LAUNCHED();
            }
            if (P.n_dws > 0) {
                k_pp_items<1><<<dim3(P.n_dws, gx), 256, 0, ctx->stream>>>(pp, ctx->node_soa.as<double>(), n_list,
                                                                           base, T, ctx->memo.as<double>());
                LAUNCHED();
            }
            if (P.n_sws > 0) {
                k_pp_items<2><<<dim3(P.n_sws, gx), 256, 0, ctx->stream>>>(pp, ctx->node_soa.as<double>(), n_list,
                                                                           base, T, ctx->memo.as<double>());
                LAUNCHED();
            }
        }
        { KTimer kt_(ctx, KT_CHAINS);
        k_pp_chains<<<dim3(P.n_chains, gx), 256, 0, ctx->stream>>>(pp, ctx->node_soa.as<double>(), n_list, base, T,
                                                                    ctx->memo.as<double>(), ctx->cfail.as<uint8_t>()); }
        LAUNCHED();
        switch (P.ndims) {
#define CHILI_CH(D) \
    case D: { KTimer kt_(ctx, KT_CHANNEL); launch_channel<D>(ctx, base, T, m, bins, o, n_list, rec_slot, rec_dens, fuse ? &comb : nullptr); } break;
            CHILI_CH(1) CHILI_CH(4) CHILI_CH(7) CHILI_CH(10) CHILI_CH(13) CHILI_CH(16) CHILI_CH(19) CHILI_CH(22)
#undef CHILI_CH
        default: return fail(ctx, CHILI_ERR_STATE, "no phased weight kernel for this dimension");
        }
        LAUNCHED();
        if (!fuse)
            if (int rc = combine(base, T)) return rc;
    }
    return CHILI_OK;
}

int pp_pass_launch(chili_ctx *ctx, const PPPass &a) {
    const PointProgram &P = *a.pp_host;
    const long long T = a.T;
    if (T < 1 || T > 65535ll * 128) return fail(ctx, CHILI_ERR_LIMIT, "phased pass of 1 .. 65535*128 points");
    const unsigned gx = static_cast<unsigned>((T + 255) / 256);
    k_pp_nodes<<<gx, 256, 0, ctx->stream>>>(a.pp, a.mom_soa, a.mc, a.list, a.ich, a.n_list, 0, a.node_soa, a.ich_tile,
                                             T);
    LAUNCHED();
    if (P.n_tents > 0) {
        k_pp_items<0><<<dim3(P.n_tents, gx), 256, 0, ctx->stream>>>(a.pp, a.node_soa, a.n_list, 0, T, a.memo);
        LAUNCHED();
    }
    if (P.n_dws > 0) {
        k_pp_items<1><<<dim3(P.n_dws, gx), 256, 0, ctx->stream>>>(a.pp, a.node_soa, a.n_list, 0, T, a.memo);
        LAUNCHED();
    }
    if (P.n_sws > 0) {
        k_pp_items<2><<<dim3(P.n_sws, gx), 256, 0, ctx->stream>>>(a.pp, a.node_soa, a.n_list, 0, T, a.memo);
        LAUNCHED();
    }
    if (P.n_chains > 0) {
        k_pp_chains<<<dim3(P.n_chains, gx), 256, 0, ctx->stream>>>(a.pp, a.node_soa, a.n_list, 0, T, a.memo, a.cfail);
        LAUNCHED();
    }
    const dim3 gc(static_cast<unsigned>(P.nch), static_cast<unsigned>((T + 127) / 128));
    switch (P.ndims) {
#define CHILI_CH(D)                                                                                          \
    case D:                                                                                                  \
        if (a.hints)                                                                                         \
            k_pp_channel<D, true><<<gc, 128, 0, ctx->stream>>>(                                              \
                a.pp, a.grids, a.hints, a.sorted, a.widths, a.bins, a.memo, a.cfail, a.ich_tile, a.n_list,        \
                0, T, a.mr, 1, a.dcv, a.vwv, a.rec_slot, a.rec_dens);                                        \
        else                                                                                                 \
            k_pp_channel<D, false><<<gc, 128, 0, ctx->stream>>>(                                             \
                a.pp, a.grids, a.hints, a.sorted, a.widths, a.bins, a.memo, a.cfail, a.ich_tile,              \
                a.n_list, 0, T, a.mr, 1, a.dcv, a.vwv, a.rec_slot, a.rec_dens);                              \
        break;
        CHILI_CH(1) CHILI_CH(4) CHILI_CH(7) CHILI_CH(10) CHILI_CH(13) CHILI_CH(16) CHILI_CH(19) CHILI_CH(22)
#undef CHILI_CH
    default: return fail(ctx, CHILI_ERR_STATE, "no phased weight kernel for this dimension");
    }
    LAUNCHED();
    k_pp_combine<<<gx, 256, 0, ctx->stream>>>(a.pp, a.alpha, a.dcv, a.vwv, a.node_soa, a.n_list, 0, T, a.f,
                                               a.rec_val, a.rec_wgt, a.rec_ok);
    LAUNCHED();
    return CHILI_OK;
}

int compact_launch(chili_ctx *ctx, const int32_t *block_count, int nb, const uint8_t *flag, long long m,
                   long long *block_off, RoundCtl *ctl, int32_t *list) {
    k_mc_scan<<<1, 1024, 0, ctx->stream>>>(block_count, nb, flag, m, m + 1, nullptr, 0, block_off, ctl);
    LAUNCHED();
    k_mc_compact<<<static_cast<unsigned>(nb), kFwdBlock, 0, ctx->stream>>>(flag, block_off, ctl, m, list);
    LAUNCHED();
    return CHILI_OK;
}

namespace {

// Host uniforms u[m][D+1]: rows [0, m) are copied into the staging buffer
// in slices on the context's copy stream, slice s followed by
// copy_events[s]: slices that double from kFirstSlice rows (the only copy
// nothing overlaps) up to the option "upload_slice" (2^19 rows), so that the
// weight passes start early and the copies, a little faster per row than
// the weight pass, stay ahead.  The rounds of the iteration take one slice
// each, so that the upload of the next slices overlaps the whole weight pass
// of this one.
constexpr long long kFirstSlice = 1ll << 16;   // rows, a multiple of kFwdBlock

// Slice boundaries of a chunk of m rows: slices that double from kFirstSlice
// rows up to `top` rows (option "upload_slice", default kUploadSlice).
std::vector<long long> slice_bounds(long long m, long long top) {
    std::vector<long long> b{0};
    long long len = kFirstSlice;
    while (b.back() < m) {
        b.push_back(std::min(b.back() + len, m));
        len = std::min(2 * len, top);
    }
    return b;
}

int upload_host(chili_ctx *ctx, const double *u, long long m, const std::vector<long long> &sb) {
    const int D = ctx->ndims;
    const size_t row = sizeof(double) * (D + 1);
    CK(ctx->stage[0].ensure(row * static_cast<size_t>(m)));
    if (!ctx->copy_stream) CK(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    const long long nslices = static_cast<long long>(sb.size()) - 1;
    while (static_cast<long long>(ctx->copy_events.size()) < nslices + 1) {
        cudaEvent_t e;
        CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ctx->copy_events.push_back(e);
    }
    // the staging buffer is free once the work queued before on the
    // context's stream (earlier readers of it) is done
    CK(cudaEventRecord(ctx->copy_events[nslices], ctx->stream));
    CK(cudaStreamWaitEvent(ctx->copy_stream, ctx->copy_events[nslices], 0));
    double *dst = ctx->stage[0].as<double>();
    for (long long s = 0; s < nslices; ++s) {
        const long long s0 = sb[s], len = sb[s + 1] - s0;
        CK(cudaMemcpyAsync(dst + s0 * (D + 1), u + s0 * (D + 1), row * static_cast<size_t>(len),
                           cudaMemcpyHostToDevice, ctx->copy_stream));
        CK(cudaEventRecord(ctx->copy_events[s], ctx->copy_stream));
    }
    return CHILI_OK;
}

// The phased weight pass of a multichannel chunk: records of the n_pre
// PreProcess-accepted points of the chunk of m counters.
int launch_pipeline(chili_ctx *ctx, const double *mom_soa, const int32_t *ich, long long m, long long n_pre, int bins,
                    bool opt, RoundCtl *ctl_pre, double *rec_val, double *rec_wgt, uint8_t *rec_ok, int32_t *rec_slot,
                    double *rec_dens) {
    const PointProgram *pp = ctx->point_prog.as<PointProgram>();
    const long long *n_list = reinterpret_cast<const long long *>(
        reinterpret_cast<const char *>(ctl_pre) + offsetof(RoundCtl, n_acc));
    const PPFusedOut fused{rec_val, rec_wgt, rec_ok};
    return pipeline_run(ctx, mom_soa, m, ctx->list.as<int32_t>(), ich, n_list,
                        n_pre, bins, opt, rec_slot, rec_dens, [&](long long base, long long T) -> int {
                            const unsigned gx = static_cast<unsigned>((T + 255) / 256);
                            {
                                KTimer kt_(ctx, KT_COMBINE);
                                k_pp_combine<<<gx, 256, 0, ctx->stream>>>(
                                    pp, alpha_ptr(ctx), ctx->dcv.as<double>(), ctx->vwv.as<double>(),
                                    ctx->node_soa.as<double>(), n_list, base, T, ctx->f_dev.as<IntegrandDesc>(),
                                    rec_val, rec_wgt, rec_ok);
                            }
                            LAUNCHED();
                            return CHILI_OK;
                        }, &fused);
}

// Hint tables of the grid set (grid.cuh, find_bin_hinted), rebuilt after
// every change of the edges.
int rebuild_hints(chili_ctx *ctx) {
    ctx->hints_stale = false;
    const int H = kHintPerBin * ctx->bins;
    CK(ctx->hints.ensure(sizeof(uint32_t) * static_cast<size_t>(ctx->g_nch) * ctx->dims * H));
    CK(ctx->sorted.ensure(static_cast<size_t>(ctx->g_nch) * ctx->dims));
    CK(ctx->widths.ensure(sizeof(double) * static_cast<size_t>(ctx->g_nch) * ctx->dims * ctx->bins));
    k_build_hints<<<dim3(ctx->dims, ctx->g_nch), 128, 0, ctx->stream>>>(ctx->edges.as<double>(), ctx->dims, ctx->bins,
                                                                        ctx->hints.as<uint32_t>(),
                                                                        ctx->sorted.as<uint8_t>(),
                                                                        ctx->widths.as<double>());
    LAUNCHED();
    return CHILI_OK;
}

}  // namespace

extern "C" {

int chili_gpu_create(int device, chili_ctx **out) {
    chili_ctx *ctx = nullptr;
    if (!out) return fail(nullptr, CHILI_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return fail(nullptr, CHILI_ERR_CUDA, "no CUDA device available");
    }
    if (device < 0 || device >= ndev) return fail(nullptr, CHILI_ERR_INVALID_ARG, "device index out of range");
    ctx = new chili_ctx();
    ctx->device = device;
    int rc;
    if ((rc = set_device(ctx)) != CHILI_OK) {
        delete ctx;
        return rc;
    }
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return fail(nullptr, CHILI_ERR_CUDA, "cudaStreamCreate failed");
    }
    ctx->own_stream = true;
    if (cudaMallocHost(reinterpret_cast<void **>(&ctx->ctl_host), 2 * sizeof(RoundCtl)) != cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void **>(&ctx->iter_host), sizeof(long long) * kIterCtl) != cudaSuccess) {
        if (ctx->ctl_host) cudaFreeHost(ctx->ctl_host);
        cudaStreamDestroy(ctx->stream);
        delete ctx;
        return fail(nullptr, CHILI_ERR_CUDA, "cudaMallocHost failed");
    }
    cudaDeviceGetAttribute(&ctx->max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, device);
    cudaFuncSetAttribute(k_mc_accum, cudaFuncAttributeMaxDynamicSharedMemorySize, ctx->max_smem_optin);
    cudaFuncSetAttribute(k_mc_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, ctx->max_smem_optin);
    cudaFuncSetAttribute(k_vegas_iter<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, ctx->max_smem_optin);
    cudaFuncSetAttribute(k_grid_adapt, cudaFuncAttributeMaxDynamicSharedMemorySize, ctx->max_smem_optin);
    cudaGetLastError();
    *out = ctx;
    return CHILI_OK;
}

int chili_gpu_destroy(chili_ctx *ctx) {
    if (!ctx) return CHILI_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    DevBuf *bufs[] = {&ctx->edges, &ctx->edges_tmp, &ctx->progs, &ctx->point_prog, &ctx->node_soa, &ctx->memo, &ctx->cfail, &ctx->dcv, &ctx->vwv, &ctx->hints, &ctx->sorted, &ctx->widths, &ctx->ich_tile, &ctx->alpha_buf, &ctx->f_dev, &ctx->mom_soa,
                      &ctx->ich, &ctx->flag, &ctx->list, &ctx->block_count, &ctx->block_off, &ctx->part,
                      &ctx->hist, &ctx->round_res, &ctx->acc, &ctx->ctl, &ctx->status, &ctx->v_part,
                      &ctx->v_hist, &ctx->v_train, &ctx->v_out, &ctx->rec, &ctx->ctl3, &ctx->unw, &ctx->iter_ctl,
                      &ctx->mom_soa_alt, &ctx->ich_alt, &ctx->flag_alt, &ctx->block_count_alt, &ctx->arrivals,
                      &ctx->v_arrive};
    for (DevBuf *b : bufs) b->release();
    flow_release(ctx);
    batch_release(ctx);
    for (auto &b : ctx->stage) b.release();
    if (ctx->ctl_host) cudaFreeHost(ctx->ctl_host);
    if (ctx->iter_host) cudaFreeHost(ctx->iter_host);
    collect_times(ctx);
    for (cudaEvent_t e : ctx->event_pool) cudaEventDestroy(e);
    for (cudaEvent_t e : ctx->copy_events) cudaEventDestroy(e);
    for (int k = 0; k < 2; ++k) {
        if (ctx->fwd_done[k]) cudaEventDestroy(ctx->fwd_done[k]);
        if (ctx->round_done[k]) cudaEventDestroy(ctx->round_done[k]);
    }
    if (ctx->fwd_stream) {
        cudaStreamSynchronize(ctx->fwd_stream);
        cudaStreamDestroy(ctx->fwd_stream);
    }
    if (ctx->copy_stream) {
        cudaStreamSynchronize(ctx->copy_stream);
        cudaStreamDestroy(ctx->copy_stream);
    }
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return CHILI_OK;
}

const char *chili_gpu_last_error(const chili_ctx *ctx) {
    return ctx ? ctx->err.c_str() : g_last_error.c_str();
}

int chili_gpu_set_stream(chili_ctx *ctx, void *stream) {
    if (!ctx) return fail(nullptr, CHILI_ERR_INVALID_ARG, "ctx is NULL");
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    if (stream) {
        if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
        ctx->stream = static_cast<cudaStream_t>(stream);
        ctx->own_stream = false;
    } else if (!ctx->own_stream) {
        CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        ctx->own_stream = true;
    }
    return CHILI_OK;
}

int chili_gpu_synchronize(chili_ctx *ctx) {
    if (!ctx) return fail(nullptr, CHILI_ERR_INVALID_ARG, "ctx is NULL");
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->timing) collect_times(ctx);
    return CHILI_OK;
}

int chili_gpu_kernel_time(chili_ctx *ctx, const char *kernel, double *ms, uint64_t *launches) {
    if (!ctx || !kernel) return fail(ctx, CHILI_ERR_INVALID_ARG, "NULL argument");
    CK(cudaStreamSynchronize(ctx->stream));
    collect_times(ctx);
    for (int k = 0; kTimedKernels[k]; ++k) {
        if (std::strcmp(kTimedKernels[k], kernel) == 0) {
            if (ms) *ms = ctx->ktime_ms[k];
            if (launches) *launches = ctx->klaunches[k];
            return CHILI_OK;
        }
    }
    return fail(ctx, CHILI_ERR_INVALID_ARG, std::string("not a timed kernel: ") + kernel);
}

uint64_t chili_gpu_launch_count(const chili_ctx *ctx) { return ctx ? ctx->launches : 0; }

int chili_gpu_set_option(chili_ctx *ctx, const char *name, int64_t value) {
    if (!ctx || !name) return fail(ctx, CHILI_ERR_INVALID_ARG, "NULL argument");
    if (std::strcmp(name, "point_program") == 0) {
        ctx->use_pp = value != 0;
        return CHILI_OK;
    }
    if (std::strcmp(name, "vegas_fused") == 0) {
        ctx->vegas_fused = value != 0;
        return CHILI_OK;
    }
    if (std::strcmp(name, "vegas_gen_ppt") == 0) {
        if (value != 1 && value != 2 && value != 4) return fail(ctx, CHILI_ERR_INVALID_ARG, "vegas_gen_ppt: 1, 2 or 4");
        ctx->gen_ppt = value;
        return CHILI_OK;
    }
    if (std::strcmp(name, "pipeline_fuse") == 0) {
        ctx->fuse_combine = value != 0;
        return CHILI_OK;
    }
    if (std::strcmp(name, "pipeline") == 0) {
        ctx->use_pipeline = value != 0;
        return CHILI_OK;
    }
    if (std::strcmp(name, "kernel_timing") == 0) {
        CK(cudaStreamSynchronize(ctx->stream));
        collect_times(ctx);
        ctx->timing = value != 0;
        for (double &t : ctx->ktime_ms) t = 0;
        for (auto &n : ctx->klaunches) n = 0;
        return CHILI_OK;
    }
    if (std::strcmp(name, "max_rounds") == 0) {
        if (value < 1) return fail(ctx, CHILI_ERR_INVALID_ARG, "max_rounds must be >= 1");
        ctx->max_rounds = value;
        return CHILI_OK;
    }
    if (std::strcmp(name, "defer_train") == 0) {
        ctx->defer_train = value != 0;
        return CHILI_OK;
    }
    if (std::strcmp(name, "batch_retry") == 0) {
        ctx->batch_retry = value != 0;
        return CHILI_OK;
    }
    if (std::strcmp(name, "batch_grouped") == 0) {
        ctx->batch_grouped = value != 0;
        return CHILI_OK;
    }
    if (std::strcmp(name, "batch_wave_streams") == 0) {
        if (value < 1 || value > 4) return fail(ctx, CHILI_ERR_INVALID_ARG, "batch_wave_streams in [1, 4]");
        ctx->batch_wave_streams = value;
        return CHILI_OK;
    }
    if (std::strcmp(name, "batch_wave_points") == 0) {
        if (value < 1 || value > (1ll << 30)) return fail(ctx, CHILI_ERR_INVALID_ARG, "batch_wave_points in [1, 2^30]");
        ctx->batch_wave = value;
        return CHILI_OK;
    }
    if (std::strcmp(name, "batch_channel_points") == 0) {
        if (value < 128 || value > 4096 || value % 128)
            return fail(ctx, CHILI_ERR_INVALID_ARG, "batch_channel_points: a multiple of 128 in [128, 4096]");
        ctx->batch_ch_pts = value;
        return CHILI_OK;
    }
    if (std::strcmp(name, "batch_phased") == 0) {
        ctx->batch_phased = value != 0;
        return CHILI_OK;
    }
    if (std::strcmp(name, "upload_slice") == 0) {
        if (value < kFirstSlice || value > (1ll << 24) || value % kFwdBlock)
            return fail(ctx, CHILI_ERR_INVALID_ARG, "upload_slice in [2^16, 2^24] rows, a multiple of 256");
        ctx->upload_slice = value;
        return CHILI_OK;
    }
    if (std::strcmp(name, "pipeline_sync") == 0) {
        ctx->pipe_sync = value != 0;
        return CHILI_OK;
    }
    if (std::strcmp(name, "hist_shared") == 0) {
        ctx->hist_shared = value != 0;
        return CHILI_OK;
    }
    if (std::strcmp(name, "channel_tables") == 0) {
        ctx->channel_tables = value != 0;
        return CHILI_OK;
    }
    if (std::strcmp(name, "flow_streamed") == 0) {
        ctx->flow_streamed = value != 0;
        return CHILI_OK;
    }
    if (std::strcmp(name, "pipeline_tile") == 0) {
        if (value < 1024 || value > (1ll << 24)) return fail(ctx, CHILI_ERR_INVALID_ARG, "pipeline_tile outside [1024, 2^24]");
        ctx->pipe_tile = value;
        return CHILI_OK;
    }
    return fail(ctx, CHILI_ERR_INVALID_ARG, std::string("unknown option ") + name);
}

// --------------------------------------------------------------------- grids
int chili_gpu_set_grids(chili_ctx *ctx, const double *edges, int nch, int dims, int bins) {
    if (!ctx || !edges) return fail(ctx, CHILI_ERR_INVALID_ARG, "NULL argument");
    if (nch < 1 || nch > CHILI_MAX_CHANNELS || dims < 1 || dims > CHILI_MAX_DIMS || bins < 2 ||
        bins > CHILI_MAX_BINS)
        return fail(ctx, CHILI_ERR_LIMIT, "grid shape outside the compiled limits");
    if (ctx->nch > 0 && (nch != ctx->nch || dims != ctx->ndims))
        return fail(ctx, CHILI_ERR_INVALID_ARG, "grid count/dims do not match the channels");
    int rc;
    if ((rc = set_device(ctx))) return rc;
    const size_t bytes = sizeof(double) * nch * dims * (bins + 1);
    CK(ctx->edges.ensure(bytes));
    CK(ctx->edges_tmp.ensure(bytes));
    Arg a;
    if ((rc = resolve(ctx, edges, bytes, 0, true, a))) return rc;
    CK(cudaMemcpyAsync(ctx->edges.p, a.dev, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    ctx->g_nch = nch;
    ctx->dims = dims;
    ctx->bins = bins;
    if ((rc = rebuild_hints(ctx))) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return CHILI_OK;
}

int chili_gpu_get_grids(chili_ctx *ctx, double *edges, int nch, int dims, int bins) {
    if (!ctx || !edges) return fail(ctx, CHILI_ERR_INVALID_ARG, "NULL argument");
    int rc;
    if ((rc = need_grids(ctx))) return rc;
    if (nch != ctx->g_nch || dims != ctx->dims || bins != ctx->bins)
        return fail(ctx, CHILI_ERR_INVALID_ARG, "grid shape mismatch");
    const size_t bytes = sizeof(double) * nch * dims * (bins + 1);
    Arg a;
    if ((rc = resolve(ctx, edges, bytes, 0, false, a))) return rc;
    CK(cudaMemcpyAsync(a.dev, ctx->edges.p, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    if ((rc = finish_out(ctx, a))) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return CHILI_OK;
}

int chili_gpu_grid_map(chili_ctx *ctx, int ch, const double *u, double *x, double *jac, int64_t n) {
    if (!ctx) return fail(nullptr, CHILI_ERR_INVALID_ARG, "ctx is NULL");
    int rc;
    if ((rc = need_grids(ctx))) return rc;
    if (ch < 0 || ch >= ctx->g_nch || n < 0 || !u || !x || !jac) return fail(ctx, CHILI_ERR_INVALID_ARG, "bad argument");
    if (n == 0) return CHILI_OK;
    const int D = ctx->dims, B = ctx->bins;
    Arg au, ax, aj;
    if ((rc = resolve(ctx, u, sizeof(double) * n * D, 0, true, au))) return rc;
    if ((rc = resolve(ctx, x, sizeof(double) * n * D, 1, false, ax))) return rc;
    if ((rc = resolve(ctx, jac, sizeof(double) * n, 2, false, aj))) return rc;
    const double *g = ctx->edges.as<double>() + static_cast<size_t>(ch) * D * (B + 1);
    k_grid_map<<<grid_for(n, 128), 128, 0, ctx->stream>>>(g, D, B, static_cast<const double *>(au.dev),
                                                          static_cast<double *>(ax.dev),
                                                          static_cast<double *>(aj.dev), n);
    LAUNCHED();
    if ((rc = finish_out(ctx, ax)) || (rc = finish_out(ctx, aj))) return rc;
    return sync_if_host(ctx, {&au, &ax, &aj});
}

int chili_gpu_grid_weight(chili_ctx *ctx, int ch, const double *x, double *w, int32_t *bin, int64_t n) {
    if (!ctx) return fail(nullptr, CHILI_ERR_INVALID_ARG, "ctx is NULL");
    int rc;
    if ((rc = need_grids(ctx))) return rc;
    if (ch < 0 || ch >= ctx->g_nch || n < 0 || !x || (!w && !bin)) return fail(ctx, CHILI_ERR_INVALID_ARG, "bad argument");
    if (n == 0) return CHILI_OK;
    const int D = ctx->dims, B = ctx->bins;
    Arg ax, aw, ab;
    if ((rc = resolve(ctx, x, sizeof(double) * n * D, 0, true, ax))) return rc;
    if ((rc = resolve(ctx, w, sizeof(double) * n, 1, false, aw))) return rc;
    if ((rc = resolve(ctx, bin, sizeof(int32_t) * n * D, 2, false, ab))) return rc;
    if (ctx->hints_stale)
        if ((rc = rebuild_hints(ctx))) return rc;
    const double *g = ctx->edges.as<double>() + static_cast<size_t>(ch) * D * (B + 1);
    const uint32_t *hg = ctx->hints.as<uint32_t>() + static_cast<size_t>(ch) * D * (kHintPerBin * B);
    const uint8_t *sg = ctx->sorted.as<uint8_t>() + static_cast<size_t>(ch) * D;
    k_grid_weight<<<grid_for(n, 128), 128, 0, ctx->stream>>>(g, hg, sg, D, B, static_cast<const double *>(ax.dev),
                                                             static_cast<double *>(aw.dev),
                                                             static_cast<int32_t *>(ab.dev), n);
    LAUNCHED();
    if ((rc = finish_out(ctx, aw)) || (rc = finish_out(ctx, ab))) return rc;
    return sync_if_host(ctx, {&ax, &aw, &ab});
}

static int adapt_grids(chili_ctx *ctx, int first, int count, double alpha, const double *train_dev, int skip_zero) {
    const int D = ctx->dims, B = ctx->bins;
    CK(ctx->status.ensure(sizeof(int)));
    CK(cudaMemsetAsync(ctx->status.p, 0, sizeof(int), ctx->stream));
    const size_t gsz = static_cast<size_t>(D) * (B + 1);
    // grids outside [first, first+count) keep their edges
    if (count != ctx->g_nch)
        CK(cudaMemcpyAsync(ctx->edges_tmp.p, ctx->edges.p, sizeof(double) * gsz * ctx->g_nch,
                           cudaMemcpyDeviceToDevice, ctx->stream));
    dim3 grid(D, count);
    k_grid_adapt<<<grid, 32, sizeof(double) * B, ctx->stream>>>(
        ctx->edges.as<double>() + first * gsz, ctx->edges_tmp.as<double>() + first * gsz, D, B, alpha, train_dev,
        skip_zero, ctx->status.as<int>());
    LAUNCHED();
    std::swap(ctx->edges, ctx->edges_tmp);
    return rebuild_hints(ctx);
}

int chili_gpu_grid_adapt(chili_ctx *ctx, int ch, double alpha, const double *train) {
    if (!ctx) return fail(nullptr, CHILI_ERR_INVALID_ARG, "ctx is NULL");
    int rc;
    if ((rc = need_grids(ctx))) return rc;
    if (ch < 0 || ch >= ctx->g_nch || !train) return fail(ctx, CHILI_ERR_INVALID_ARG, "bad argument");
    Arg at;
    if ((rc = resolve(ctx, train, sizeof(double) * ctx->dims * ctx->bins, 0, true, at))) return rc;
    if ((rc = adapt_grids(ctx, ch, 1, alpha, static_cast<const double *>(at.dev), 0))) return rc;
    return sync_if_host(ctx, {&at});
}

int chili_gpu_grid_split(chili_ctx *ctx, int nsplit) {
    if (!ctx) return fail(nullptr, CHILI_ERR_INVALID_ARG, "ctx is NULL");
    int rc;
    if ((rc = need_grids(ctx))) return rc;
    if (nsplit < 2 || nsplit > 4) return fail(ctx, CHILI_ERR_INVALID_ARG, "nsplit must be 2, 3 or 4");
    const int nb = ctx->bins * nsplit;
    if (nb > CHILI_MAX_BINS) return fail(ctx, CHILI_ERR_LIMIT, "split grid exceeds CHILI_MAX_BINS");
    const size_t bytes = sizeof(double) * ctx->g_nch * ctx->dims * (nb + 1);
    CK(ctx->edges_tmp.ensure(bytes));
    const long long total = static_cast<long long>(ctx->g_nch) * ctx->dims * ctx->bins;
    k_grid_split<<<grid_for(total, 128), 128, 0, ctx->stream>>>(ctx->edges.as<double>(), ctx->edges_tmp.as<double>(),
                                                                ctx->g_nch, ctx->dims, ctx->bins, nsplit);
    LAUNCHED();
    CK(cudaStreamSynchronize(ctx->stream));
    std::swap(ctx->edges, ctx->edges_tmp);
    CK(ctx->edges_tmp.ensure(bytes));
    ctx->bins = nb;
    return rebuild_hints(ctx);
}

// ----------------------------------------------------------------- integrand
int chili_gpu_set_integrand(chili_ctx *ctx, int kind, const double *params, int nparams) {
    if (!ctx) return fail(nullptr, CHILI_ERR_INVALID_ARG, "ctx is NULL");
    if (kind < CHILI_FUNC_UNIT || kind > CHILI_FUNC_PROPAGATOR_TOP2)
        return fail(ctx, CHILI_ERR_INVALID_ARG, "unknown integrand kind");
    if (nparams < 0 || nparams > CHILI_MAX_INTEGRAND_PARAMS || (nparams > 0 && !params))
        return fail(ctx, CHILI_ERR_LIMIT, "integrand parameter count outside [0, CHILI_MAX_INTEGRAND_PARAMS]");
    const int need = kind == CHILI_FUNC_CAMEL ? 2 : (kind == CHILI_FUNC_UNIT ? 0 : 3);
    if (nparams < need) return fail(ctx, CHILI_ERR_INVALID_ARG, "too few integrand parameters");
    int rc;
    if ((rc = set_device(ctx))) return rc;
    ctx->f_host.kind = kind;
    ctx->f_host.nparams = nparams;
    for (int i = 0; i < nparams; ++i) ctx->f_host.p[i] = params[i];
    CK(ctx->f_dev.ensure(sizeof(IntegrandDesc)));
    CK(cudaMemcpyAsync(ctx->f_dev.p, &ctx->f_host, sizeof(IntegrandDesc), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->f_set = true;
    return CHILI_OK;
}

int chili_gpu_set_preprocess(chili_ctx *ctx, int kind) {
    if (!ctx) return fail(nullptr, CHILI_ERR_INVALID_ARG, "ctx is NULL");
    if (kind != CHILI_PRE_ACCEPT_ALL && kind != CHILI_PRE_FINITE)
        return fail(ctx, CHILI_ERR_INVALID_ARG,
                    kind == CHILI_PRE_CUTS ? "CHILI_PRE_CUTS is set with chili_gpu_set_preprocess_cuts"
                                           : "unknown preprocess kind");
    int rc;
    if ((rc = set_device(ctx))) return rc;
    ctx->f_host.pre = kind;
    CK(ctx->f_dev.ensure(sizeof(IntegrandDesc)));
    CK(cudaMemcpyAsync(ctx->f_dev.p, &ctx->f_host, sizeof(IntegrandDesc), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return CHILI_OK;
}

int chili_gpu_set_preprocess_cuts(chili_ctx *ctx, double sqrts, double ptmin, double etamax, double delta_r) {
    if (!ctx) return fail(nullptr, CHILI_ERR_INVALID_ARG, "ctx is NULL");
    if (int rc = need_channels(ctx)) return rc;
    if (!(sqrts > 0) || !(ptmin >= 0) || !(etamax >= 0) || !(delta_r >= 0))
        return fail(ctx, CHILI_ERR_INVALID_ARG, "cut values must be >= 0 (sqrts > 0)");
    if (int rc = set_device(ctx)) return rc;
    ctx->f_host.pre = CHILI_PRE_CUTS;
    ctx->f_host.n_ext = ctx->n_ext;
    ctx->f_host.cut[0] = sqrts;
    ctx->f_host.cut[1] = ptmin;
    ctx->f_host.cut[2] = etamax;
    ctx->f_host.cut[3] = delta_r;
    CK(ctx->f_dev.ensure(sizeof(IntegrandDesc)));
    CK(cudaMemcpyAsync(ctx->f_dev.p, &ctx->f_host, sizeof(IntegrandDesc), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return CHILI_OK;
}

// ----------------------------------------------------------------- plain VEGAS
int chili_gpu_vegas_iterate(chili_ctx *ctx, uint64_t ncalls, uint64_t seed, uint64_t counter_base,
                            const double *u, double alpha, int adapt, chili_stats *stats_out, double *train_out) {
    if (!ctx) return fail(nullptr, CHILI_ERR_INVALID_ARG, "ctx is NULL");
    int rc;
    if ((rc = need_grids(ctx))) return rc;
    if (!ctx->f_set || ctx->f_host.kind != CHILI_FUNC_CAMEL)
        return fail(ctx, CHILI_ERR_STATE, "plain VEGAS needs the camel integrand");
    if (ctx->f_host.nparams < 2 + 2 * ctx->dims)
        return fail(ctx, CHILI_ERR_INVALID_ARG, "camel needs 2 + 2*dims parameters");
    if (ncalls < 2) return fail(ctx, CHILI_ERR_INVALID_ARG, "ncalls must be at least 2");
    const int D = ctx->dims, B = ctx->bins, nh = D * B;
    const long long n = static_cast<long long>(ncalls);
    Arg au, ast, atr;
    if ((rc = resolve(ctx, u, sizeof(double) * n * D, 0, true, au))) return rc;
    if ((rc = resolve(ctx, stats_out, sizeof(chili_stats), 1, false, ast))) return rc;
    if ((rc = resolve(ctx, train_out, sizeof(double) * nh, 2, false, atr))) return rc;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    const size_t hist_bytes = sizeof(double) * nh;
    const bool smem = hist_bytes <= 48 * 1024;
    if (smem && adapt && ctx->vegas_fused && ctx->g_nch == 1 &&
        sizeof(double) * B * (kVegasBlock / 32) <= 48 * 1024) {
        // the whole iteration in one launch (k_vegas_step): points, a
        // two-level ordered fold and the adaptation
        const long long nb = std::min<long long>(grid_for(n, kVegasBlock), static_cast<long long>(sms) * 4);
        const long long ngrp = (nb + kStepGroup - 1) / kStepGroup;
        CK(ctx->v_part.ensure(sizeof(double) * 6 * (nb + ngrp)));
        CK(ctx->v_hist.ensure(hist_bytes * (nb + ngrp)));
        CK(ctx->v_train.ensure(hist_bytes));
        CK(ctx->v_out.ensure(sizeof(double) * 6));
        CK(ctx->status.ensure(sizeof(int)));
        const size_t arrive_bytes = sizeof(unsigned) * (1 + ngrp);
        if (ctx->v_arrive.cap < arrive_bytes) {
            CK(ctx->v_arrive.ensure(arrive_bytes));
            CK(cudaMemsetAsync(ctx->v_arrive.p, 0, ctx->v_arrive.cap, ctx->stream));
        }
        CK(ctx->edges_tmp.ensure(sizeof(double) * D * (B + 1)));
        using StepKernel = void (*)(const double *, double *, int, int, uint64_t, uint64_t, const double *, long long,
                                    const IntegrandDesc *, double *, double *, double *, double *, double *, double *,
                                    double, int, unsigned *, int *);
        StepKernel kern = k_vegas_step<0>;
        switch (D) {
#define CHILI_ST(d) \
    case d: kern = k_vegas_step<d>; break;
            CHILI_ST(1) CHILI_ST(2) CHILI_ST(3) CHILI_ST(4) CHILI_ST(5) CHILI_ST(6) CHILI_ST(7) CHILI_ST(8)
            CHILI_ST(10) CHILI_ST(12) CHILI_ST(16)
#undef CHILI_ST
            default: break;
        }
        double *train_dev = train_out ? static_cast<double *>(atr.dev) : ctx->v_train.as<double>();
        double *out_dev = stats_out ? static_cast<double *>(ast.dev) : ctx->v_out.as<double>();
        {
            KTimer kt_(ctx, KT_VEGAS_STEP);
            kern<<<static_cast<unsigned>(nb), kVegasBlock,
                   std::max(hist_bytes, sizeof(double) * B * (kVegasBlock / 32)), ctx->stream>>>(
                ctx->edges.as<double>(), ctx->edges_tmp.as<double>(), D, B, seed, counter_base,
                static_cast<const double *>(au.dev), n, ctx->f_dev.as<IntegrandDesc>(), ctx->v_part.as<double>(),
                ctx->v_hist.as<double>(), ctx->v_part.as<double>() + 6 * nb, ctx->v_hist.as<double>() + nh * nb,
                train_dev, out_dev, alpha, 1, ctx->v_arrive.as<unsigned>(), ctx->status.as<int>());
        }
        LAUNCHED();
        std::swap(ctx->edges, ctx->edges_tmp);
        ctx->hints_stale = true;  // rebuilt where a bin search uses them
        if ((rc = finish_out(ctx, ast)) || (rc = finish_out(ctx, atr))) return rc;
        return sync_if_host(ctx, {&au, &ast, &atr});
    }
    long long nblocks = std::min<long long>(grid_for(n, kVegasBlock), static_cast<long long>(sms) * 4);
    CK(ctx->v_part.ensure(sizeof(double) * 6 * nblocks));
    CK(ctx->v_hist.ensure(smem ? hist_bytes * nblocks : hist_bytes));
    CK(ctx->v_train.ensure(hist_bytes));
    CK(ctx->v_out.ensure(sizeof(double) * 6));
    if (!smem) CK(cudaMemsetAsync(ctx->v_hist.p, 0, hist_bytes, ctx->stream));
    {
    using IterKernel = void (*)(const double *, int, int, uint64_t, uint64_t, const double *, long long,
                                const IntegrandDesc *, double *, double *, int);
    IterKernel kern = k_vegas_iter<0>;  // the histogram stays below 48 KB of shared memory here
    switch (D) {
#define CHILI_IT(d) \
    case d: kern = k_vegas_iter<d>; break;
        CHILI_IT(1) CHILI_IT(2) CHILI_IT(3) CHILI_IT(4) CHILI_IT(5) CHILI_IT(6) CHILI_IT(7) CHILI_IT(8)
        CHILI_IT(10) CHILI_IT(12) CHILI_IT(16)
#undef CHILI_IT
        default: break;
    }
    KTimer kt_(ctx, KT_VEGAS);
    kern<<<static_cast<unsigned>(nblocks), kVegasBlock, smem ? hist_bytes : 0, ctx->stream>>>(
        ctx->edges.as<double>(), D, B, seed, counter_base, static_cast<const double *>(au.dev), n,
        ctx->f_dev.as<IntegrandDesc>(), ctx->v_part.as<double>(), ctx->v_hist.as<double>(), smem ? 1 : 0);
    }
    LAUNCHED();
    double *train = smem ? ctx->v_train.as<double>() : ctx->v_hist.as<double>();
    k_vegas_finalize<<<1, 256, 0, ctx->stream>>>(ctx->v_part.as<double>(), static_cast<int>(nblocks),
                                                 ctx->v_hist.as<double>(), smem ? 1 : 0, nh, train,
                                                 ctx->v_out.as<double>());
    LAUNCHED();
    if (train_out) CK(cudaMemcpyAsync(atr.dev, train, hist_bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    if (stats_out) CK(cudaMemcpyAsync(ast.dev, ctx->v_out.p, sizeof(chili_stats), cudaMemcpyDeviceToDevice, ctx->stream));
    if (adapt) {
        if ((rc = adapt_grids(ctx, 0, 1, alpha, train, 0))) return rc;
    }
    if ((rc = finish_out(ctx, ast)) || (rc = finish_out(ctx, atr))) return rc;
    return sync_if_host(ctx, {&au, &ast, &atr});
}

int chili_gpu_vegas_generate(chili_ctx *ctx, uint64_t n, uint64_t seed, uint64_t counter_base, double *x_out,
                             double *w_out) {
    if (!ctx) return fail(nullptr, CHILI_ERR_INVALID_ARG, "ctx is NULL");
    int rc;
    if ((rc = need_grids(ctx))) return rc;
    if (!ctx->f_set || ctx->f_host.kind != CHILI_FUNC_CAMEL)
        return fail(ctx, CHILI_ERR_STATE, "plain VEGAS needs the camel integrand");
    if (ctx->f_host.nparams < 2 + 2 * ctx->dims)
        return fail(ctx, CHILI_ERR_INVALID_ARG, "camel needs 2 + 2*dims parameters");
    if (!x_out || !w_out) return fail(ctx, CHILI_ERR_INVALID_ARG, "x_out and w_out are required");
    if (n == 0) return CHILI_OK;
    if (n > (1ull << 40)) return fail(ctx, CHILI_ERR_LIMIT, "n must be at most 2^40");
    const int D = ctx->dims, B = ctx->bins;
    // points per thread: 4 where the staged tile stays small, else 1
    const size_t grid_doubles = (static_cast<size_t>(D) * (B + 1) + 1) / 2 * 2;
    int ppt = static_cast<int>(ctx->gen_ppt);
    if (sizeof(double) * (grid_doubles + static_cast<size_t>(kGenTile) * ppt * (D + 1)) > 64 * 1024) ppt = 1;
    const size_t smem = sizeof(double) * (grid_doubles + static_cast<size_t>(kGenTile) * ppt * (D + 1));
    if (smem > 200 * 1024) return fail(ctx, CHILI_ERR_LIMIT, "grid too large for the shared-memory staging");
    const long long nn = static_cast<long long>(n);
    Arg ax, aw;
    if ((rc = resolve(ctx, x_out, sizeof(double) * nn * D, 0, false, ax))) return rc;
    if ((rc = resolve(ctx, w_out, sizeof(double) * nn, 1, false, aw))) return rc;
    using GenKernel = void (*)(const double *, int, int, uint64_t, uint64_t, long long, const IntegrandDesc *,
                               double *, double *);
    GenKernel kern = k_vegas_generate<0, 1>;
    switch (D * 8 + ppt) {
#define CHILI_GEN(d)                                             \
    case d * 8 + 1: kern = k_vegas_generate<d, 1>; break;       \
    case d * 8 + 2: kern = k_vegas_generate<d, 2>; break;       \
    case d * 8 + 4: kern = k_vegas_generate<d, 4>; break;
        CHILI_GEN(1) CHILI_GEN(2) CHILI_GEN(3) CHILI_GEN(4) CHILI_GEN(5) CHILI_GEN(6) CHILI_GEN(7) CHILI_GEN(8)
        CHILI_GEN(10) CHILI_GEN(12) CHILI_GEN(16)
#undef CHILI_GEN
        default: ppt = 1; break;
    }
    if (smem > 48 * 1024)
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    int sms = 148, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kGenTile, smem));
    const long long tiles = (nn + static_cast<long long>(kGenTile) * ppt - 1) / (static_cast<long long>(kGenTile) * ppt);
    const long long nblocks = std::min<long long>(tiles, static_cast<long long>(sms) * std::max(per_sm, 1));
    {
        KTimer kt_(ctx, KT_VEGAS_GEN);
        kern<<<static_cast<unsigned>(nblocks), kGenTile, smem, ctx->stream>>>(
            ctx->edges.as<double>(), D, B, seed, counter_base, nn, ctx->f_dev.as<IntegrandDesc>(),
            static_cast<double *>(ax.dev), static_cast<double *>(aw.dev));
    }
    LAUNCHED();
    if ((rc = finish_out(ctx, ax)) || (rc = finish_out(ctx, aw))) return rc;
    return sync_if_host(ctx, {&ax, &aw});
}

// ------------------------------------------------------------------ channels
int chili_gpu_set_channels(chili_ctx *ctx, const chili_channel_desc *descs, int nch, const chili_cuts *cuts,
                           double sqrts, int n_ext) {
    if (!ctx) return fail(nullptr, CHILI_ERR_INVALID_ARG, "ctx is NULL");
    if (!(sqrts > 0)) return fail(ctx, CHILI_ERR_INVALID_ARG, "sqrts must be positive");
    std::vector<ChannelProgram> progs;
    const std::string why = build_channel_programs(descs, nch, cuts, sqrts, n_ext, progs);
    if (!why.empty()) return fail(ctx, CHILI_ERR_INVALID_ARG, why);
    int rc;
    if ((rc = set_device(ctx))) return rc;
    CK(ctx->progs.ensure(sizeof(ChannelProgram) * nch));
    CK(cudaMemcpyAsync(ctx->progs.p, progs.data(), sizeof(ChannelProgram) * nch, cudaMemcpyHostToDevice,
                       ctx->stream));
    ctx->nch = nch;
    ctx->n_ext = n_ext;
    ctx->ndims = progs[0].ndims;
    ctx->sqrts = sqrts;
    ctx->ch_info.assign(nch, {});
    ctx->ch_decays.assign(nch, {});
    ctx->ch_ptmin.assign(nch, {});
    for (int k = 0; k < nch; ++k) {
        ctx->ch_info[k].assign(descs[k].info, descs[k].info + descs[k].n_info);
        ctx->ch_decays[k].assign(descs[k].decays, descs[k].decays + descs[k].n_decays);
        ctx->ch_ptmin[k].assign(progs[k].info_ptmin, progs[k].info_ptmin + progs[k].n_info);
    }
    {
        std::vector<PointProgram> pp(1);
        ctx->have_pp = build_point_program(progs, pp[0]);
        if (ctx->have_pp) {
            ctx->pp_host = pp[0];
            CK(ctx->point_prog.ensure(sizeof(PointProgram)));
            CK(cudaMemcpyAsync(ctx->point_prog.p, pp.data(), sizeof(PointProgram), cudaMemcpyHostToDevice,
                               ctx->stream));
            k_pp_prepare<<<1, PP_MAX_DWS, 0, ctx->stream>>>(ctx->point_prog.as<PointProgram>());
            LAUNCHED();
            CK(cudaStreamSynchronize(ctx->stream));
        }
    }
    // alpha = 1/nch (MultiChannel.cc:62-67), best = alpha, min_diff = +inf
    std::vector<double> a(4 * CHILI_MAX_CHANNELS, 0.0);
    for (int i = 0; i < nch; ++i) a[i] = 1.0 / static_cast<double>(nch);
    a[3 * CHILI_MAX_CHANNELS] = INFINITY;
    CK(ctx->alpha_buf.ensure(sizeof(double) * a.size()));
    CK(cudaMemcpyAsync(ctx->alpha_buf.p, a.data(), sizeof(double) * a.size(), cudaMemcpyHostToDevice, ctx->stream));
    k_alpha_update<<<1, 32, 0, ctx->stream>>>(alpha_ptr(ctx), best_ptr(ctx), mindiff_ptr(ctx), cp_ptr(ctx), nullptr,
                                              nch, 0.0, 0.0, 0);
    LAUNCHED();
    ctx->alpha_set = true;
    // best_weights start empty in the reference; they read back as NaN until
    // the first MaxDifference update
    std::vector<double> nanv(nch, NAN);
    CK(cudaMemcpyAsync(best_ptr(ctx), nanv.data(), sizeof(double) * nch, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->g_nch > 0 && (ctx->g_nch != nch || ctx->dims != ctx->ndims)) {
        ctx->edges.release();
        ctx->g_nch = 0;
    }
    return CHILI_OK;
}

int chili_gpu_check_channels(const chili_channel_desc *descs, int nch, const chili_cuts *cuts, double sqrts,
                             int n_ext, char *err, size_t err_len) {
    std::vector<ChannelProgram> progs;
    std::string why = sqrts > 0 ? build_channel_programs(descs, nch, cuts, sqrts, n_ext, progs)
                                : std::string("sqrts must be positive");
    if (err && err_len) {
        std::strncpy(err, why.c_str(), err_len - 1);
        err[err_len - 1] = 0;
    }
    return why.empty() ? CHILI_OK : CHILI_ERR_INVALID_ARG;
}

int chili_gpu_ndims(const chili_ctx *ctx) { return ctx ? ctx->ndims : -1; }

int chili_gpu_fsmapper_generate(chili_ctx *ctx, int ch, const double *x, double *mom, int64_t n) {
    if (!ctx) return fail(nullptr, CHILI_ERR_INVALID_ARG, "ctx is NULL");
    int rc;
    if ((rc = need_channels(ctx))) return rc;
    if (ch < 0 || ch >= ctx->nch || !x || !mom || n < 0) return fail(ctx, CHILI_ERR_INVALID_ARG, "bad argument");
    if (n == 0) return CHILI_OK;
    Arg ax, am;
    if ((rc = resolve(ctx, x, sizeof(double) * n * ctx->ndims, 0, true, ax))) return rc;
    if ((rc = resolve(ctx, mom, sizeof(double) * n * ctx->n_ext * 4, 1, false, am))) return rc;
    k_fs_generate<<<grid_for(n, 128), 128, 0, ctx->stream>>>(ctx->progs.as<ChannelProgram>() + ch,
                                                             static_cast<const double *>(ax.dev),
                                                             static_cast<double *>(am.dev), n);
    LAUNCHED();
    if ((rc = finish_out(ctx, am))) return rc;
    return sync_if_host(ctx, {&ax, &am});
}

namespace {
int fsmapper_weight(chili_ctx *ctx, int ch, const double *mom, double *x, double *w, int64_t n, bool x_in) {
    if (!ctx) return fail(nullptr, CHILI_ERR_INVALID_ARG, "ctx is NULL");
    int rc;
    if ((rc = need_channels(ctx))) return rc;
    if (ch < 0 || ch >= ctx->nch || !mom || !w || n < 0 || (x_in && !x))
        return fail(ctx, CHILI_ERR_INVALID_ARG, "bad argument");
    if (n == 0) return CHILI_OK;
    Arg am, ax, aw;
    if ((rc = resolve(ctx, mom, sizeof(double) * n * ctx->n_ext * 4, 0, true, am))) return rc;
    if ((rc = resolve(ctx, x, sizeof(double) * n * ctx->ndims, 1, x_in, ax))) return rc;
    if ((rc = resolve(ctx, w, sizeof(double) * n, 2, false, aw))) return rc;
    k_fs_weight<<<grid_for(n, 128), 128, 0, ctx->stream>>>(ctx->progs.as<ChannelProgram>() + ch,
                                                           static_cast<const double *>(am.dev),
                                                           static_cast<double *>(ax.dev),
                                                           static_cast<double *>(aw.dev), n, x_in ? 1 : 0);
    LAUNCHED();
    if ((rc = finish_out(ctx, ax)) || (rc = finish_out(ctx, aw))) return rc;
    return sync_if_host(ctx, {&am, &ax, &aw});
}
}  // namespace

int chili_gpu_fsmapper_weight(chili_ctx *ctx, int ch, const double *mom, double *x_out, double *w, int64_t n) {
    return fsmapper_weight(ctx, ch, mom, x_out, w, n, false);
}

int chili_gpu_fsmapper_weight_inout(chili_ctx *ctx, int ch, const double *mom, double *x, double *w, int64_t n) {
    return fsmapper_weight(ctx, ch, mom, x, w, n, true);
}

// -------------------------------------------------------------- multichannel
int chili_gpu_set_alpha(chili_ctx *ctx, const double *alpha, int nch) {
    if (!ctx || !alpha) return fail(ctx, CHILI_ERR_INVALID_ARG, "NULL argument");
    int rc;
    if ((rc = need_channels(ctx))) return rc;
    if (nch != ctx->nch) return fail(ctx, CHILI_ERR_INVALID_ARG, "alpha length != channel count");
    Arg a;
    if ((rc = resolve(ctx, alpha, sizeof(double) * nch, 0, true, a))) return rc;
    CK(cudaMemcpyAsync(alpha_ptr(ctx), a.dev, sizeof(double) * nch, cudaMemcpyDeviceToDevice, ctx->stream));
    k_alpha_update<<<1, 32, 0, ctx->stream>>>(alpha_ptr(ctx), best_ptr(ctx), mindiff_ptr(ctx), cp_ptr(ctx), nullptr,
                                              nch, 0.0, 0.0, 0);
    LAUNCHED();
    CK(cudaStreamSynchronize(ctx->stream));
    return CHILI_OK;
}

int chili_gpu_get_alpha(chili_ctx *ctx, double *alpha, double *best_alpha, double *min_diff, int nch) {
    if (!ctx) return fail(nullptr, CHILI_ERR_INVALID_ARG, "ctx is NULL");
    int rc;
    if ((rc = need_channels(ctx))) return rc;
    if (nch != ctx->nch) return fail(ctx, CHILI_ERR_INVALID_ARG, "alpha length != channel count");
    std::vector<double> h(4 * CHILI_MAX_CHANNELS);
    CK(cudaMemcpyAsync(h.data(), ctx->alpha_buf.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (alpha) std::memcpy(alpha, h.data(), sizeof(double) * nch);
    if (best_alpha) std::memcpy(best_alpha, h.data() + CHILI_MAX_CHANNELS, sizeof(double) * nch);
    if (min_diff) *min_diff = h[3 * CHILI_MAX_CHANNELS];
    return CHILI_OK;
}

int chili_gpu_select_channel(chili_ctx *ctx, const double *v, int32_t *ich, int64_t n) {
    if (!ctx) return fail(nullptr, CHILI_ERR_INVALID_ARG, "ctx is NULL");
    int rc;
    if ((rc = need_channels(ctx))) return rc;
    if (!v || !ich || n < 0) return fail(ctx, CHILI_ERR_INVALID_ARG, "bad argument");
    if (n == 0) return CHILI_OK;
    Arg av, ai;
    if ((rc = resolve(ctx, v, sizeof(double) * n, 0, true, av))) return rc;
    if ((rc = resolve(ctx, ich, sizeof(int32_t) * n, 1, false, ai))) return rc;
    k_select<<<grid_for(n, 256), 256, 0, ctx->stream>>>(cp_ptr(ctx), ctx->nch, static_cast<const double *>(av.dev),
                                                        static_cast<int32_t *>(ai.dev), n);
    LAUNCHED();
    if ((rc = finish_out(ctx, ai))) return rc;
    return sync_if_host(ctx, {&av, &ai});
}

static int need_mc(chili_ctx *ctx) {
    int rc;
    if ((rc = need_channels(ctx))) return rc;
    if ((rc = need_grids(ctx))) return rc;
    if (ctx->g_nch != ctx->nch || ctx->dims != ctx->ndims)
        return fail(ctx, CHILI_ERR_STATE, "grids do not match the channels (nch x ndims)");
    return CHILI_OK;
}

int chili_gpu_multichannel_weight(chili_ctx *ctx, const double *mom, const int32_t *ich, double *wgt, double *dens,
                                  double *x_ich, int64_t n) {
    if (!ctx) return fail(nullptr, CHILI_ERR_INVALID_ARG, "ctx is NULL");
    int rc;
    if ((rc = need_mc(ctx))) return rc;
    if (!mom || !ich || !wgt || n < 0) return fail(ctx, CHILI_ERR_INVALID_ARG, "bad argument");
    if (n == 0) return CHILI_OK;
    Arg am, ai, aw, ad, ax;
    if ((rc = resolve(ctx, mom, sizeof(double) * n * ctx->n_ext * 4, 0, true, am))) return rc;
    if ((rc = resolve(ctx, ich, sizeof(int32_t) * n, 1, true, ai))) return rc;
    if ((rc = resolve(ctx, wgt, sizeof(double) * n, 2, false, aw))) return rc;
    if ((rc = resolve(ctx, dens, sizeof(double) * n * ctx->nch, 3, false, ad))) return rc;
    if ((rc = resolve(ctx, x_ich, sizeof(double) * n * ctx->ndims, 4, false, ax))) return rc;
    k_mc_weight_batch<<<grid_for(n, 128), 128, 0, ctx->stream>>>(
        ctx->progs.as<ChannelProgram>(), ctx->edges.as<double>(), alpha_ptr(ctx), ctx->nch, ctx->ndims, ctx->bins,
        ctx->n_ext, static_cast<const double *>(am.dev), static_cast<const int32_t *>(ai.dev),
        static_cast<double *>(aw.dev), static_cast<double *>(ad.dev), static_cast<double *>(ax.dev), n, pp_ptr(ctx));
    LAUNCHED();
    if ((rc = finish_out(ctx, aw)) || (rc = finish_out(ctx, ad)) || (rc = finish_out(ctx, ax))) return rc;
    return sync_if_host(ctx, {&am, &ai, &aw, &ad, &ax});
}

int chili_gpu_multichannel_iterate(chili_ctx *ctx, const chili_multichannel_params *params, uint64_t seed,
                                   uint64_t counter_base, const double *u, int64_t n_u, int guard_alpha,
                                   chili_stats *stats_out, chili_mc_iter_info *info) {
    if (!ctx) return fail(nullptr, CHILI_ERR_INVALID_ARG, "ctx is NULL");
    int rc;
    if ((rc = need_mc(ctx))) return rc;
    if (!params) return fail(ctx, CHILI_ERR_INVALID_ARG, "params is NULL");
    if (!ctx->f_set) return fail(ctx, CHILI_ERR_STATE, "no integrand set");
    if (ctx->f_host.kind == CHILI_FUNC_CAMEL) return fail(ctx, CHILI_ERR_STATE, "the camel is not a phase-space integrand");
    if (u && n_u <= 0) return fail(ctx, CHILI_ERR_INVALID_ARG, "n_u must be positive when u is given");
    const long long ncalls = static_cast<long long>(params->ncalls);
    if (ncalls < 1) return fail(ctx, CHILI_ERR_INVALID_ARG, "ncalls must be positive");
    const int nch = ctx->nch, D = ctx->ndims, B = ctx->bins, NE = ctx->n_ext;
    const bool opt = params->should_optimize != 0;
    // uniforms in device memory are read in place; host uniforms are staged
    // chunk by chunk, only the rows the chunk consumes
    const double *ud = nullptr;
    const bool u_host = u && !is_device_ptr(u);
    if (u && !u_host) ud = u;
    const size_t hist_n = static_cast<size_t>(nch) * D * B;
    CK(ctx->hist.ensure(sizeof(double) * hist_n));
    CK(ctx->acc.ensure(sizeof(IterAcc)));
    CK(ctx->ctl.ensure(sizeof(RoundCtl)));
    CK(ctx->round_res.ensure(sizeof(double) * (kPartFixed + nch)));
    CK(cudaMemsetAsync(ctx->hist.p, 0, sizeof(double) * hist_n, ctx->stream));
    {
        IterAcc a0{};
        a0.st[1] = 1.7976931348623157e308;  // StatsData min = lim::max()
        a0.st[2] = 2.2250738585072014e-308; // StatsData max = lim::min()
        CK(cudaMemcpyAsync(ctx->acc.p, &a0, sizeof(IterAcc), cudaMemcpyHostToDevice, ctx->stream));
    }
    const size_t acc_smem = sizeof(double) * (kWgtBlock / 32) * nch;
    // the histogram adds staged in shared memory when one block can hold the
    // whole histogram (option "hist_shared")
    const bool hist_smem = ctx->hist_shared && sizeof(double) * hist_n <= static_cast<size_t>(ctx->max_smem_optin);

    long long needed = ncalls, tried = 0, weighted = 0, drawn = 0, chunks = 0;
    unsigned long long rounds = 0;
    const bool pipe = pipeline_dims_ok(D) && ctx->have_pp && ctx->use_pp && ctx->use_pipeline;
    if (u_host) CK(ctx->iter_ctl.ensure(sizeof(long long) * kIterCtl));
    long long *iter = ctx->iter_ctl.as<long long>();
    while (needed > 0) {
        // chunk: enough counters for `needed` accepted, non-NaN points at the
        // rates of the previous iteration, with a 2% margin
        const double rate = std::max(ctx->accept_rate * (1.0 - ctx->nan_rate), 0.02);
        long long m = static_cast<long long>(static_cast<double>(needed) / rate * 1.02) + 2048;
        m = std::min<long long>(m, 1ll << 24);
        {
            // keep the per-chunk buffers within ~8 GB
            const PointProgram &P = ctx->pp_host;
            long long per = 8ll * (4 * NE + nch + 4) + 4ll * D + 8;
            if (pipe) per += 8ll * (4 * P.n_nodes + P.n_memo) + P.n_chains;
            m = std::min<long long>(m, std::max<long long>(1 << 16, (8ll << 30) / per));
        }
        if (u) {
            m = std::min<long long>(m, n_u - tried);
            if (m <= 0) return fail(ctx, CHILI_ERR_LIMIT, "the given uniforms ran out before ncalls points were accepted");
        }
        // Host uniforms: the chunk's rows are uploaded in slices and every
        // slice is queued as one round without a host round trip; the device
        // keeps the count still needed and the chunk's totals (iter), and the
        // rounds after the one that completes the iteration do no work.
        // Otherwise the chunk is one round, its record read back at its end.
        const std::vector<long long> sb = u_host ? slice_bounds(m, ctx->upload_slice) : std::vector<long long>{0, m};
        const long long S = u_host ? std::min(m, std::max(ctx->upload_slice, kFirstSlice)) : m;  // rows of the largest round
        const long long n_rounds = static_cast<long long>(sb.size()) - 1;
        drawn += m;
        ++chunks;
        if (u_host) {
            // the gate is set before upload_host records the event the
            // slice copies (and so every forward launch of the chunk, on
            // the forward stream) wait on
            k_iter_init<<<1, 1, 0, ctx->stream>>>(iter, needed);
            LAUNCHED();
            if ((rc = upload_host(ctx, u + tried * (D + 1), m, sb))) return rc;
        }
        // buffers for a whole number of 2^16 points (the chunk size follows
        // the acceptance rate and would otherwise reallocate, synchronising
        // the device, whenever it grows a little)
        const long long Sa = (S + 65535) / 65536 * 65536;
        const long long nb_f = (Sa + kFwdBlock - 1) / kFwdBlock;
        const long long nb_w = (Sa + kWgtBlock - 1) / kWgtBlock;
        CK(ctx->mom_soa.ensure(sizeof(double) * 4 * NE * Sa));
        CK(ctx->ich.ensure(sizeof(int32_t) * Sa));
        CK(ctx->flag.ensure(Sa));
        CK(ctx->list.ensure(sizeof(int32_t) * Sa));
        CK(ctx->block_count.ensure(sizeof(int32_t) * nb_f));
        CK(ctx->block_off.ensure(sizeof(long long) * nb_f));
        CK(ctx->part.ensure(sizeof(double) * (kPartFixed + nch) * nb_w));
        CK(ctx->rec.ensure(Sa * (2 * sizeof(double) + 1 + sizeof(int32_t) * D + sizeof(double) * nch) + 256));
        CK(ctx->ctl3.ensure(3 * sizeof(RoundCtl)));
        RoundCtl *ctl_pre = ctx->ctl3.as<RoundCtl>(), *ctl_list = ctl_pre + 1;
        if (u_host) {
            // the second set of forward buffers and the forward stream
            CK(ctx->mom_soa_alt.ensure(sizeof(double) * 4 * NE * Sa));
            CK(ctx->ich_alt.ensure(sizeof(int32_t) * Sa));
            CK(ctx->flag_alt.ensure(Sa));
            CK(ctx->block_count_alt.ensure(sizeof(int32_t) * nb_f));
            if (!ctx->fwd_stream) {
                CK(cudaStreamCreateWithFlags(&ctx->fwd_stream, cudaStreamNonBlocking));
                for (int k = 0; k < 2; ++k) {
                    CK(cudaEventCreateWithFlags(&ctx->fwd_done[k], cudaEventDisableTiming));
                    CK(cudaEventCreateWithFlags(&ctx->round_done[k], cudaEventDisableTiming));
                }
            }
        }
        for (long long q = 0; q < n_rounds; ++q) {
            // this round's rows of the chunk: [r0, r0 + mm)
            const long long r0 = sb[q];
            const long long mm = sb[q + 1] - r0;
            const long long nbf = (mm + kFwdBlock - 1) / kFwdBlock, nbw = (mm + kWgtBlock - 1) / kWgtBlock;
            const long long *gate = u_host ? iter : nullptr;
            // records with stride mm
            double *rec_val = ctx->rec.as<double>();
            double *rec_wgt = rec_val + mm;
            double *rec_dens = rec_wgt + mm;
            int32_t *rec_slot = reinterpret_cast<int32_t *>(rec_dens + static_cast<size_t>(nch) * mm);
            uint8_t *rec_ok = reinterpret_cast<uint8_t *>(rec_slot + static_cast<size_t>(D) * mm);
            // host-uniform rounds alternate between two sets of forward
            // buffers, so that the forward pass of round q + 1 (on the
            // forward stream) runs beside the weight pass of round q
            const int par = u_host ? static_cast<int>(q & 1) : 0;
            double *mom = (par ? ctx->mom_soa_alt : ctx->mom_soa).as<double>();
            int32_t *ich = (par ? ctx->ich_alt : ctx->ich).as<int32_t>();
            uint8_t *flag = (par ? ctx->flag_alt : ctx->flag).as<uint8_t>();
            int32_t *bcount = (par ? ctx->block_count_alt : ctx->block_count).as<int32_t>();
            {
                const double *u_in = ud ? ud + (tried + r0) * (D + 1) : nullptr;
                const cudaStream_t main = ctx->stream;
                if (u_host) {
                    // the forward launch waits (on the device) for its slice's
                    // copy and for the round that last used its buffers
                    CK(cudaStreamWaitEvent(ctx->fwd_stream, ctx->copy_events[q], 0));
                    if (q >= 2) CK(cudaStreamWaitEvent(ctx->fwd_stream, ctx->round_done[par], 0));
                    u_in = ctx->stage[0].as<double>() + r0 * (D + 1);
                    ctx->stream = ctx->fwd_stream;
                }
                {
                    KTimer kt_(ctx, KT_FORWARD);
                    k_mc_forward<<<static_cast<unsigned>(nbf), kFwdBlock, 0, ctx->stream>>>(
                        ctx->progs.as<ChannelProgram>(), ctx->edges.as<double>(), cp_ptr(ctx), nch, D, B, seed,
                        counter_base + tried + r0, u_in, mm, ctx->f_dev.as<IntegrandDesc>(), NE, mom, ich, flag,
                        bcount, gate);
                }
                ctx->stream = main;
                LAUNCHED();
                if (u_host) {
                    CK(cudaEventRecord(ctx->fwd_done[par], ctx->fwd_stream));
                    CK(cudaStreamWaitEvent(main, ctx->fwd_done[par], 0));
                }
            }
            // offsets of every PreProcess-accepted point (no cut at this stage)
            {
                KTimer kt_(ctx, KT_ROUND_OTHER);
                k_mc_scan<<<1, 1024, 0, ctx->stream>>>(bcount, static_cast<int>(nbf), flag, mm, mm + 1, gate, 0,
                                                       ctx->block_off.as<long long>(), ctl_pre);
                LAUNCHED();
                k_mc_compact<<<static_cast<unsigned>(nbf), kFwdBlock, 0, ctx->stream>>>(
                    flag, ctx->block_off.as<long long>(), ctl_pre, mm, ctx->list.as<int32_t>());
                LAUNCHED();
            }
            if (pipe) {
                // the launches are sized by the accepted count, read back here;
                // a queued host-uniform round (or any round with the option
                // "pipeline_sync" 0) does not wait for it: its launches cover
                // all mm points and the threads past the device-side count
                // return at once
                long long n_pre = mm;
                if ((!u_host && ctx->pipe_sync) || mm > ctx->pipe_tile) {
                    CK(cudaMemcpyAsync(ctx->ctl_host, ctl_pre, sizeof(RoundCtl), cudaMemcpyDeviceToHost,
                                       ctx->stream));
                    CK(cudaStreamSynchronize(ctx->stream));
                    n_pre = ctx->ctl_host->n_acc;
                }
                int rc2 = launch_pipeline(ctx, mom, ich, mm, n_pre, B, opt, ctl_pre, rec_val, rec_wgt, rec_ok,
                                          rec_slot, rec_dens);
                if (rc2) return rc2;
            } else {
                KTimer kt_(ctx, KT_WEIGHT);
                k_mc_weight<<<static_cast<unsigned>(nbw), kWgtBlock, 0, ctx->stream>>>(
                    ctx->progs.as<ChannelProgram>(), ctx->edges.as<double>(), alpha_ptr(ctx), nch, D, B, NE,
                    mom, mm, ich, ctx->list.as<int32_t>(), ctl_pre, ctx->f_dev.as<IntegrandDesc>(), opt ? 1 : 0,
                    rec_val, rec_wgt, rec_ok, rec_slot, rec_dens, pp_ptr(ctx));
                LAUNCHED();
            }
            // the cut: the needed-th record whose value is not NaN (the
            // device's count when the rounds are queued)
            {
                KTimer kt_(ctx, KT_ROUND_OTHER);
                k_block_count<<<static_cast<unsigned>(nbf), kFwdBlock, 0, ctx->stream>>>(rec_ok, ctl_pre, bcount);
                LAUNCHED();
                k_mc_scan<<<1, 1024, 0, ctx->stream>>>(bcount, static_cast<int>(nbf), rec_ok, mm, needed, gate, 1,
                                                       ctx->block_off.as<long long>(), ctl_list);
                LAUNCHED();
                k_cut_finalize<<<1, 1, 0, ctx->stream>>>(ctl_list, ctl_pre, ctx->list.as<int32_t>(), mm, needed,
                                                         u_host ? iter : nullptr, ctx->ctl.as<RoundCtl>());
                LAUNCHED();
            }
            {
                KTimer kt_(ctx, KT_ACCUM);
                k_mc_accum<<<static_cast<unsigned>(nbw), kWgtBlock, acc_smem, ctx->stream>>>(
                    ctx->ctl.as<RoundCtl>(), mm, nch, D, static_cast<int>(hist_n), rec_val, rec_wgt, rec_ok, rec_slot,
                    rec_dens, opt ? 1 : 0, guard_alpha ? 1 : 0, hist_smem ? nullptr : ctx->hist.as<double>(),
                    ctx->part.as<double>());
                LAUNCHED();
                if (hist_smem && opt) {
                    k_mc_hist<<<static_cast<unsigned>(std::min<long long>(nbw, ctx->sms)), 1024,
                                sizeof(double) * hist_n, ctx->stream>>>(ctx->ctl.as<RoundCtl>(), mm, D,
                                                                        static_cast<int>(hist_n), rec_val, rec_slot,
                                                                        ctx->hist.as<double>());
                    LAUNCHED();
                }
            }
            {
                KTimer kt_(ctx, KT_ROUND_OTHER);
                k_mc_reduce<<<kPartFixed + nch, 256, 0, ctx->stream>>>(ctx->part.as<double>(), nch,
                                                                       ctx->ctl.as<RoundCtl>(),
                                                                       ctx->round_res.as<double>());
                LAUNCHED();
                k_mc_accumulate<<<1, 256, 0, ctx->stream>>>(ctx->round_res.as<double>(), nch,
                                                            ctx->ctl.as<RoundCtl>(), ctx->acc.as<IterAcc>());
                LAUNCHED();
            }
            if (u_host) {
                CK(cudaEventRecord(ctx->round_done[par], ctx->stream));
                continue;
            }
            CK(cudaMemcpyAsync(ctx->ctl_host, ctx->ctl.p, sizeof(RoundCtl), cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaMemcpyAsync(ctx->ctl_host + 1, ctl_pre, sizeof(RoundCtl), cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
            if (ctx->timing) collect_times(ctx);
            const RoundCtl r = ctx->ctl_host[0];
            if (r.cut <= 0 || r.cut > mm || r.n_acc < 0 || r.nan_round < 0 || r.nan_round > r.n_acc)
                return fail(ctx, CHILI_ERR_CUDA, "inconsistent round record");
            tried += r.cut;
            needed -= (r.n_acc - r.nan_round);
            weighted += ctx->ctl_host[1].n_acc;
            ctx->accept_rate = std::max(0.02, static_cast<double>(r.n_acc) / static_cast<double>(r.cut));
            if (r.n_acc > 0) ctx->nan_rate = std::min(0.5, static_cast<double>(r.nan_round) / static_cast<double>(r.n_acc));
        }
        if (u_host) {
            // the queued rounds' totals
            CK(cudaMemcpyAsync(ctx->iter_host, iter, sizeof(long long) * kIterCtl, cudaMemcpyDeviceToHost,
                               ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
            if (ctx->timing) collect_times(ctx);
            const long long *t = ctx->iter_host;  // remaining, tried, accepted, NaN, weighted
            if (t[1] <= 0 || t[1] > m || t[2] < 0 || t[3] < 0 || t[3] > t[2] || t[0] > needed ||
                needed - t[0] != t[2] - t[3])
                return fail(ctx, CHILI_ERR_CUDA, "inconsistent round record");
            tried += t[1];
            needed = t[0];
            weighted += t[4];
            ctx->accept_rate = std::max(0.02, static_cast<double>(t[2]) / static_cast<double>(t[1]));
            if (t[2] > 0) ctx->nan_rate = std::min(0.5, static_cast<double>(t[3]) / static_cast<double>(t[2]));
        }
        rounds += static_cast<unsigned long long>(n_rounds);
        if (rounds > static_cast<unsigned long long>(ctx->max_rounds))
            return fail(ctx, CHILI_ERR_TIMEOUT, "ncalls not reached after max_rounds rounds (every point rejected or NaN?)");
    }
    IterAcc acc_h;
    if (opt && !ctx->defer_train) {
        KTimer kt_(ctx, KT_ITER_END);
        k_alpha_update<<<1, 32, 0, ctx->stream>>>(alpha_ptr(ctx), best_ptr(ctx), mindiff_ptr(ctx), cp_ptr(ctx),
                                                  acc_train_ptr(ctx), nch, params->beta,
                                                  params->min_alpha, 1);
        LAUNCHED();
        if ((rc = adapt_grids(ctx, 0, nch, params->grid_alpha, ctx->hist.as<double>(), 1))) return rc;
    }
    CK(cudaMemcpyAsync(&acc_h, ctx->acc.p, sizeof(IterAcc), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (stats_out) std::memcpy(stats_out, acc_h.st, sizeof(chili_stats));
    if (info) {
        info->points_tried = static_cast<uint64_t>(tried);
        info->points_accepted = static_cast<uint64_t>(ncalls);
        info->rejected_pre = static_cast<uint64_t>(acc_h.rejected_pre);
        info->rejected_nan = static_cast<uint64_t>(acc_h.nan_count);
        info->weight_max = acc_h.wmax;
        info->nonfinite_alpha_terms = acc_h.nonfinite;
        info->points_weighted = static_cast<uint64_t>(weighted);
        info->points_drawn = static_cast<uint64_t>(drawn);
        info->chunks = static_cast<uint64_t>(chunks);
    }
    return CHILI_OK;
}

int chili_gpu_multichannel_train(chili_ctx *ctx, const chili_multichannel_params *params, const double *hist,
                                 const double *alpha_train) {
    if (!ctx || !params || !hist || !alpha_train) return fail(ctx, CHILI_ERR_INVALID_ARG, "NULL argument");
    int rc;
    if ((rc = set_device(ctx))) return rc;
    if ((rc = need_mc(ctx))) return rc;
    const int nch = ctx->nch;
    const size_t hist_n = static_cast<size_t>(nch) * ctx->ndims * ctx->bins;
    CK(ctx->hist.ensure(sizeof(double) * hist_n));
    CK(ctx->acc.ensure(sizeof(IterAcc)));
    Arg ah, aa;
    if ((rc = resolve(ctx, hist, sizeof(double) * hist_n, 0, true, ah))) return rc;
    if ((rc = resolve(ctx, alpha_train, sizeof(double) * nch, 1, true, aa))) return rc;
    CK(cudaMemcpyAsync(ctx->hist.p, ah.dev, sizeof(double) * hist_n, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(acc_train_ptr(ctx), aa.dev, sizeof(double) * nch, cudaMemcpyDeviceToDevice, ctx->stream));
    k_alpha_update<<<1, 32, 0, ctx->stream>>>(alpha_ptr(ctx), best_ptr(ctx), mindiff_ptr(ctx), cp_ptr(ctx),
                                              acc_train_ptr(ctx), nch, params->beta, params->min_alpha, 1);
    LAUNCHED();
    if ((rc = adapt_grids(ctx, 0, nch, params->grid_alpha, ctx->hist.as<double>(), 1))) return rc;
    // host inputs were staged: their buffers are free once the copies ran
    return sync_if_host(ctx, {&ah, &aa});
}

int chili_gpu_get_training(chili_ctx *ctx, double *hist, double *alpha_train) {
    if (!ctx) return fail(nullptr, CHILI_ERR_INVALID_ARG, "ctx is NULL");
    int rc;
    if ((rc = need_mc(ctx))) return rc;
    if (!ctx->hist.p || !ctx->acc.p) return fail(ctx, CHILI_ERR_STATE, "no iteration has run");
    const size_t hist_n = static_cast<size_t>(ctx->nch) * ctx->ndims * ctx->bins;
    Arg ah, aa;
    if ((rc = resolve(ctx, hist, sizeof(double) * hist_n, 0, false, ah))) return rc;
    if ((rc = resolve(ctx, alpha_train, sizeof(double) * ctx->nch, 1, false, aa))) return rc;
    if (hist) CK(cudaMemcpyAsync(ah.dev, ctx->hist.p, sizeof(double) * hist_n, cudaMemcpyDeviceToDevice, ctx->stream));
    if (alpha_train)
        CK(cudaMemcpyAsync(aa.dev, acc_train_ptr(ctx), sizeof(double) * ctx->nch,
                           cudaMemcpyDeviceToDevice, ctx->stream));
    if ((rc = finish_out(ctx, ah)) || (rc = finish_out(ctx, aa))) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return CHILI_OK;
}

namespace {
// [hist | atrain | n, sum, sum2, n_finite | max, -min] of the last iteration
__global__ void k_pack_training(const double *__restrict__ hist, long long hist_n, const IterAcc *__restrict__ acc,
                                int nch, double *__restrict__ buf) {
    const long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (t < hist_n) buf[t] = hist[t];
    if (t < nch) buf[hist_n + t] = acc->atrain[t];
    if (t == 0) {
        double *s = buf + hist_n + nch;
        s[0] = acc->st[0];
        s[1] = acc->st[3];
        s[2] = acc->st[4];
        s[3] = acc->st[5];
        s[4] = acc->st[2];
        s[5] = -acc->st[1];
    }
}
}  // namespace

int chili_gpu_pack_training(chili_ctx *ctx, double *buf, int64_t len) {
    if (!ctx || !buf) return fail(ctx, CHILI_ERR_INVALID_ARG, "NULL argument");
    int rc;
    if ((rc = need_mc(ctx))) return rc;
    if (!ctx->hist.p || !ctx->acc.p) return fail(ctx, CHILI_ERR_STATE, "no iteration has run");
    const long long hist_n = static_cast<long long>(ctx->nch) * ctx->ndims * ctx->bins;
    const long long need = hist_n + ctx->nch + 6;
    if (len < need) return fail(ctx, CHILI_ERR_INVALID_ARG, "buffer shorter than nch*dims*bins + nch + 6");
    Arg ab;
    if ((rc = resolve(ctx, buf, sizeof(double) * need, 0, false, ab))) return rc;
    const long long nt = std::max<long long>(hist_n, ctx->nch);
    k_pack_training<<<grid_for(nt, 256), 256, 0, ctx->stream>>>(ctx->hist.as<double>(), hist_n,
                                                                ctx->acc.as<IterAcc>(), ctx->nch,
                                                                static_cast<double *>(ab.dev));
    LAUNCHED();
    if ((rc = finish_out(ctx, ab))) return rc;
    return sync_if_host(ctx, {&ab});
}

int chili_gpu_generate(chili_ctx *ctx, int64_t n, uint64_t seed, uint64_t counter_base, double *mom, double *wgt,
                       int32_t *ch) {
    if (!ctx) return fail(nullptr, CHILI_ERR_INVALID_ARG, "ctx is NULL");
    int rc;
    if ((rc = need_mc(ctx))) return rc;
    if (!ctx->f_set) return fail(ctx, CHILI_ERR_STATE, "no integrand set");
    if (n < 0) return fail(ctx, CHILI_ERR_INVALID_ARG, "n < 0");
    if (n == 0) return CHILI_OK;
    Arg am, aw, ac;
    if ((rc = resolve(ctx, mom, sizeof(double) * n * ctx->n_ext * 4, 0, false, am))) return rc;
    if ((rc = resolve(ctx, wgt, sizeof(double) * n, 1, false, aw))) return rc;
    if ((rc = resolve(ctx, ch, sizeof(int32_t) * n, 2, false, ac))) return rc;
    k_generate<<<grid_for(n, 128), 128, 0, ctx->stream>>>(
        ctx->progs.as<ChannelProgram>(), ctx->edges.as<double>(), alpha_ptr(ctx), cp_ptr(ctx), ctx->nch, ctx->ndims,
        ctx->bins, ctx->n_ext, seed, counter_base, n, ctx->f_dev.as<IntegrandDesc>(), static_cast<double *>(am.dev),
        static_cast<double *>(aw.dev), static_cast<int32_t *>(ac.dev), pp_ptr(ctx));
    LAUNCHED();
    if ((rc = finish_out(ctx, am)) || (rc = finish_out(ctx, aw)) || (rc = finish_out(ctx, ac))) return rc;
    return sync_if_host(ctx, {&am, &aw, &ac});
}

int chili_gpu_generate_unweighted(chili_ctx *ctx, int64_t n, uint64_t seed, uint64_t counter_base, double w_max,
                                  double *mom, double *wgt, int32_t *ch, int64_t max_events, int64_t *n_events,
                                  chili_unweight_info *info) {
    if (!ctx) return fail(nullptr, CHILI_ERR_INVALID_ARG, "ctx is NULL");
    int rc;
    if ((rc = need_mc(ctx))) return rc;
    if (!ctx->f_set) return fail(ctx, CHILI_ERR_STATE, "no integrand set");
    if (ctx->f_host.kind == CHILI_FUNC_CAMEL) return fail(ctx, CHILI_ERR_STATE, "the camel is not a phase-space integrand");
    if (n < 0 || max_events < 0) return fail(ctx, CHILI_ERR_INVALID_ARG, "n and max_events must be >= 0");
    if (!(w_max > 0) || !std::isfinite(w_max)) return fail(ctx, CHILI_ERR_INVALID_ARG, "w_max must be finite and > 0");
    const int nch = ctx->nch, D = ctx->ndims, B = ctx->bins, NE = ctx->n_ext;
    Arg am, aw, ac;
    if ((rc = resolve(ctx, mom, sizeof(double) * max_events * NE * 4, 0, false, am))) return rc;
    if ((rc = resolve(ctx, wgt, sizeof(double) * max_events, 1, false, aw))) return rc;
    if ((rc = resolve(ctx, ch, sizeof(int32_t) * max_events, 2, false, ac))) return rc;
    const bool pipe = pipeline_dims_ok(D) && ctx->have_pp && ctx->use_pp && ctx->use_pipeline;
    long long done = 0, kept = 0, n_pre_tot = 0;
    double sum = 0, over = 0, vmax = -1.7976931348623157e308;
    while (done < n) {
        long long m = std::min<long long>(n - done, 1ll << 24);
        {
            // keep the per-chunk buffers within ~8 GB, as an iteration does
            const PointProgram &P = ctx->pp_host;
            long long per = 8ll * (4 * NE + nch + 4) + 4ll * D + 16;
            if (pipe) per += 8ll * (4 * P.n_nodes + P.n_memo) + P.n_chains;
            m = std::min<long long>(m, std::max<long long>(1 << 16, (8ll << 30) / per));
        }
        const long long nb_f = (m + kFwdBlock - 1) / kFwdBlock;
        const long long nb_w = (m + kWgtBlock - 1) / kWgtBlock;
        CK(ctx->mom_soa.ensure(sizeof(double) * 4 * NE * m));
        CK(ctx->ich.ensure(sizeof(int32_t) * m));
        CK(ctx->flag.ensure(m));
        CK(ctx->list.ensure(sizeof(int32_t) * m));
        CK(ctx->block_count.ensure(sizeof(int32_t) * nb_f));
        CK(ctx->block_off.ensure(sizeof(long long) * nb_f));
        CK(ctx->rec.ensure(m * (2 * sizeof(double) + 1 + sizeof(int32_t) * D + sizeof(double) * nch) + 256));
        CK(ctx->ctl3.ensure(3 * sizeof(RoundCtl)));
        // keep flags [m] | kept list [m] | partials [nb_f][3] | sums [3] | control
        const size_t off_list = (static_cast<size_t>(m) + 15) & ~static_cast<size_t>(15);
        const size_t off_part = off_list + sizeof(int32_t) * ((static_cast<size_t>(m) + 3) & ~static_cast<size_t>(3));
        const size_t off_out = off_part + sizeof(double) * 3 * nb_f;
        const size_t off_ctl = off_out + sizeof(double) * 4;
        CK(ctx->unw.ensure(off_ctl + sizeof(RoundCtl)));
        char *ub = ctx->unw.as<char>();
        uint8_t *keep = reinterpret_cast<uint8_t *>(ub);
        int32_t *kept_list = reinterpret_cast<int32_t *>(ub + off_list);
        double *part = reinterpret_cast<double *>(ub + off_part);
        double *outs = reinterpret_cast<double *>(ub + off_out);
        RoundCtl *ctl_keep = reinterpret_cast<RoundCtl *>(ub + off_ctl);
        RoundCtl *ctl_pre = ctx->ctl3.as<RoundCtl>();
        double *rec_val = ctx->rec.as<double>();
        double *rec_wgt = rec_val + m;
        double *rec_dens = rec_wgt + m;
        int32_t *rec_slot = reinterpret_cast<int32_t *>(rec_dens + static_cast<size_t>(nch) * m);
        uint8_t *rec_ok = reinterpret_cast<uint8_t *>(rec_slot + static_cast<size_t>(D) * m);
        const uint64_t ctr0 = counter_base + static_cast<uint64_t>(done);
        k_mc_forward<<<static_cast<unsigned>(nb_f), kFwdBlock, 0, ctx->stream>>>(
            ctx->progs.as<ChannelProgram>(), ctx->edges.as<double>(), cp_ptr(ctx), nch, D, B, seed, ctr0, nullptr, m,
            ctx->f_dev.as<IntegrandDesc>(), NE, ctx->mom_soa.as<double>(), ctx->ich.as<int32_t>(),
            ctx->flag.as<uint8_t>(), ctx->block_count.as<int32_t>(), nullptr);
        LAUNCHED();
        k_mc_scan<<<1, 1024, 0, ctx->stream>>>(ctx->block_count.as<int32_t>(), static_cast<int>(nb_f),
                                               ctx->flag.as<uint8_t>(), m, m + 1, nullptr, 0,
                                               ctx->block_off.as<long long>(), ctl_pre);
        LAUNCHED();
        k_mc_compact<<<static_cast<unsigned>(nb_f), kFwdBlock, 0, ctx->stream>>>(
            ctx->flag.as<uint8_t>(), ctx->block_off.as<long long>(), ctl_pre, m, ctx->list.as<int32_t>());
        LAUNCHED();
        CK(cudaMemcpyAsync(ctx->ctl_host, ctl_pre, sizeof(RoundCtl), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        const long long n_pre = ctx->ctl_host->n_acc;
        if (n_pre < 0 || n_pre > m) return fail(ctx, CHILI_ERR_CUDA, "inconsistent point list");
        n_pre_tot += n_pre;
        if (pipe) {
            if ((rc = launch_pipeline(ctx, ctx->mom_soa.as<double>(), ctx->ich.as<int32_t>(), m, n_pre, B, false,
                                      ctl_pre, rec_val, rec_wgt, rec_ok, rec_slot, rec_dens)))
                return rc;
        } else {
            k_mc_weight<<<static_cast<unsigned>(nb_w), kWgtBlock, 0, ctx->stream>>>(
                ctx->progs.as<ChannelProgram>(), ctx->edges.as<double>(), alpha_ptr(ctx), nch, D, B, NE,
                ctx->mom_soa.as<double>(), m, ctx->ich.as<int32_t>(), ctx->list.as<int32_t>(), ctl_pre,
                ctx->f_dev.as<IntegrandDesc>(), 0, rec_val, rec_wgt, rec_ok, rec_slot, rec_dens, pp_ptr(ctx));
            LAUNCHED();
        }
        k_unw_flag<<<static_cast<unsigned>(nb_f), kFwdBlock, 0, ctx->stream>>>(
            ctx->list.as<int32_t>(), ctl_pre, rec_val, seed, ctr0, w_max, m, keep, part);
        LAUNCHED();
        k_unw_reduce<<<1, 256, 0, ctx->stream>>>(part, nb_f, outs);
        LAUNCHED();
        k_block_count<<<static_cast<unsigned>(nb_f), kFwdBlock, 0, ctx->stream>>>(keep, ctl_pre,
                                                                                 ctx->block_count.as<int32_t>());
        LAUNCHED();
        k_mc_scan<<<1, 1024, 0, ctx->stream>>>(ctx->block_count.as<int32_t>(), static_cast<int>(nb_f), keep, m,
                                               m + 1, nullptr, 0, ctx->block_off.as<long long>(), ctl_keep);
        LAUNCHED();
        k_mc_compact<<<static_cast<unsigned>(nb_f), kFwdBlock, 0, ctx->stream>>>(
            keep, ctx->block_off.as<long long>(), ctl_keep, m, kept_list);
        LAUNCHED();
        k_unw_write<<<static_cast<unsigned>(nb_f), kFwdBlock, 0, ctx->stream>>>(
            kept_list, ctl_keep, ctx->list.as<int32_t>(), ctx->mom_soa.as<double>(), m, NE, ctx->ich.as<int32_t>(),
            rec_val, w_max, kept, max_events, static_cast<double *>(am.dev), static_cast<double *>(aw.dev),
            static_cast<int32_t *>(ac.dev));
        LAUNCHED();
        double h[3];
        RoundCtl rk;
        CK(cudaMemcpyAsync(h, outs, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(&rk, ctl_keep, sizeof(RoundCtl), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (rk.n_acc < 0 || rk.n_acc > n_pre) return fail(ctx, CHILI_ERR_CUDA, "inconsistent kept count");
        kept += rk.n_acc;
        sum += h[0];
        vmax = std::max(vmax, h[1]);
        over += h[2];
        done += m;
    }
    // copy back only the events written
    const long long written = std::min<long long>(kept, max_events);
    if (am.host) am.bytes = sizeof(double) * written * NE * 4;
    if (aw.host) aw.bytes = sizeof(double) * written;
    if (ac.host) ac.bytes = sizeof(int32_t) * written;
    if ((rc = finish_out(ctx, am)) || (rc = finish_out(ctx, aw)) || (rc = finish_out(ctx, ac))) return rc;
    if ((rc = sync_if_host(ctx, {&am, &aw, &ac}))) return rc;
    if (n_events) *n_events = kept;
    if (info) {
        info->points = static_cast<uint64_t>(n);
        info->rejected_pre = static_cast<uint64_t>(n - n_pre_tot);
        info->kept = static_cast<uint64_t>(kept);
        info->overweight = static_cast<uint64_t>(over);
        info->sum = sum;
        info->max = n_pre_tot < n ? std::max(vmax, 0.0) : vmax;  // rejected points have value 0
    }
    return CHILI_OK;
}

int chili_gpu_evaluate_batch(chili_ctx *ctx, int ch, const double *u, double *out, int64_t n) {
    if (!ctx) return fail(nullptr, CHILI_ERR_INVALID_ARG, "ctx is NULL");
    int rc;
    if ((rc = need_channels(ctx))) return rc;
    if (!ctx->f_set) return fail(ctx, CHILI_ERR_STATE, "no integrand set");
    if (ch < 0 || ch >= ctx->nch || !u || !out || n < 0) return fail(ctx, CHILI_ERR_INVALID_ARG, "bad argument");
    if (n == 0) return CHILI_OK;
    Arg au, ao;
    if ((rc = resolve(ctx, u, sizeof(double) * n * ctx->ndims, 0, true, au))) return rc;
    if ((rc = resolve(ctx, out, sizeof(double) * n, 1, false, ao))) return rc;
    k_evaluate_batch<<<grid_for(n, 128), 128, 0, ctx->stream>>>(ctx->progs.as<ChannelProgram>() + ch,
                                                                static_cast<const double *>(au.dev),
                                                                static_cast<double *>(ao.dev), n,
                                                                ctx->f_dev.as<IntegrandDesc>());
    LAUNCHED();
    if ((rc = finish_out(ctx, ao))) return rc;
    return sync_if_host(ctx, {&au, &ao});
}

}  // extern "C"

// ------------------------------------------------------------ no allocation
// chili_gpu_vegas_iterate_noalloc: the plain-VEGAS accumulation kernel with its
// scratch (the integrand descriptor and one StatsData partial per block) in a
// file-scope device array instead of memory from cudaMalloc.  Every GPU that
// loads the library holds the array until the process exits.
constexpr int kNoAllocMaxBlocks = 1184;  // partials for at most 1184 blocks
constexpr size_t kNoAllocDescDoubles = (sizeof(IntegrandDesc) + sizeof(double) - 1) / sizeof(double);
constexpr size_t kNoAllocScratchDoubles = kNoAllocDescDoubles + 6 * kNoAllocMaxBlocks;
static __device__ __align__(256) double chili_noalloc_scratch[kNoAllocScratchDoubles];

namespace {
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
double *g_noalloc_ptr[kNoAllocMaxDevices] = {nullptr};

// Device address of the scratch array on the current device, looked up once
// per device (with that device current) and cached.
cudaError_t noalloc_scratch(int dev, double **out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        double *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&p), chili_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return cudaSuccess;
}

// Writes the integrand descriptor into the scratch array.  The descriptor
// travels as a kernel argument (copied at launch), so no host memory is
// read after the call returns.
__global__ void k_noalloc_store_desc(IntegrandDesc *dst, const IntegrandDesc src) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *dst = src;
}

bool on_device(const void *p, int dev) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == dev;
}
}  // namespace

extern "C" int chili_gpu_vegas_iterate_noalloc(void *stream, const double *edges, int dims, int bins,
                                               const double *camel_params, int nparams, uint64_t ncalls,
                                               uint64_t seed, uint64_t counter_base, double *stats_out,
                                               double *train_out) {
    chili_ctx *ctx = nullptr;  // for the error macros: errors go to the library's last error
    if (!edges || !camel_params || !stats_out || !train_out)
        return fail(ctx, CHILI_ERR_INVALID_ARG, "NULL argument");
    if (dims < 1 || dims > CHILI_MAX_DIMS || bins < 2 || bins > CHILI_MAX_BINS)
        return fail(ctx, CHILI_ERR_LIMIT, "dims must lie in [1, CHILI_MAX_DIMS] and bins in [2, CHILI_MAX_BINS]");
    if (nparams < 2 + 2 * dims || nparams > CHILI_MAX_INTEGRAND_PARAMS)
        return fail(ctx, CHILI_ERR_LIMIT, "camel needs 2 + 2*dims parameters, at most CHILI_MAX_INTEGRAND_PARAMS");
    if (ncalls < 2 || ncalls > (1ull << 40)) return fail(ctx, CHILI_ERR_LIMIT, "ncalls must lie in [2, 2^40]");
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(ctx, CHILI_ERR_LIMIT, "device index beyond 63");
    if (!on_device(edges, dev) || !on_device(stats_out, dev) || !on_device(train_out, dev))
        return fail(ctx, CHILI_ERR_INVALID_ARG, "edges, stats_out and train_out must be device memory of the current device");
    double *scratch = nullptr;
    CK(noalloc_scratch(dev, &scratch));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    IntegrandDesc desc{};
    desc.kind = CHILI_FUNC_CAMEL;
    desc.nparams = nparams;
    desc.pre = CHILI_PRE_ACCEPT_ALL;
    for (int i = 0; i < nparams; ++i) desc.p[i] = camel_params[i];
    IntegrandDesc *desc_dev = reinterpret_cast<IntegrandDesc *>(scratch);
    double *part = scratch + kNoAllocDescDoubles;
    k_noalloc_store_desc<<<1, 1, 0, st>>>(desc_dev, desc);
    CK(cudaGetLastError());
    const int nh = dims * bins;
    CK(cudaMemsetAsync(train_out, 0, sizeof(double) * nh, st));  // the histogram starts at zero
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long n = static_cast<long long>(ncalls);
    const long long nblocks = std::min<long long>(std::min<long long>(grid_for(n, kVegasBlock), sms * 4ll),
                                                  kNoAllocMaxBlocks);
    k_vegas_iter<0><<<static_cast<unsigned>(nblocks), kVegasBlock, 0, st>>>(edges, dims, bins, seed, counter_base,
                                                                          nullptr, n, desc_dev, part, train_out, 0);
    CK(cudaGetLastError());
    k_vegas_finalize<<<1, 256, 0, st>>>(part, static_cast<int>(nblocks), nullptr, 0, nh, train_out, stats_out);
    CK(cudaGetLastError());
    return CHILI_OK;
}

