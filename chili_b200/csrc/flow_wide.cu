// flow_wide.cu -- launchers of the wide-conditioner coupling kernels
// (flow_wide.cuh): H = 128 or 256 hidden units, 2..4 hidden layers, weights
// streamed from global memory per tile.
#include <cuda_runtime.h>

#include <algorithm>

#define CHILI_FLOW_LAYERS_ONLY
#define CHILI_FLOW_WIDE_KERNELS
#include "flow_launch.h"

using namespace chili_flow;

namespace {

template <class K>
int smem_attr(chili_ctx *ctx, K kernel, size_t bytes) {
    CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
    return CHILI_OK;
}

template <int H, int MODE, bool SAVE>
int launch_fwd_t(chili_ctx *ctx, const WideFwdArgs &a, int sms) {
    static bool attr = false;
    constexpr int smem = wide_fwd_smem<H>();
    if (!attr) {
        if (int rc = smem_attr(ctx, k_flow_layer_wide<H, MODE, SAVE>, smem)) return rc;
        attr = true;
    }
    const long long tiles = (a.n + 127) / 128;
    const unsigned grid = static_cast<unsigned>(std::min<long long>(tiles, sms));
    KTimer kt_(ctx, KT_FLOW_LAYER);
    k_flow_layer_wide<H, MODE, SAVE><<<grid, kWFwdThreads, smem, ctx->stream>>>(a);
    LAUNCHED();
    return CHILI_OK;
}

template <int H>
int launch_fwd_h(chili_ctx *ctx, int mode, bool save, const WideFwdArgs &a, int sms) {
    if (mode == 0) return save ? launch_fwd_t<H, 0, true>(ctx, a, sms) : launch_fwd_t<H, 0, false>(ctx, a, sms);
    return launch_fwd_t<H, 1, false>(ctx, a, sms);
}

template <int H>
int launch_bwd_h(chili_ctx *ctx, const WideBwdArgs &a, int sms) {
    static bool attr = false;
    if (!attr) {
        if (int rc = smem_attr(ctx, k_flow_layer_bwd_wide<H>, kWBwdSmem)) return rc;
        attr = true;
    }
    const long long tiles = (a.n + 127) / 128;
    const unsigned grid = static_cast<unsigned>(std::min<long long>(tiles, sms));
    KTimer kt_(ctx, KT_FLOW_BWD);
    k_flow_layer_bwd_wide<H><<<grid, kWBwdThreads, kWBwdSmem, ctx->stream>>>(a);
    LAUNCHED();
    return CHILI_OK;
}

int check_layer(chili_ctx *ctx, const WideLayer &L) {
    if ((L.H != 128 && L.H != 256) || L.nh < 2 || L.nh > kWMaxNH || L.db < 1 || L.db > kMaxDB || L.da < 1 ||
        L.da > kMaxDA)
        return fail(ctx, CHILI_ERR_LIMIT, "wide coupling layer outside H in {128, 256}, 2..4 hidden layers");
    return CHILI_OK;
}

}  // namespace

int flow_launch_layer_wide(chili_ctx *ctx, int mode, bool save, const WideFwdArgs &a, int sms) {
    if (int rc = check_layer(ctx, a.L)) return rc;
    return a.L.H == 256 ? launch_fwd_h<256>(ctx, mode, save, a, sms) : launch_fwd_h<128>(ctx, mode, save, a, sms);
}

int flow_launch_bwd_wide(chili_ctx *ctx, const WideBwdArgs &a, int sms) {
    if (int rc = check_layer(ctx, a.L)) return rc;
    return a.L.H == 256 ? launch_bwd_h<256>(ctx, a, sms) : launch_bwd_h<128>(ctx, a, sms);
}

int flow_launch_wgrad_wide(chili_ctx *ctx, const WideWgradArgs &a, int nsplit) {
    static bool attr = false;
    if (!attr) {
        if (int rc = smem_attr(ctx, k_flow_wgrad_wide, kWgWideSmem)) return rc;
        attr = true;
    }
    if (a.nitems < 1 || a.nitems > 16) return fail(ctx, CHILI_ERR_LIMIT, "wide weight gradient: 1..16 products");
    KTimer kt_(ctx, KT_FLOW_WGRAD);
    k_flow_wgrad_wide<<<dim3(nsplit, a.nitems), 128, kWgWideSmem, ctx->stream>>>(a);
    LAUNCHED();
    return CHILI_OK;
}

int flow_launch_pack_wide(chili_ctx *ctx, const WidePackArgs &a) {
    const long long most = std::max<long long>(static_cast<long long>(a.H) * a.H, static_cast<long long>(kPF) * a.H);
    k_flow_pack_wide<<<dim3(static_cast<unsigned>((most + 255) / 256), a.nh + 1), 256, 0, ctx->stream>>>(a);
    LAUNCHED();
    return CHILI_OK;
}
