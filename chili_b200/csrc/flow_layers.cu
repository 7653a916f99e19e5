// flow_layers.cu -- launchers of the coupling-layer kernels (flow.cuh).
#include <cuda_runtime.h>

#include <algorithm>

#define CHILI_FLOW_LAYERS_ONLY
#include "flow_launch.h"

using namespace chili_flow;

namespace {

template <class K>
int smem_attr(chili_ctx *ctx, K kernel, size_t bytes) {
    CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
    return CHILI_OK;
}

template <int DB, int MODE, bool SAVE>
int launch_layer_t(chili_ctx *ctx, const LayerArgs &a, int sms) {
    static bool attr = false;
    if (!attr) {
        if (int rc = smem_attr(ctx, k_flow_layer<DB, MODE, SAVE>, kFwdSmem)) return rc;
        attr = true;
    }
    const long long tiles = (a.n + 127) / 128;
    const unsigned grid = static_cast<unsigned>(std::min<long long>(tiles, sms));
    KTimer kt_(ctx, KT_FLOW_LAYER);
    k_flow_layer<DB, MODE, SAVE><<<grid, kFwdThreads, kFwdSmem, ctx->stream>>>(a);
    LAUNCHED();
    return CHILI_OK;
}

template <int MODE, bool SAVE>
int launch_layer(chili_ctx *ctx, const LayerArgs &a, int sms) {
    switch (a.L.db) {
    case 1: return launch_layer_t<1, MODE, SAVE>(ctx, a, sms);
    case 2: return launch_layer_t<2, MODE, SAVE>(ctx, a, sms);
    case 3: return launch_layer_t<3, MODE, SAVE>(ctx, a, sms);
    case 4: return launch_layer_t<4, MODE, SAVE>(ctx, a, sms);
    case 5: return launch_layer_t<5, MODE, SAVE>(ctx, a, sms);
    default: return fail(ctx, CHILI_ERR_LIMIT, "coupling layer transforms more than 5 dimensions");
    }
}

template <int DB>
int launch_bwd_t(chili_ctx *ctx, const BwdArgs &a, int sms) {
    static bool attr = false;
    if (!attr) {
        if (int rc = smem_attr(ctx, k_flow_layer_bwd<DB>, kBwdSmem)) return rc;
        attr = true;
    }
    const long long tiles = (a.n + 127) / 128;
    const unsigned grid = static_cast<unsigned>(std::min<long long>(tiles, sms));
    KTimer kt_(ctx, KT_FLOW_BWD);
    k_flow_layer_bwd<DB><<<grid, kBwdThreads, kBwdSmem, ctx->stream>>>(a);
    LAUNCHED();
    return CHILI_OK;
}

int launch_bwd_db(chili_ctx *ctx, const BwdArgs &a, int sms) {
    switch (a.L.db) {
    case 1: return launch_bwd_t<1>(ctx, a, sms);
    case 2: return launch_bwd_t<2>(ctx, a, sms);
    case 3: return launch_bwd_t<3>(ctx, a, sms);
    case 4: return launch_bwd_t<4>(ctx, a, sms);
    case 5: return launch_bwd_t<5>(ctx, a, sms);
    default: return fail(ctx, CHILI_ERR_LIMIT, "coupling layer transforms more than 5 dimensions");
    }
}

}  // namespace

int flow_launch_layer(chili_ctx *ctx, int mode, bool save, const LayerArgs &a, int sms) {
    if (mode == 0) return save ? launch_layer<0, true>(ctx, a, sms) : launch_layer<0, false>(ctx, a, sms);
    return launch_layer<1, false>(ctx, a, sms);
}

int flow_launch_bwd(chili_ctx *ctx, const BwdArgs &a, int sms) { return launch_bwd_db(ctx, a, sms); }
