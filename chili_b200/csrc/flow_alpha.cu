// flow_alpha.cu -- launchers of the channel-weight network's training kernel
// and of the flow-path physics kernel (flow_phys.cuh).
#include <cuda_runtime.h>
#include <math_constants.h>

#define CHILI_FLOW_LAYERS_ONLY
#include "flow_launch.h"

using namespace chili_flow;

namespace {

template <class K>
int smem_attr(chili_ctx *ctx, K kernel, size_t bytes) {
    CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
    return CHILI_OK;
}

constexpr int kAlphaSplit = 148;

template <int NCH, int NF>
int launch_alpha_t(chili_ctx *ctx, const AlphaTrainArgs &a) {
    const size_t bytes = alpha_train_smem<NCH, NF>(a.L.total);
    static size_t attr = 0;
    if (attr < bytes) {
        if (int rc = smem_attr(ctx, k_alpha_train<NCH, NF>, bytes)) return rc;
        attr = bytes;
    }
    KTimer kt_(ctx, KT_ALPHA_TRAIN);
    k_alpha_train<NCH, NF><<<kAlphaSplit, kAlphaBlock, bytes, ctx->stream>>>(a);
    LAUNCHED();
    return CHILI_OK;
}

int launch_alpha(chili_ctx *ctx, const AlphaTrainArgs &a) {
    const int nch = a.L.nch, F = a.L.F;
    if (nch <= 16 && F <= 16) return launch_alpha_t<16, 16>(ctx, a);
    if (nch <= 64 && F <= 32) return launch_alpha_t<64, 32>(ctx, a);
    return fail(ctx, CHILI_ERR_LIMIT, "channel-weight network limited to 64 channels and 32 features");
}

template <bool TRAIN, int NCH, int NF>
int launch_combine_t(chili_ctx *ctx, const CombineArgs &a, unsigned blocks) {
    const size_t bytes = TRAIN ? 0 : sizeof(float) * AlphaSmem<NCH, NF>::kTotal;
    if constexpr (!TRAIN) {
        static size_t attr = 0;
        if (attr < bytes) {
            if (int rc = smem_attr(ctx, k_flow_combine<TRAIN, NCH, NF>, bytes)) return rc;
            attr = bytes;
        }
    }
    KTimer kt_(ctx, KT_FLOW_PHYS);
    k_flow_combine<TRAIN, NCH, NF><<<blocks, 128, bytes, ctx->stream>>>(a);
    LAUNCHED();
    return CHILI_OK;
}

template <bool TRAIN>
int launch_combine(chili_ctx *ctx, const CombineArgs &a, unsigned blocks) {
    const int nch = a.L.nch, F = a.L.F;
    if (nch <= 16 && F <= 16) return launch_combine_t<TRAIN, 16, 16>(ctx, a, blocks);
    if (nch <= 64 && F <= 32) return launch_combine_t<TRAIN, 64, 32>(ctx, a, blocks);
    return fail(ctx, CHILI_ERR_LIMIT, "channel-weight network limited to 64 channels and 32 features");
}

}  // namespace

int flow_launch_alpha(chili_ctx *ctx, const AlphaTrainArgs &a) { return launch_alpha(ctx, a); }
int flow_launch_combine(chili_ctx *ctx, bool train, const CombineArgs &a, unsigned blocks) {
    return train ? launch_combine<true>(ctx, a, blocks) : launch_combine<false>(ctx, a, blocks);
}
