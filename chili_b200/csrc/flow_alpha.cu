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

template <int NCH, int NF>
int launch_phys_t(chili_ctx *ctx, const PhysArgs &a, unsigned blocks) {
    const size_t bytes = sizeof(double) * 2 * kMaxAlphaCh + sizeof(float) * a.L.total;
    static size_t attr = 0;
    if (attr < bytes) {
        if (int rc = smem_attr(ctx, k_flow_phys<NCH, NF>, bytes)) return rc;
        attr = bytes;
    }
    k_flow_phys<NCH, NF><<<blocks, kPhysBlock, bytes, ctx->stream>>>(a);
    LAUNCHED();
    return CHILI_OK;
}

int launch_phys(chili_ctx *ctx, const PhysArgs &a, unsigned blocks) {
    const int nch = a.L.nch, F = a.L.F;
    if (nch <= 16 && F <= 16) return launch_phys_t<16, 16>(ctx, a, blocks);
    if (nch <= 64 && F <= 32) return launch_phys_t<64, 32>(ctx, a, blocks);
    return fail(ctx, CHILI_ERR_LIMIT, "channel-weight network limited to 64 channels and 32 features");
}

}  // namespace

int flow_launch_alpha(chili_ctx *ctx, const AlphaTrainArgs &a) { return launch_alpha(ctx, a); }
int flow_launch_phys(chili_ctx *ctx, const PhysArgs &a, unsigned blocks) { return launch_phys(ctx, a, blocks); }
