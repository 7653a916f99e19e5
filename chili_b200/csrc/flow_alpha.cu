// flow_alpha.cu -- launchers of the channel-weight network's tensor-core
// kernels (flow_alpha_tc.cuh: training and sampling) and of the flow-path
// physics kernel that prepares the network's rows (flow_phys.cuh).
#include <cuda_runtime.h>
#include <math_constants.h>

#define CHILI_FLOW_LAYERS_ONLY
#include "flow_alpha_tc.cuh"
#include "flow_launch.h"

using namespace chili_flow;

namespace {

template <class K>
int smem_attr(chili_ctx *ctx, K kernel, size_t bytes) {
    CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
    return CHILI_OK;
}

constexpr int kAlphaSplit = 148;

template <bool TRAIN, int NCHP>
int launch_alpha_t(chili_ctx *ctx, const AlphaTcArgs &a, unsigned blocks) {
    constexpr size_t bytes = TRAIN ? kASmemTrain : kASmemEval;
    auto kernel = TRAIN ? k_alpha_train_tc<NCHP> : k_alpha_eval_tc<NCHP>;
    static bool attr = false;
    if (!attr) {
        if (int rc = smem_attr(ctx, kernel, bytes)) return rc;
        attr = true;
    }
    KTimer kt_(ctx, TRAIN ? KT_ALPHA_TRAIN : KT_ALPHA_EVAL);
    kernel<<<blocks, kAThreads, bytes, ctx->stream>>>(a);
    LAUNCHED();
    return CHILI_OK;
}

template <bool TRAIN>
int launch_alpha(chili_ctx *ctx, const AlphaTcArgs &a, unsigned blocks) {
    // a0 holds the F features and the constant column within its first 32
    if (a.L.F + 1 > 32) return fail(ctx, CHILI_ERR_LIMIT, "channel-weight network limited to 31 features");
    if (a.L.nch <= 16) return launch_alpha_t<TRAIN, 16>(ctx, a, blocks);
    if (a.L.nch <= 64) return launch_alpha_t<TRAIN, 64>(ctx, a, blocks);
    return fail(ctx, CHILI_ERR_LIMIT, "channel-weight network limited to 64 channels");
}

template <int NCH>
int launch_combine_t(chili_ctx *ctx, const CombineArgs &a, unsigned blocks) {
    KTimer kt_(ctx, KT_FLOW_PHYS);
    k_flow_combine<NCH><<<blocks, 128, 0, ctx->stream>>>(a);
    LAUNCHED();
    return CHILI_OK;
}

}  // namespace

int flow_launch_alpha(chili_ctx *ctx, const AlphaTcArgs &a) { return launch_alpha<true>(ctx, a, kAlphaSplit); }

int flow_launch_alpha_eval(chili_ctx *ctx, const AlphaTcArgs &a, int sms) {
    const long long tiles = (a.n + 127) / 128;
    const unsigned blocks = static_cast<unsigned>(std::max<long long>(1, std::min<long long>(tiles, 4ll * sms)));
    return launch_alpha<false>(ctx, a, blocks);
}

int flow_launch_alpha_pack(chili_ctx *ctx, const float *w, const AlphaLayout &L, uint8_t *tiles) {
    k_alpha_pack<<<(3 * 64 * 64 + 255) / 256, 256, 0, ctx->stream>>>(w, L, tiles);
    LAUNCHED();
    return CHILI_OK;
}

int flow_launch_combine(chili_ctx *ctx, const CombineArgs &a, unsigned blocks) {
    if (a.nch <= 16) return launch_combine_t<16>(ctx, a, blocks);
    if (a.nch <= 64) return launch_combine_t<64>(ctx, a, blocks);
    return fail(ctx, CHILI_ERR_LIMIT, "channel-weight network limited to 64 channels");
}
