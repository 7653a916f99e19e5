// flow_launch.h -- launchers of the learned proposal's heavy kernels, each
// in its own translation unit so that they compile in parallel
// (flow_layers.cu: coupling layers; flow_alpha.cu: channel-weight network and
// the last step of the flow-path points).
#pragma once

#include "context.h"
#include "flow_phys.cuh"
#include "flow_wide.cuh"

// Coupling-layer forward (mode 0: density direction, 1: sampling), one block
// per SM at most.
int flow_launch_layer(chili_ctx *ctx, int mode, bool save, const chili_flow::LayerArgs &a, int sms);
int flow_launch_bwd(chili_ctx *ctx, const chili_flow::BwdArgs &a, int sms);
// The channel-weight network on the tensor cores (flow_alpha_tc.cuh):
// training (forward, loss, backward, weight-gradient partials of kAlphaSplit
// CTAs), sampling (the values of the rows), and the packing of its bf16 tiles.
int flow_launch_alpha(chili_ctx *ctx, const chili_flow::AlphaTcArgs &a);
int flow_launch_alpha_eval(chili_ctx *ctx, const chili_flow::AlphaTcArgs &a, int sms);
int flow_launch_alpha_pack(chili_ctx *ctx, const float *w, const chili_flow::AlphaLayout &L, uint8_t *tiles);
// The last step of a flow-path tile: the rows of the channel-weight network.
int flow_launch_combine(chili_ctx *ctx, const chili_flow::CombineArgs &a, unsigned blocks);

// The wide-conditioner kernels (flow_wide.cuh; flow_wide.cu).
int flow_launch_layer_wide(chili_ctx *ctx, int mode, bool save, const chili_flow::WideFwdArgs &a, int sms);
int flow_launch_bwd_wide(chili_ctx *ctx, const chili_flow::WideBwdArgs &a, int sms);
int flow_launch_wgrad_wide(chili_ctx *ctx, const chili_flow::WideWgradArgs &a, int nsplit);
int flow_launch_pack_wide(chili_ctx *ctx, const chili_flow::WidePackArgs &a);
