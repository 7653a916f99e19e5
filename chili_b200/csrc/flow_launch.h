// flow_launch.h -- launchers of the learned proposal's heavy kernels, each
// in its own translation unit so that they compile in parallel
// (flow_layers.cu: coupling layers; flow_alpha.cu: channel-weight network and
// the flow-path physics).
#pragma once

#include "context.h"
#include "flow_phys.cuh"

// Coupling-layer forward (mode 0: density direction, 1: sampling), one block
// per SM at most.
int flow_launch_layer(chili_ctx *ctx, int mode, bool save, const chili_flow::LayerArgs &a, int sms);
int flow_launch_bwd(chili_ctx *ctx, const chili_flow::BwdArgs &a, int sms);
int flow_launch_alpha(chili_ctx *ctx, const chili_flow::AlphaTrainArgs &a);
int flow_launch_phys(chili_ctx *ctx, const chili_flow::PhysArgs &a, unsigned blocks);
