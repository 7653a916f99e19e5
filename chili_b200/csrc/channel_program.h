// channel_program.h -- the flattened, table-driven form of one FSMapper
// channel (include/Channel/Channel.hh:15-77) that the kernels execute.
//
// FSMapper keeps momenta and masses in hash maps keyed by the current bitmask
// and recurses through std::map lookups (Channel.cc:63-256).  The host builder
// (channel_program.cpp) resolves all of that once: every current used by the
// channel gets a slot (slots 0..n_ext-1 are the external legs, idx 1<<i), the
// decays are listed in std::map order, and the recursive s-channel decay tree
// is unrolled into the order in which DecayParts consumes uniforms.  Every
// per-decay constant that depends only on the cuts (smin2, cuts.smin, SMax) is
// computed on the host with the reference's expression.
#pragma once

#include <cstdint>

#include "chili_gpu.h"

#define CHILI_MAX_SLOTS (2 * CHILI_MAX_EXT)
#define CHILI_MAX_DECAYS CHILI_MAX_EXT

struct ChannelProgram {
    int32_t n_ext;    // external legs, incoming included
    int32_t ndims;    // 3*(n_ext-2) - 2
    int32_t n_slots;  // externals + compound currents
    int32_t n_info;   // t-channel entries
    int32_t n_decay;  // DecayMap entries, std::map order
    int32_t n_sdec;   // DecayParts calls in uniform-consumption order
    double sqrts, ptmax, inv16pi3;

    double slot_m2[CHILI_MAX_SLOTS];  // squared masses of the outgoing legs

    int8_t info_slot[CHILI_MAX_EXT];
    double info_ptmin[CHILI_MAX_EXT];   // FSMapper::m_ptmin (Channel.hh:20-26)
    double info_etamax[CHILI_MAX_EXT];  // cuts.etamax.at(idx)

    int8_t dec_parent[CHILI_MAX_DECAYS], dec_c1[CHILI_MAX_DECAYS], dec_c2[CHILI_MAX_DECAYS];
    int8_t dec_massless[CHILI_MAX_DECAYS];
    double dec_mass[CHILI_MAX_DECAYS], dec_width[CHILI_MAX_DECAYS];
    double dec_smin2[CHILI_MAX_DECAYS];     // ptmin1*ptmin2*2/pi/pi*dR^2 (Channel.cc:150)
    double dec_cut_smin[CHILI_MAX_DECAYS];  // cuts.smin[idx1|idx2] (Channel.cc:151)
    double dec_smax[CHILI_MAX_DECAYS];      // SMax(sqrts, cuts, idx) (Cuts.hh:21-29)

    int8_t sdec_ab[CHILI_MAX_DECAYS], sdec_a[CHILI_MAX_DECAYS], sdec_b[CHILI_MAX_DECAYS];
};

// The whole channel set seen from one point: quantities that several
// channels share are listed once.
//   nodes   momenta of the external legs and of every distinct compound
//           current, node = node_a + node_b (the reference's tmp_mom sum)
//   tents   t-channel entries other than the last, keyed by (node, ptmin,
//           etamax cut): pT jacobian factor, eta factor and 3 uniforms
//   chains  whole t-channel chains (ordered tents + last node): weight and
//           last uniform, or failure (Channel.cc:197)
//   dws     decay propagator weights and their uniform (Channel.cc:83-113)
//   sws     two-body decay weights and their 2 uniforms (Channel.cc:222-256)
// A channel is then the product of its parts in the reference's order.
#define PP_MAX_NODES 32
#define PP_MAX_TENTS 48
#define PP_MAX_CHAINS 64
#define PP_MAX_DWS 96
#define PP_MAX_SWS 64

struct PPChannel {
    int8_t n_dec, n_sd;
    int16_t chain;
    int16_t dw[CHILI_MAX_DECAYS];
    int16_t sw[CHILI_MAX_DECAYS];
};

struct PointProgram {
    int32_t n_ext, ndims, nch, n_nodes, n_tents, n_chains, n_dws, n_sws;
    double sqrts, ptmax, inv16pi3;
    int8_t node_a[PP_MAX_NODES], node_b[PP_MAX_NODES];
    int8_t tent_node[PP_MAX_TENTS];
    double tent_ptmin[PP_MAX_TENTS], tent_etacut[PP_MAX_TENTS];
    int8_t chain_len[PP_MAX_CHAINS], chain_last[PP_MAX_CHAINS];
    int8_t chain_tent[PP_MAX_CHAINS][CHILI_MAX_EXT];
    int8_t dw_node[PP_MAX_DWS], dw_c1[PP_MAX_DWS], dw_c2[PP_MAX_DWS], dw_massless[PP_MAX_DWS];
    double dw_mass[PP_MAX_DWS], dw_width[PP_MAX_DWS], dw_smin2[PP_MAX_DWS], dw_cut[PP_MAX_DWS], dw_smax[PP_MAX_DWS];
    // Terms of the propagator weights that depend only on (smin, smax), for
    // smin = dw_smin_c (the value smin takes whenever the decay products'
    // masses are below the cut; filled on the device by k_pp_prepare):
    // massless: pow(smin, 0.01), pow(smax, 0.01); massive: atan((smin-m2)/mw),
    // atan((smax-m2)/mw).
    double dw_smin_c[PP_MAX_DWS], dw_t1[PP_MAX_DWS], dw_t2[PP_MAX_DWS];
    int8_t sw_a[PP_MAX_SWS], sw_b[PP_MAX_SWS];
    PPChannel ch[CHILI_MAX_CHANNELS];
    // Phased evaluation: every item's outputs live in a memo buffer of
    // n_memo slots per point (tent t: fac, g, x0, x1, x2 at memo_tent+5t;
    // dw d: w, x at memo_dw+2d; sw s: w, r1, r2 at memo_sw+3s; chain c: w,
    // x at memo_chain+2c).  pos_src[c][p] is the memo slot of channel c's
    // uniform p; pos_src_fail[c][p] the same when c's chain fails, where the
    // s-channel uniforms move down by one and the last position keeps the
    // value the previous channels left there (-1).
    int32_t memo_tent, memo_dw, memo_sw, memo_chain, n_memo;
    int16_t pos_src[CHILI_MAX_CHANNELS][CHILI_MAX_DIMS];
    int16_t pos_src_fail[CHILI_MAX_CHANNELS][CHILI_MAX_DIMS];
};

#ifdef __cplusplus
#include <string>
#include <vector>
// Builds the programs; returns an empty string on success, else the reason.
std::string build_channel_programs(const chili_channel_desc *descs, int nch, const chili_cuts *cuts,
                                   double sqrts, int n_ext, std::vector<ChannelProgram> &out);
// Deduplicates the per-channel programs into one PointProgram; false when the
// set exceeds the PP_MAX_* limits (the per-channel kernels are used then).
bool build_point_program(const std::vector<ChannelProgram> &progs, PointProgram &pp);
#endif
