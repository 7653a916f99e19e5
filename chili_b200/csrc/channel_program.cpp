// channel_program.cpp -- host builder of ChannelProgram tables from
// ChannelDescription + Cuts (see channel_program.h).
#include "channel_program.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <set>
#include <sstream>
#include <tuple>

namespace {

using Key = std::tuple<uint32_t, double, double>;  // ParticleInfo order (ChannelNode.cc:293-301)
Key key_of(const chili_particle_info &p) { return Key{p.idx, p.mass, p.width}; }

bool is_power2(uint32_t v) { return (v & (v - 1)) == 0; }

struct Lookup {
    std::map<uint32_t, double> smin, ptmin, etamax;
    std::map<std::pair<int, int>, double> delta_r;
    std::vector<double> sexternal;
};

}  // namespace

std::string build_channel_programs(const chili_channel_desc *descs, int nch, const chili_cuts *cuts,
                                   double sqrts, int n_ext, std::vector<ChannelProgram> &out) {
    std::ostringstream err;
    if (!descs || !cuts || nch <= 0) return "null channel descriptions or cuts";
    if (nch > CHILI_MAX_CHANNELS) return "too many channels";
    if (n_ext < 3 || n_ext > CHILI_MAX_EXT) return "n_ext outside [3, CHILI_MAX_EXT]";
    const int nout = n_ext - 2;
    if (cuts->n_sexternal != nout) return "cuts.sexternal must hold n_ext-2 entries";
    Lookup L;
    for (int i = 0; i < cuts->n_sexternal; ++i) L.sexternal.push_back(cuts->sexternal[i]);
    for (int i = 0; i < cuts->n_smin; ++i) L.smin[cuts->smin[i].idx] = cuts->smin[i].value;
    for (int i = 0; i < cuts->n_ptmin; ++i) L.ptmin[cuts->ptmin[i].idx] = cuts->ptmin[i].value;
    for (int i = 0; i < cuts->n_etamax; ++i) L.etamax[cuts->etamax[i].idx] = cuts->etamax[i].value;
    for (int i = 0; i < cuts->n_deltaR; ++i)
        L.delta_r[{cuts->deltaR[i].pid1, cuts->deltaR[i].pid2}] = cuts->deltaR[i].value;

    const uint32_t all_out = ((1u << n_ext) - 1u) & ~3u;
    const int ndims = 3 * nout - 2;  // FSMapper::NDims (Channel.hh:33)
    out.assign(nch, ChannelProgram{});
    for (int c = 0; c < nch; ++c) {
        const chili_channel_desc &d = descs[c];
        ChannelProgram &P = out[c];
        std::memset(&P, 0, sizeof(P));
        P.n_ext = n_ext;
        P.ndims = ndims;
        P.sqrts = sqrts;
        P.ptmax = sqrts / 2.0;
        P.inv16pi3 = 1.0 / (16 * std::pow(M_PI, 3));  // Channel.cc:243
        if (d.n_info < 1 || d.n_info > nout || !d.info) {
            err << "channel " << c << ": n_info outside [1, n_ext-2]";
            return err.str();
        }
        if (d.n_decays < 0 || d.n_decays > CHILI_MAX_DECAYS || (d.n_decays > 0 && !d.decays)) {
            err << "channel " << c << ": bad decay count";
            return err.str();
        }
        // slots: externals first
        std::map<uint32_t, int> slot;
        for (int i = 0; i < n_ext; ++i) slot[1u << i] = i;
        for (int i = 0; i < nout; ++i) P.slot_m2[i + 2] = L.sexternal[i];  // Channel.cc:25-26
        int n_slots = n_ext;

        // DecayMap in std::map order, keyed by (idx, mass, width)
        std::map<Key, const chili_decay *> decays;
        for (int k = 0; k < d.n_decays; ++k) {
            const chili_decay &dec = d.decays[k];
            if (!decays.emplace(key_of(dec.parent), &dec).second) {
                err << "channel " << c << ": duplicate decay parent " << dec.parent.idx;
                return err.str();
            }
            const uint32_t p = dec.parent.idx, a = dec.child1.idx, b = dec.child2.idx;
            if ((a & b) || (a | b) != p || (p & ~all_out) || is_power2(p) || a == 0 || b == 0) {
                err << "channel " << c << ": decay " << p << " -> (" << a << ", " << b
                    << ") is not a split of outgoing legs";
                return err.str();
            }
        }
        for (const auto &kv : decays) {
            const uint32_t p = std::get<0>(kv.first);
            if (!slot.count(p)) {
                if (n_slots >= CHILI_MAX_SLOTS) return "too many currents";
                slot[p] = n_slots++;
            }
        }
        P.n_slots = n_slots;
        int k = 0;
        for (const auto &kv : decays) {
            const chili_decay &dec = *kv.second;
            const auto pt1 = L.ptmin.find(dec.child1.idx), pt2 = L.ptmin.find(dec.child2.idx);
            if (pt1 == L.ptmin.end() || pt2 == L.ptmin.end()) {
                err << "channel " << c << ": cuts.ptmin lacks a decay product";
                return err.str();
            }
            for (uint32_t child : {dec.child1.idx, dec.child2.idx}) {
                if (!slot.count(child)) {
                    err << "channel " << c << ": decay product " << child << " has no decay of its own";
                    return err.str();
                }
            }
            const auto dr = L.delta_r.find({dec.child1.pid, dec.child2.pid});
            const double delta_r = dr == L.delta_r.end() ? 0 : dr->second;
            // Channel.cc:150-152, the same expressions evaluated on the host
            const double smin2 = pt1->second * pt2->second * 2 / M_PI / M_PI * std::pow(delta_r, 2);
            const auto sm = L.smin.find(dec.child1.idx | dec.child2.idx);
            double smax = sqrts;  // SMax (Cuts.hh:21-29)
            for (unsigned i = 0; i < L.sexternal.size(); ++i)
                if (!(dec.parent.idx & (1u << (i + 2)))) smax -= std::sqrt(L.sexternal[i]);
            smax = smax * smax;
            P.dec_parent[k] = static_cast<int8_t>(slot[dec.parent.idx]);
            P.dec_c1[k] = static_cast<int8_t>(slot[dec.child1.idx]);
            P.dec_c2[k] = static_cast<int8_t>(slot[dec.child2.idx]);
            P.dec_massless[k] = (std::abs(dec.parent.mass) < 1e-16 || dec.parent.width < 1e-16) ? 1 : 0;
            P.dec_mass[k] = dec.parent.mass;
            P.dec_width[k] = dec.parent.width;
            P.dec_smin2[k] = smin2;
            P.dec_cut_smin[k] = sm == L.smin.end() ? 0.0 : sm->second;
            P.dec_smax[k] = smax;
            ++k;
        }
        P.n_decay = k;

        // t-channel list (FSMapper ctor, Channel.hh:18-30)
        P.n_info = d.n_info;
        uint32_t covered = 0;
        for (int i = 0; i < d.n_info; ++i) {
            const chili_particle_info &in = d.info[i];
            if (!slot.count(in.idx) || (in.idx & 3u)) {
                err << "channel " << c << ": t-channel entry " << in.idx << " is neither an outgoing leg nor a decaying current";
                return err.str();
            }
            if (!is_power2(in.idx) && !decays.count(key_of(in))) {
                err << "channel " << c << ": t-channel current " << in.idx << " has no matching decay";
                return err.str();
            }
            const auto pt = L.ptmin.find(in.idx);
            const auto eta = L.etamax.find(in.idx);
            if (pt == L.ptmin.end() || eta == L.etamax.end()) {
                err << "channel " << c << ": cuts.ptmin/etamax lack entry " << in.idx;
                return err.str();
            }
            if (covered & in.idx) {
                err << "channel " << c << ": t-channel entries overlap";
                return err.str();
            }
            covered |= in.idx;
            P.info_slot[i] = static_cast<int8_t>(slot[in.idx]);
            P.info_ptmin[i] = pt->second != 0 ? pt->second : 1.0;
            P.info_etamax[i] = eta->second;
        }
        if (covered != all_out) {
            err << "channel " << c << ": t-channel entries do not cover all outgoing legs";
            return err.str();
        }

        // s-channel schedule: GenSChan/DecayParts recursion (Channel.cc:204-245)
        int ns = 0;
        bool bad = false;
        std::vector<const chili_particle_info *> stack;
        auto visit = [&](auto &&self, const chili_particle_info &ab) -> void {
            const auto it = decays.find(key_of(ab));
            if (it == decays.end()) {
                bad = true;
                return;
            }
            const chili_decay &dec = *it->second;
            if (ns >= CHILI_MAX_DECAYS) {
                bad = true;
                return;
            }
            P.sdec_ab[ns] = static_cast<int8_t>(slot[ab.idx]);
            P.sdec_a[ns] = static_cast<int8_t>(slot[dec.child1.idx]);
            P.sdec_b[ns] = static_cast<int8_t>(slot[dec.child2.idx]);
            ++ns;
            if (!is_power2(dec.child1.idx)) self(self, dec.child1);
            if (!is_power2(dec.child2.idx)) self(self, dec.child2);
        };
        for (int i = 0; i < d.n_info; ++i)
            if (!is_power2(d.info[i].idx)) visit(visit, d.info[i]);
        if (bad) {
            err << "channel " << c << ": a decaying current has no matching DecayMap entry";
            return err.str();
        }
        P.n_sdec = ns;
        const int used = P.n_decay + 3 * (P.n_info - 1) + 1 + 2 * P.n_sdec;
        if (used != ndims) {
            err << "channel " << c << ": consumes " << used << " uniforms, NDims is " << ndims;
            return err.str();
        }
    }
    return std::string();
}

bool build_point_program(const std::vector<ChannelProgram> &progs, PointProgram &pp) {
    std::memset(&pp, 0, sizeof(pp));
    if (progs.empty()) return false;
    const ChannelProgram &p0 = progs[0];
    pp.n_ext = p0.n_ext;
    pp.ndims = p0.ndims;
    pp.nch = static_cast<int32_t>(progs.size());
    pp.sqrts = p0.sqrts;
    pp.ptmax = p0.ptmax;
    pp.inv16pi3 = p0.inv16pi3;
    std::map<std::pair<int, int>, int> node_of_pair;
    std::map<std::tuple<int, double, double>, int> tent_of;
    std::map<std::pair<std::vector<int>, int>, int> chain_of;
    std::map<std::tuple<int, int, int, int, double, double, double, double, double>, int> dw_of;
    std::map<std::pair<int, int>, int> sw_of;
    int n_nodes = p0.n_ext;
    for (size_t c = 0; c < progs.size(); ++c) {
        const ChannelProgram &P = progs[c];
        if (P.n_ext != p0.n_ext || P.sqrts != p0.sqrts) return false;
        int node[CHILI_MAX_SLOTS];
        for (int s = 0; s < P.n_slots; ++s) node[s] = s < P.n_ext ? s : -1;
        PPChannel &C = pp.ch[c];
        // compound currents in decay (std::map) order: children come first
        for (int k = 0; k < P.n_decay; ++k) {
            const int a = node[P.dec_c1[k]], b = node[P.dec_c2[k]];
            if (a < 0 || b < 0) return false;
            auto it = node_of_pair.find({a, b});
            int nd;
            if (it == node_of_pair.end()) {
                if (n_nodes >= PP_MAX_NODES) return false;
                nd = n_nodes++;
                pp.node_a[nd] = static_cast<int8_t>(a);
                pp.node_b[nd] = static_cast<int8_t>(b);
                node_of_pair[{a, b}] = nd;
            } else {
                nd = it->second;
            }
            node[P.dec_parent[k]] = nd;
        }
        for (int k = 0; k < P.n_decay; ++k) {
            const auto key = std::make_tuple(node[P.dec_parent[k]], node[P.dec_c1[k]], node[P.dec_c2[k]],
                                             static_cast<int>(P.dec_massless[k]), P.dec_mass[k], P.dec_width[k],
                                             P.dec_smin2[k], P.dec_cut_smin[k], P.dec_smax[k]);
            auto it = dw_of.find(key);
            int id;
            if (it == dw_of.end()) {
                if (pp.n_dws >= PP_MAX_DWS) return false;
                id = pp.n_dws++;
                pp.dw_node[id] = static_cast<int8_t>(node[P.dec_parent[k]]);
                pp.dw_c1[id] = static_cast<int8_t>(node[P.dec_c1[k]]);
                pp.dw_c2[id] = static_cast<int8_t>(node[P.dec_c2[k]]);
                pp.dw_massless[id] = P.dec_massless[k];
                pp.dw_mass[id] = P.dec_mass[k];
                pp.dw_width[id] = P.dec_width[k];
                pp.dw_smin2[id] = P.dec_smin2[k];
                pp.dw_cut[id] = P.dec_cut_smin[k];
                pp.dw_smax[id] = P.dec_smax[k];
                // smin when smin1 < max(smin2, cut): evaluated with std::max
                // semantics in the same order as the device (Channel.cc:151)
                {
                    const double a = (0.0 < P.dec_smin2[k]) ? P.dec_smin2[k] : 0.0;
                    pp.dw_smin_c[id] = (a < P.dec_cut_smin[k]) ? P.dec_cut_smin[k] : a;
                }
                dw_of[key] = id;
            } else {
                id = it->second;
            }
            C.dw[k] = static_cast<int16_t>(id);
        }
        C.n_dec = static_cast<int8_t>(P.n_decay);
        std::vector<int> tents;
        for (int i = 0; i + 1 < P.n_info; ++i) {
            const auto key = std::make_tuple(node[P.info_slot[i]], P.info_ptmin[i], P.info_etamax[i]);
            auto it = tent_of.find(key);
            int id;
            if (it == tent_of.end()) {
                if (pp.n_tents >= PP_MAX_TENTS) return false;
                id = pp.n_tents++;
                pp.tent_node[id] = static_cast<int8_t>(node[P.info_slot[i]]);
                pp.tent_ptmin[id] = P.info_ptmin[i];
                pp.tent_etacut[id] = P.info_etamax[i];
                tent_of[key] = id;
            } else {
                id = it->second;
            }
            tents.push_back(id);
        }
        const int last = node[P.info_slot[P.n_info - 1]];
        auto ck = std::make_pair(tents, last);
        auto cit = chain_of.find(ck);
        int cid;
        if (cit == chain_of.end()) {
            if (pp.n_chains >= PP_MAX_CHAINS) return false;
            cid = pp.n_chains++;
            pp.chain_len[cid] = static_cast<int8_t>(tents.size());
            for (size_t t = 0; t < tents.size(); ++t) pp.chain_tent[cid][t] = static_cast<int8_t>(tents[t]);
            pp.chain_last[cid] = static_cast<int8_t>(last);
            chain_of[ck] = cid;
        } else {
            cid = cit->second;
        }
        C.chain = static_cast<int16_t>(cid);
        for (int k = 0; k < P.n_sdec; ++k) {
            const std::pair<int, int> key{node[P.sdec_a[k]], node[P.sdec_b[k]]};
            auto it = sw_of.find(key);
            int id;
            if (it == sw_of.end()) {
                if (pp.n_sws >= PP_MAX_SWS) return false;
                id = pp.n_sws++;
                pp.sw_a[id] = static_cast<int8_t>(key.first);
                pp.sw_b[id] = static_cast<int8_t>(key.second);
                sw_of[key] = id;
            } else {
                id = it->second;
            }
            C.sw[k] = static_cast<int16_t>(id);
        }
        C.n_sd = static_cast<int8_t>(P.n_sdec);
    }
    pp.n_nodes = n_nodes;
    pp.memo_tent = 0;
    pp.memo_dw = pp.memo_tent + 5 * pp.n_tents;
    pp.memo_sw = pp.memo_dw + 2 * pp.n_dws;
    pp.memo_chain = pp.memo_sw + 3 * pp.n_sws;
    pp.n_memo = pp.memo_chain + 2 * pp.n_chains;
    for (int c = 0; c < pp.nch; ++c) {
        const PPChannel &C = pp.ch[c];
        for (int fail = 0; fail < 2; ++fail) {
            int16_t *pos = fail ? pp.pos_src_fail[c] : pp.pos_src[c];
            int p = 0;
            for (int k = 0; k < C.n_dec; ++k) pos[p++] = static_cast<int16_t>(pp.memo_dw + 2 * C.dw[k] + 1);
            for (int i = 0; i < pp.chain_len[C.chain]; ++i) {
                const int t = pp.chain_tent[C.chain][i];
                for (int q = 0; q < 3; ++q) pos[p++] = static_cast<int16_t>(pp.memo_tent + 5 * t + 2 + q);
            }
            if (!fail) pos[p++] = static_cast<int16_t>(pp.memo_chain + 2 * C.chain + 1);
            for (int k = 0; k < C.n_sd; ++k) {
                pos[p++] = static_cast<int16_t>(pp.memo_sw + 3 * C.sw[k] + 1);
                pos[p++] = static_cast<int16_t>(pp.memo_sw + 3 * C.sw[k] + 2);
            }
            if (fail) pos[p++] = -1;
            if (p != pp.ndims) return false;
        }
    }
    return true;
}
