// construct.cpp -- host enumeration of the FSMapper channel descriptions of a
// process: the reference's ConstructChannels (src/Channel/ChannelNode.cc:
// 74-291), feeding chili_gpu_set_channels.  Setup-time code, not on the
// device path.
//
// The output order and the choice among descriptions that the reference's
// comparisons treat as equal are part of the result: ParticleInfo compares
// (idx, mass, width) and ignores the pid (ChannelNode.cc:293-306), a
// ChannelDescription compares its info list only (:308-316), and std::set
// keeps the first of equal elements.  So this file uses the same standard
// containers with the same comparisons and the same insertion sequence:
// std::unordered_map for the currents (its iteration order sets the order of
// the depth-first search), std::set / std::map for everything ordered.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <set>
#include <stack>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "chili_gpu.h"

namespace {

struct PInfo {
    uint32_t idx = 0;
    int pid = 0;
    double mass = 0, width = 0;
};

bool operator<(const PInfo &a, const PInfo &b) {
    if (a.idx == b.idx) {
        if (a.mass == b.mass) return a.width < b.width;
        return a.mass < b.mass;
    }
    return a.idx < b.idx;
}
bool operator==(const PInfo &a, const PInfo &b) { return a.mass == b.mass && a.idx == b.idx && a.width == b.width; }
bool operator!=(const PInfo &a, const PInfo &b) { return !(a == b); }
bool operator>(const PInfo &a, const PInfo &b) { return b < a && b != a; }

struct Greater {
    bool operator()(const PInfo &a, const PInfo &b) const { return a > b; }
};

using Prods = std::pair<PInfo, PInfo>;
using Currents = std::unordered_map<unsigned int, std::set<PInfo>>;
using Chain = std::map<PInfo, std::set<Prods>, Greater>;

struct Desc {
    std::vector<PInfo> info;
    std::map<PInfo, Prods> decays;
};

bool operator<(const Desc &a, const Desc &b) {
    if (a.info.size() == b.info.size()) {
        for (size_t i = 0; i < a.info.size(); ++i) {
            if (a.info[i] < b.info[i]) return true;
            if (a.info[i] > b.info[i]) return false;
        }
        return false;
    }
    return a.info.size() < b.info.size();
}

struct Frame {
    std::set<int> pid;
    std::vector<unsigned int> avail;
    std::vector<unsigned int> currents{};
    unsigned int idx_sum = 0;
    size_t schans = 0;
};

// Bit helpers of the enumeration (the reference's ChannelUtils.hh): the next
// integer with the same number of set bits (Anderson's bit hacks), set bits
// as their values, population count.
unsigned int next_same_popcount(unsigned int v) {
    const unsigned int t = v | (v - 1);
    return (t + 1) | (((~t & -~t) - 1) >> (__builtin_ctz(v) + 1));
}
std::vector<unsigned int> set_bit_values(unsigned int v, unsigned int n) {
    std::vector<unsigned int> out;
    for (unsigned int i = 0; i < n; ++i)
        if (v & (1u << i)) out.push_back(v & (1u << i));
    return out;
}
unsigned int popcount(unsigned int v) { return static_cast<unsigned int>(__builtin_popcount(v)); }

struct CutTables {
    std::vector<double> sexternal;
    std::map<std::pair<int, int>, double> deltaR;
    std::unordered_map<unsigned int, double> smin, ptmin, etamax;
};

struct Failure {
    std::string what;
};

class ModelView {
  public:
    explicit ModelView(const chili_model *m) : m_(m) {
        for (int i = 0; i < m->n_masses; ++i) mass_[m->masses[i].idx] = m->masses[i].value;
        for (int i = 0; i < m->n_widths; ++i) width_[m->widths[i].idx] = m->widths[i].value;
    }
    // Model::Mass / Width const (Model.hh:17-21): .at(|pid|), which throws in
    // the reference when the model does not know the flavour
    double mass(int pid) const { return lookup(mass_, pid, "mass"); }
    double width(int pid) const { return lookup(width_, pid, "width"); }
    std::vector<int> combinable(int f1, int f2) const {
        int32_t buf[64];
        const int n = m_->combinable(f1, f2, buf, 64, m_->user);
        if (n < 0 || n > 64)
            throw Failure{"Combinable(" + std::to_string(f1) + ", " + std::to_string(f2) +
                          ") returned " + std::to_string(n) + " (0..64 allowed)"};
        return std::vector<int>(buf, buf + n);
    }

  private:
    double lookup(const std::unordered_map<unsigned int, double> &t, int pid, const char *what) const {
        const auto it = t.find(static_cast<unsigned int>(std::abs(pid)));
        if (it == t.end()) throw Failure{std::string("the model has no ") + what + " for flavour " + std::to_string(pid)};
        return it->second;
    }
    const chili_model *m_;
    std::unordered_map<unsigned int, double> mass_, width_;
};

// The enumeration proper (ChannelNode.cc:98-291) on completed cut tables.
std::set<Desc> enumerate(const std::vector<int> &flavs, const ModelView &model, CutTables &cuts, size_t smax) {
    const unsigned int n = static_cast<unsigned int>(flavs.size());
    Currents comps;
    Chain chain;
    for (unsigned int i = 0; i < n; ++i) {
        PInfo p;
        p.idx = 1u << i;
        p.pid = flavs[i];
        p.mass = model.mass(p.pid);
        p.width = model.width(p.pid);
        comps[p.idx].insert(p);
    }
    // currents of 2 .. n-1 outgoing legs, at most smax + 1 legs each
    for (unsigned int nset = 2; nset < n; ++nset) {
        unsigned int cur = (1u << nset) - 1;
        while (cur < (1u << n) && popcount(cur) - 1 <= smax) {
            const auto legs = set_bit_values(cur, n);
            for (unsigned int iset = 1; iset < nset; ++iset) {
                unsigned int sel = (1u << iset) - 1;
                while (sel < (1u << (nset - 1))) {
                    unsigned int sub1 = 0;
                    for (unsigned int i = 0; i < legs.size(); ++i) sub1 += legs[i] * ((sel >> i) & 1);
                    const unsigned int sub2 = cur ^ sub1;
                    if ((sub1 & 1u) || (sub2 & 1u)) break;  // incoming legs never join a current
                    if ((sub1 & 2u) || (sub2 & 2u)) break;
                    if (comps.find(sub1) == comps.end() || comps.find(sub2) == comps.end()) {
                        sel = next_same_popcount(sel);
                        continue;
                    }
                    std::set<int> made;
                    for (const auto &a : comps[sub1])
                        for (const auto &b : comps[sub2]) {
                            const auto f = model.combinable(a.pid, b.pid);
                            made.insert(f.begin(), f.end());
                        }
                    if (made.empty()) {
                        sel = next_same_popcount(sel);
                        continue;
                    }
                    for (int f : made) {
                        PInfo p;
                        p.pid = f;
                        p.idx = cur;
                        p.mass = model.mass(f);
                        p.width = model.width(f);
                        comps[cur].insert(p);
                    }
                    cuts.ptmin[cur] = 0;
                    cuts.etamax[cur] = 99;
                    const auto left = comps[sub1];
                    const auto right = comps[sub2];
                    for (const auto &a : left)
                        for (const auto &b : right) {
                            for (int f : model.combinable(a.pid, b.pid)) {
                                PInfo p;
                                p.pid = f;
                                p.idx = cur;
                                p.mass = model.mass(f);
                                p.width = model.width(f);
                                if (a < b) chain[p].insert({a, b});
                                else chain[p].insert({b, a});
                            }
                        }
                    sel = next_same_popcount(sel);
                }
            }
            cur = next_same_popcount(cur);
        }
    }

    // depth-first search over ordered sequences of disjoint currents whose
    // flavours chain from the first incoming leg (the t-channel lists)
    std::vector<unsigned int> avail;
    for (const auto &c : comps) avail.push_back(c.first);
    std::stack<Frame> st;
    const unsigned int full = (1u << n) - 1;
    st.push(Frame{std::set<int>{comps[1].begin()->pid}, avail});
    std::set<Desc> channels;
    while (!st.empty()) {
        Frame top = st.top();
        st.pop();
        if (top.idx_sum > full) continue;
        if (top.idx_sum == full) {
            std::vector<Desc> old(1);
            for (unsigned int c : top.currents) {
                if (c == 1 || c == 2) continue;
                std::vector<PInfo> opts;
                for (const auto &ci : comps[c]) opts.push_back(PInfo{c, ci.pid, model.mass(ci.pid), model.width(ci.pid)});
                std::vector<Desc> next;
                for (const auto &d : old)
                    for (const auto &o : opts) {
                        Desc e = d;
                        e.info.push_back(o);
                        std::sort(e.info.begin(), e.info.end(), Greater{});
                        next.push_back(e);
                    }
                old = next;
            }
            channels.insert(old.begin(), old.end());
            continue;
        }
        if (top.avail.empty()) continue;
        for (size_t i = 0; i < top.avail.size(); ++i) {
            Frame d = top;
            d.schans += popcount(top.avail[i]) - 1;
            if (d.schans > smax) continue;
            if (d.idx_sum & top.avail[i]) continue;
            std::set<int> made;
            for (int p1 : d.pid)
                for (const auto &ci : comps[top.avail[i]]) {
                    const auto f = model.combinable(p1, ci.pid);
                    made.insert(f.begin(), f.end());
                }
            if (made.empty()) continue;
            d.pid = made;
            d.idx_sum += top.avail[i];
            d.currents.push_back(top.avail[i]);
            d.avail.erase(d.avail.begin() + static_cast<long>(i));
            st.push(d);
        }
    }

    // the s-channel decays, parents in descending order
    for (const auto &dec : chain) {
        std::set<Desc> next;
        for (const auto &ch : channels) {
            bool add = std::binary_search(ch.info.begin(), ch.info.end(), dec.first, Greater{});
            for (const auto &pr : ch.decays) add |= pr.second.first == dec.first || pr.second.second == dec.first;
            if (add) {
                for (const auto &prods : dec.second) {
                    Desc c = ch;
                    c.decays[dec.first] = prods;
                    next.insert(c);
                }
            } else {
                next.insert(ch);
            }
        }
        channels = next;
    }
    return channels;
}

}  // namespace

struct chili_channel_list {
    std::vector<std::vector<chili_particle_info>> infos;
    std::vector<std::vector<chili_decay>> decays;
    std::vector<chili_channel_desc> descs;
    std::vector<double> sexternal;
    std::vector<chili_pid_pair_value> deltaR;
    std::vector<chili_idx_value> smin, ptmin, etamax;
    chili_cuts cuts{};
};

namespace {

chili_particle_info to_c(const PInfo &p) { return chili_particle_info{p.idx, p.pid, p.mass, p.width}; }

std::vector<chili_idx_value> sorted_table(const std::unordered_map<unsigned int, double> &t) {
    std::vector<chili_idx_value> v;
    for (const auto &kv : t) v.push_back(chili_idx_value{kv.first, kv.second});
    std::sort(v.begin(), v.end(), [](const chili_idx_value &a, const chili_idx_value &b) { return a.idx < b.idx; });
    return v;
}

void set_err(char *err, size_t len, const std::string &msg) {
    if (err && len) std::snprintf(err, len, "%s", msg.c_str());
}

}  // namespace

extern "C" {

int chili_construct_channels(double sqrts, const int32_t *flavs, int n_flavs, const chili_model *model,
                             const chili_cuts *cuts, int smax, chili_channel_list **out, char *err, size_t err_len) {
    set_err(err, err_len, "");
    if (!flavs || !model || !model->combinable || !out || n_flavs < 3 || n_flavs > CHILI_MAX_EXT || smax < 0 ||
        !(sqrts > 0) || (model->n_masses > 0 && !model->masses) || (model->n_widths > 0 && !model->widths)) {
        set_err(err, err_len, "flavours (3..CHILI_MAX_EXT), model with Combinable, smax >= 0, sqrts > 0 required");
        return CHILI_ERR_INVALID_ARG;
    }
    *out = nullptr;
    (void)sqrts;  // the FSMapper construction happens in chili_gpu_set_channels
    const std::vector<int> fl(flavs, flavs + n_flavs);
    try {
        const ModelView mv(model);
        CutTables ct;
        if (!cuts) {
            // the first ConstructChannels overload (ChannelNode.cc:74-96):
            // Delta R 0.4 between every pair of flavours (0 with a top),
            // pT > 30 and |eta| < 99 on every leg, smin = m^2
            for (int f1 : fl)
                for (int f2 : fl) ct.deltaR[{f1, f2}] = (std::abs(f1) == 6 || std::abs(f2) == 6) ? 0.0 : 0.4;
            for (int i = 0; i < n_flavs; ++i) {
                const unsigned int idx = 1u << i;
                const double m = mv.mass(fl[i]);
                ct.smin[idx] = m * m;
                ct.ptmin[idx] = 30;
                ct.etamax[idx] = 99;
                if (i > 1) ct.sexternal.push_back(m * m);
            }
        } else {
            if ((cuts->n_sexternal > 0 && !cuts->sexternal) || (cuts->n_deltaR > 0 && !cuts->deltaR) ||
                (cuts->n_smin > 0 && !cuts->smin) || (cuts->n_ptmin > 0 && !cuts->ptmin) ||
                (cuts->n_etamax > 0 && !cuts->etamax)) {
                set_err(err, err_len, "cut table with a count but no entries");
                return CHILI_ERR_INVALID_ARG;
            }
            ct.sexternal.assign(cuts->sexternal, cuts->sexternal + cuts->n_sexternal);
            for (int i = 0; i < cuts->n_deltaR; ++i) ct.deltaR[{cuts->deltaR[i].pid1, cuts->deltaR[i].pid2}] = cuts->deltaR[i].value;
            for (int i = 0; i < cuts->n_smin; ++i) ct.smin[cuts->smin[i].idx] = cuts->smin[i].value;
            for (int i = 0; i < cuts->n_ptmin; ++i) ct.ptmin[cuts->ptmin[i].idx] = cuts->ptmin[i].value;
            for (int i = 0; i < cuts->n_etamax; ++i) ct.etamax[cuts->etamax[i].idx] = cuts->etamax[i].value;
        }
        const std::set<Desc> chans = enumerate(fl, mv, ct, static_cast<size_t>(smax));
        auto *L = new chili_channel_list();
        for (const auto &d : chans) {
            std::vector<chili_particle_info> info;
            for (const auto &p : d.info) info.push_back(to_c(p));
            std::vector<chili_decay> dec;
            for (const auto &kv : d.decays) dec.push_back(chili_decay{to_c(kv.first), to_c(kv.second.first), to_c(kv.second.second)});
            L->infos.push_back(std::move(info));
            L->decays.push_back(std::move(dec));
        }
        for (size_t i = 0; i < L->infos.size(); ++i)
            L->descs.push_back(chili_channel_desc{static_cast<int32_t>(L->infos[i].size()), L->infos[i].data(),
                                                  static_cast<int32_t>(L->decays[i].size()), L->decays[i].data()});
        L->sexternal = ct.sexternal;
        for (const auto &kv : ct.deltaR) L->deltaR.push_back(chili_pid_pair_value{kv.first.first, kv.first.second, kv.second});
        L->smin = sorted_table(ct.smin);
        L->ptmin = sorted_table(ct.ptmin);
        L->etamax = sorted_table(ct.etamax);
        L->cuts = chili_cuts{static_cast<int32_t>(L->sexternal.size()), L->sexternal.data(),
                             static_cast<int32_t>(L->deltaR.size()), L->deltaR.data(),
                             static_cast<int32_t>(L->smin.size()), L->smin.data(),
                             static_cast<int32_t>(L->ptmin.size()), L->ptmin.data(),
                             static_cast<int32_t>(L->etamax.size()), L->etamax.data()};
        *out = L;
        return CHILI_OK;
    } catch (const Failure &f) {
        set_err(err, err_len, f.what);
        return CHILI_ERR_INVALID_ARG;
    } catch (const std::exception &e) {
        set_err(err, err_len, e.what());
        return CHILI_ERR_INVALID_ARG;
    }
}

int chili_channel_list_get(const chili_channel_list *list, const chili_channel_desc **descs, int *nch,
                           const chili_cuts **cuts) {
    if (!list) return CHILI_ERR_INVALID_ARG;
    if (descs) *descs = list->descs.empty() ? nullptr : list->descs.data();
    if (nch) *nch = static_cast<int>(list->descs.size());
    if (cuts) *cuts = &list->cuts;
    return CHILI_OK;
}

void chili_channel_list_free(chili_channel_list *list) { delete list; }

}  // extern "C"
