// ref_driver.cc -- flat C entry points over the UNMODIFIED Chili reference
// sources, compiled into oracle/_ref/libchili_ref.so by oracle/Makefile.
//
// TEST INFRASTRUCTURE ONLY: used by tests/, by bench.py's CPU-baseline and
// reference legs, and to pin the C restatement in oracle/port/.  Nothing in
// the product links it.
//
// Every arithmetic step below is a call into the reference (AdaptiveMap,
// Vegas, StatsData, FSMapper, Integrand, MultiChannel); the driver only
// supplies inputs that the reference normally draws from its global mt19937
// (Random.hh:8-52).  Those uniforms are handed to the real libstdc++
// distributions through ReplayEngine, a URNG whose two 32-bit outputs make
// std::generate_canonical<double,53> return the given 53-bit uniform exactly.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <limits>
#include <memory>
#include <random>
#include <sstream>
#include <stdexcept>
#include <unordered_map>
#include <vector>

#include "Channel/Channel.hh"
#include "Channel/ChannelNode.hh"
#include "Channel/Integrand.hh"
#include "Channel/MultiChannel.hh"
#include "Model/Model.hh"
#include "Integrator/AdaptiveMap.hh"
#include "Integrator/Statistics.hh"
#include "Integrator/Vegas.hh"
#include "Tools/Cuts.hh"
#include "Tools/FourVector.hh"

#include "chili_gpu.h"

// MultiChannel keeps its channel weights private; it befriends
// YAML::convert<MultiChannel> (MultiChannel.hh:116), which this driver
// defines to read and write them.
namespace YAML {
template <> struct convert<chili::MultiChannel> {
    static std::vector<double> &alpha(chili::MultiChannel &m) { return m.channel_weights; }
    static std::vector<double> &best(chili::MultiChannel &m) { return m.best_weights; }
    static double &min_diff(chili::MultiChannel &m) { return m.min_diff; }
};
}  // namespace YAML

namespace {

using chili::FourVector;
using MCAccess = YAML::convert<chili::MultiChannel>;

// Replays a given uniform u = k * 2^-53 through generate_canonical<double,53>
// of a 32-bit engine: sum = lo + hi * 2^32 = u * 2^64 exactly.
struct ReplayEngine {
    using result_type = uint32_t;
    static constexpr result_type min() { return 0; }
    static constexpr result_type max() { return 0xffffffffu; }
    uint32_t words[2]{};
    int next = 0;
    explicit ReplayEngine(double u) {
        const uint64_t k = static_cast<uint64_t>(std::ldexp(u, 64));
        words[0] = static_cast<uint32_t>(k & 0xffffffffu);
        words[1] = static_cast<uint32_t>(k >> 32);
    }
    result_type operator()() { return words[next++ & 1]; }
};

double replay_uniform(double u) {
    ReplayEngine eng(u);
    std::uniform_real_distribution<double> dist;  // Random::Generate (Random.hh:19-21)
    return dist(eng);
}

size_t replay_select(const std::vector<double> &alpha, double u) {
    ReplayEngine eng(u);  // Random::SelectIndex (Random.hh:43-45)
    std::discrete_distribution<size_t> dist(alpha.begin(), alpha.end());
    return dist(eng);
}

void fill_stats(const chili::StatsData &s, chili_stats *out) {
    std::memcpy(out, &s, sizeof(chili_stats));  // 6 doubles, same order
}

chili::ParticleInfo to_info(const chili_particle_info &p) {
    chili::ParticleInfo info;
    info.idx = p.idx;
    info.pid = p.pid;
    info.mass = p.mass;
    info.width = p.width;
    return info;
}

chili::Cuts to_cuts(const chili_cuts *c) {
    chili::Cuts cuts;
    for (int i = 0; i < c->n_sexternal; ++i) cuts.sexternal.push_back(c->sexternal[i]);
    for (int i = 0; i < c->n_deltaR; ++i)
        cuts.deltaR[{c->deltaR[i].pid1, c->deltaR[i].pid2}] = c->deltaR[i].value;
    for (int i = 0; i < c->n_smin; ++i) cuts.smin[c->smin[i].idx] = c->smin[i].value;
    for (int i = 0; i < c->n_ptmin; ++i) cuts.ptmin[c->ptmin[i].idx] = c->ptmin[i].value;
    for (int i = 0; i < c->n_etamax; ++i) cuts.etamax[c->etamax[i].idx] = c->etamax[i].value;
    return cuts;
}

chili::ChannelDescription to_desc(const chili_channel_desc &d) {
    chili::ChannelDescription desc;
    for (int i = 0; i < d.n_info; ++i) desc.info.push_back(to_info(d.info[i]));
    for (int i = 0; i < d.n_decays; ++i)
        desc.decays[to_info(d.decays[i].parent)] = {to_info(d.decays[i].child1),
                                                     to_info(d.decays[i].child2)};
    return desc;
}

// ---------------------------------------------------------------- integrands
// These are the user callbacks (Integrand.hh:41-47); they are not reference
// code and are written identically in oracle/port and in the CUDA kernels.
double camel(const std::vector<double> &x, const std::vector<double> &p) {
    const size_t d = x.size();
    const double s = p[0], norm = p[1];
    double d1 = 0, d2 = 0;
    for (size_t i = 0; i < d; ++i) {
        double t = x[i] - p[2 + i];
        d1 += t * t;
        t = x[i] - p[2 + d + i];
        d2 += t * t;
    }
    const double s2 = s * s;
    return norm * (std::exp(-d1 / s2) + std::exp(-d2 / s2));
}

double propagator(const std::vector<FourVector> &mom, const std::vector<double> &p, bool top2) {
    const double m2 = p[0] * p[0], mw2 = p[0] * p[0] * p[1] * p[1], mt2 = p[2] * p[2];
    const size_t n = mom.size();
    double sum = 0, big1 = 0, big2 = 0;
    for (size_t i = 2; i < n; ++i) {
        for (size_t j = i + 1; j < n; ++j) {
            const double d = (mom[i] + mom[j]).Mass2() - m2;
            const double bw = 1.0 / (d * d + mw2);
            sum += bw;
            if (bw > big1) {
                big2 = big1;
                big1 = bw;
            } else if (bw > big2) {
                big2 = bw;
            }
        }
    }
    double tprod = 1;
    for (size_t j = 2; j < n; ++j) tprod *= 1.0 / (std::abs((mom[0] + mom[j]).Mass2()) + mt2);
    return (top2 ? big1 * big2 : sum) * tprod;
}

// The reference logs through spdlog inside the hot loop (e.g.
// ChannelElements.cc:92,99) and writes NaN retries to std::cerr
// (MultiChannel.hh:231-232).  The driver silences both so that the CPU
// baseline is timed on arithmetic, not on terminal I/O.
struct Quiet {
    std::streambuf *saved;
    Quiet() : saved(std::cerr.rdbuf(nullptr)) { spdlog::set_level(spdlog::level::off); }
    ~Quiet() {
        std::cerr.clear();
        std::cerr.rdbuf(saved);
    }
};

struct MC {
    int n_ext = 0, ndims = 0, bins = 0;
    chili::Integrand<FourVector> integrand;
    chili::MultiChannel mc;
    chili_multichannel_params params{};
    std::vector<double> fparams;
    int fkind = CHILI_FUNC_UNIT;
    int pre = CHILI_PRE_FINITE;
    // last-iteration training data, copied out before Train() clears it
    std::vector<double> last_hist, last_atrain;
    uint64_t dropped_dim0 = 0;
    // the reference's MPI mode with the all-reduce done by the caller: an
    // iteration collects its training data and leaves MultiChannel::Train
    // to ref_mc_train, which runs it on the ranks' summed data
    int defer = 0;
};

}  // namespace

extern "C" {

// ------------------------------------------------------------- AdaptiveMap
static chili::AdaptiveMap make_map(int dims, int bins, const double *edges) {
    chili::AdaptiveMap map(static_cast<size_t>(dims), static_cast<size_t>(bins));
    if (edges) std::memcpy(map.Hist().data(), edges, sizeof(double) * dims * (bins + 1));
    return map;
}

void ref_am_map(int dims, int bins, const double *edges, const double *u, int64_t n,
                double *x, double *jac) {
    auto map = make_map(dims, bins, edges);
    std::vector<double> r(dims);
    for (int64_t i = 0; i < n; ++i) {
        for (int d = 0; d < dims; ++d) r[d] = u[i * dims + d];
        jac[i] = map(r);
        for (int d = 0; d < dims; ++d) x[i * dims + d] = r[d];
    }
}

void ref_am_weight(int dims, int bins, const double *edges, const double *x, int64_t n,
                   double *w, int32_t *bin) {
    auto map = make_map(dims, bins, edges);
    std::vector<double> r(dims);
    for (int64_t i = 0; i < n; ++i) {
        for (int d = 0; d < dims; ++d) {
            r[d] = x[i * dims + d];
            if (bin) {
                const size_t b = map.FindBin(d, r[d]);
                bin[i * dims + d] = b == std::numeric_limits<size_t>::max() ? -1 : static_cast<int32_t>(b);
            }
        }
        if (w) {
            // GenerateWeight reads width(i, FindBin) which is out of range for
            // FindBin == SIZE_MAX; the driver reports NaN there instead of
            // reading outside the edge table.
            bool bad = false;
            for (int d = 0; d < dims; ++d)
                if (map.FindBin(d, r[d]) == std::numeric_limits<size_t>::max()) bad = true;
            w[i] = bad ? std::nan("") : map.GenerateWeight(r);
        }
    }
}

void ref_am_adapt(int dims, int bins, const double *edges, double alpha, const double *train,
                  double *new_edges) {
    auto map = make_map(dims, bins, edges);
    std::vector<double> data(train, train + dims * bins);
    map.Adapt(alpha, data);
    std::memcpy(new_edges, map.Hist().data(), sizeof(double) * dims * (bins + 1));
}

void ref_am_split(int dims, int bins, const double *edges, int nsplit, double *new_edges) {
    auto map = make_map(dims, bins, edges);
    chili::AdaptiveMapSplit s = nsplit == 2   ? chili::AdaptiveMapSplit::half
                                : nsplit == 3 ? chili::AdaptiveMapSplit::third
                                              : chili::AdaptiveMapSplit::quarter;
    map.Split(s);
    std::memcpy(new_edges, map.Hist().data(), sizeof(double) * dims * (nsplit * bins + 1));
}

// --------------------------------------------------------------------- Vegas
// One Vegas::operator() (Vegas.cc:18-52) with the uniforms u[n*dims] in place
// of Random::Generate.  edges is updated in place when adapt != 0.
void ref_vegas_iterate(int dims, int bins, double *edges, double alpha, int adapt,
                       const double *params, int nparams, int64_t n, const double *u,
                       chili_stats *stats, double *train_out) {
    auto grid = make_map(dims, bins, edges);
    std::vector<double> p(params, params + nparams);
    std::vector<double> rans(dims), train(dims * bins);
    chili::StatsData results;
    for (int64_t i = 0; i < n; ++i) {
        for (int d = 0; d < dims; ++d) rans[d] = replay_uniform(u[i * dims + d]);
        const double wgt = grid(rans);
        const double val = camel(rans, p) * wgt;
        const double val2 = val * val;
        results += val;
        for (int j = 0; j < dims; ++j) {
            // Vegas.cc:41 with FindBin == SIZE_MAX in dimension 0 writes before
            // the histogram (heap corruption in the reference); skipped here
            const size_t b = grid.FindBin(j, rans[j]);
            if (j == 0 && b == std::numeric_limits<size_t>::max()) continue;
            train[j * bins + b] += val2;
        }
    }
    if (train_out) std::memcpy(train_out, train.data(), sizeof(double) * dims * bins);
    if (adapt) {
        grid.Adapt(alpha, train);
        std::memcpy(edges, grid.Hist().data(), sizeof(double) * dims * (bins + 1));
    }
    fill_stats(results, stats);
}

// The reference's own Vegas loop with its own mt19937 (Random.hh:49): niter
// calls of Vegas::operator() on the camel; returns the pooled StatsData.
void ref_vegas_run(int dims, int bins, double alpha, const double *params, int nparams,
                   unsigned seed, int64_t ncalls, int niter, chili_stats *out) {
    chili::Random::Instance().Seed(seed);
    chili::VegasParams vp;
    vp.ncalls = static_cast<size_t>(ncalls);
    vp.alpha = alpha;
    vp.nrefine = 0;
    chili::Vegas vegas(chili::AdaptiveMap(dims, bins), vp);
    vegas.SetVerbosity(0);
    std::vector<double> p(params, params + nparams);
    chili::Func<double> f = [p](const std::vector<double> &x) { return camel(x, p); };
    for (int it = 0; it < niter; ++it) vegas(f);
    const auto sum = vegas.Summary().sum_results;  // Vegas.hh:40-45
    fill_stats(sum, out);
}

// -------------------------------------------------------------- MultiChannel
void *ref_mc_create(const chili_channel_desc *descs, int nch, const chili_cuts *cuts,
                    double sqrts, int n_ext, int bins, const chili_multichannel_params *params) {
    try {
        auto *h = new MC();
        h->n_ext = n_ext;
        h->bins = bins;
        h->params = *params;
        const chili::Cuts c = to_cuts(cuts);
        for (int i = 0; i < nch; ++i) {
            chili::Channel<FourVector> channel;
            channel.mapping = std::make_unique<chili::FSMapper>(sqrts, static_cast<size_t>(n_ext),
                                                                to_desc(descs[i]), c);
            chili::VegasParams vp;
            vp.alpha = params->grid_alpha;
            channel.integrator = chili::Vegas(chili::AdaptiveMap(channel.mapping->NDims(), bins), vp);
            h->integrand.AddChannel(std::move(channel));
        }
        h->ndims = static_cast<int>(h->integrand.NDims());
        chili::MultiChannelParams mp;
        mp.ncalls = params->ncalls;
        mp.niterations = params->niterations;
        mp.rtol = params->rtol;
        mp.nrefine = params->nrefine;
        mp.beta = params->beta;
        mp.min_alpha = params->min_alpha;
        mp.refine_size = params->refine_size;
        mp.max_bins = params->max_bins;
        mp.should_optimize = params->should_optimize != 0;
        h->mc = chili::MultiChannel(h->integrand.NDims(), h->integrand.NChannels(), mp);
        h->integrand.PostProcess() = [](const std::vector<FourVector> &, double) { return true; };
        return h;
    } catch (...) {
        return nullptr;
    }
}

void ref_mc_destroy(void *p) { delete static_cast<MC *>(p); }
int ref_mc_ndims(void *p) { return static_cast<MC *>(p)->ndims; }

void ref_mc_set_integrand(void *p, int kind, const double *params, int nparams, int pre) {
    auto *h = static_cast<MC *>(p);
    h->fkind = kind;
    h->fparams.assign(params, params + nparams);
    h->pre = pre;
    const std::vector<double> fp = h->fparams;
    if (kind == CHILI_FUNC_UNIT) {
        h->integrand.Function() = [](const std::vector<FourVector> &) { return 1.0; };
    } else {
        const bool top2 = kind == CHILI_FUNC_PROPAGATOR_TOP2;
        h->integrand.Function() = [fp, top2](const std::vector<FourVector> &m) {
            return propagator(m, fp, top2);
        };
    }
    if (pre == CHILI_PRE_FINITE)  // src/example.cc:26-29
        h->integrand.PreProcess() = [](const std::vector<FourVector> &m) { return !std::isnan(m[0][0]); };
    else
        h->integrand.PreProcess() = [](const std::vector<FourVector> &) { return true; };
}

// CHILI_PRE_CUTS (include/chili_gpu.h) as the PreProcess callback of this
// harness (the reference's own example filters with JetCluster instead,
// src/example.cc:25-52); the same arithmetic as the CUDA library and the port.
void ref_mc_set_cuts(void *p, double sqrts, double ptmin, double etamax, double dr) {
    auto *h = static_cast<MC *>(p);
    h->pre = CHILI_PRE_CUTS;
    const int ne = h->n_ext;
    h->integrand.PreProcess() = [=](const std::vector<FourVector> &m) {
        const double half = 0.5 * sqrts * (1.0 + 1e-12);
        if (!(-m[0][0] <= half) || !(-m[1][0] <= half)) return false;
        double eta[CHILI_MAX_EXT], phi[CHILI_MAX_EXT];
        for (int i = 2; i < ne; ++i) {
            const double pt2 = m[i][1] * m[i][1] + m[i][2] * m[i][2];
            if (!(pt2 >= ptmin * ptmin) || !(pt2 > 0)) return false;
            eta[i] = std::asinh(m[i][3] / std::sqrt(pt2));
            if (!(std::fabs(eta[i]) <= etamax)) return false;
            phi[i] = std::atan2(m[i][2], m[i][1]);
        }
        for (int i = 2; i < ne; ++i)
            for (int j = i + 1; j < ne; ++j) {
                double dphi = std::fabs(phi[i] - phi[j]);
                if (dphi > 3.14159265358979323846) dphi = 2.0 * 3.14159265358979323846 - dphi;
                const double deta = eta[i] - eta[j];
                if (!(deta * deta + dphi * dphi >= dr * dr)) return false;
            }
        return true;
    };
}

// MultiChannel::SaveAs / LoadFrom (MultiChannel.hh:65-84), the reference's
// own serialisation.
int ref_mc_save(void *p, const char *path) {
    auto *h = static_cast<MC *>(p);
    return h->mc.SaveAs(h->integrand, std::string(path)) ? 0 : 1;
}
int ref_mc_load(void *p, const char *path) {
    auto *h = static_cast<MC *>(p);
    return h->mc.LoadFrom(h->integrand, std::string(path)) ? 0 : 1;
}

void ref_mc_set_grids(void *p, const double *edges) {
    auto *h = static_cast<MC *>(p);
    const size_t per = static_cast<size_t>(h->ndims) * (h->bins + 1);
    for (size_t c = 0; c < h->integrand.NChannels(); ++c)
        std::memcpy(h->integrand.GetChannel(c).integrator.Grid().Hist().data(), edges + c * per,
                    sizeof(double) * per);
}

void ref_mc_get_grids(void *p, double *edges) {
    auto *h = static_cast<MC *>(p);
    const size_t per = static_cast<size_t>(h->ndims) * (h->bins + 1);
    for (size_t c = 0; c < h->integrand.NChannels(); ++c)
        std::memcpy(edges + c * per, h->integrand.GetChannel(c).integrator.Grid().Hist().data(),
                    sizeof(double) * per);
}

void ref_mc_set_alpha(void *p, const double *alpha) {
    auto *h = static_cast<MC *>(p);
    auto &a = MCAccess::alpha(h->mc);
    std::memcpy(a.data(), alpha, sizeof(double) * a.size());
}

void ref_mc_get_alpha(void *p, double *alpha, double *best, double *min_diff) {
    auto *h = static_cast<MC *>(p);
    auto &a = MCAccess::alpha(h->mc);
    if (alpha) std::memcpy(alpha, a.data(), sizeof(double) * a.size());
    auto &b = MCAccess::best(h->mc);
    if (best) {
        for (size_t i = 0; i < a.size(); ++i) best[i] = i < b.size() ? b[i] : std::nan("");
    }
    if (min_diff) *min_diff = MCAccess::min_diff(h->mc);
}

void ref_fsm_generate(void *p, int ch, const double *x, int64_t n, double *mom) {
    auto *h = static_cast<MC *>(p);
    Quiet quiet;
    auto &mapping = h->integrand.GetChannel(ch).mapping;
    std::vector<double> r(h->ndims);
    std::vector<FourVector> point;
    for (int64_t i = 0; i < n; ++i) {
        for (int d = 0; d < h->ndims; ++d) r[d] = x[i * h->ndims + d];
        mapping->GeneratePoint(point, r);
        for (int k = 0; k < h->n_ext; ++k)
            for (int c = 0; c < 4; ++c) mom[(i * h->n_ext + k) * 4 + c] = point[k][c];
    }
}

static void load_point(const MC *h, const double *mom, int64_t i, std::vector<FourVector> &point) {
    point.resize(h->n_ext);
    for (int k = 0; k < h->n_ext; ++k) {
        const double *q = mom + (i * h->n_ext + k) * 4;
        point[k] = FourVector(q[0], q[1], q[2], q[3]);
    }
}

void ref_fsm_weight(void *p, int ch, const double *mom, int64_t n, double *x_out, double *w) {
    auto *h = static_cast<MC *>(p);
    Quiet quiet;
    auto &mapping = h->integrand.GetChannel(ch).mapping;
    std::vector<double> r;
    std::vector<FourVector> point;
    for (int64_t i = 0; i < n; ++i) {
        load_point(h, mom, i, point);
        r.assign(h->ndims, 0.0);  // positions the mapping leaves unwritten read 0
        w[i] = mapping->GenerateWeight(point, r);
        if (x_out)
            for (int d = 0; d < h->ndims; ++d) x_out[i * h->ndims + d] = r[d];
    }
}

void ref_select(const double *alpha, int nch, const double *v, int64_t n, int32_t *out) {
    std::vector<double> a(alpha, alpha + nch);
    for (int64_t i = 0; i < n; ++i) out[i] = static_cast<int32_t>(replay_select(a, v[i]));
}

// Integrand::GenerateWeight through MultiChannel::GenerateWeight
// (MultiChannel.hh:152-165) with the current channel weights.
void ref_mc_weight(void *p, const double *mom, const int32_t *ich, int64_t n, double *wgt,
                   double *dens, double *x_ich) {
    auto *h = static_cast<MC *>(p);
    Quiet quiet;
    const size_t nch = h->integrand.NChannels();
    std::vector<double> densities(nch), rans;
    std::vector<FourVector> point;
    for (int64_t i = 0; i < n; ++i) {
        load_point(h, mom, i, point);
        rans.assign(h->ndims, 0.0);
        wgt[i] = h->mc.GenerateWeight(h->integrand, point, static_cast<size_t>(ich[i]),
                                      std::ref(densities), std::ref(rans));
        if (dens) std::memcpy(dens + i * nch, densities.data(), sizeof(double) * nch);
        if (x_ich)
            for (int d = 0; d < h->ndims; ++d) x_ich[i * h->ndims + d] = rans[d];
    }
}

// One MultiChannel::operator() (MultiChannel.hh:196-251) with the uniforms
// u[k*(ndims+1)...] in place of the global generator.  The per-point body
// calls the same reference members in the same order.  Two places differ:
//  * guard != 0 drops non-finite alpha-training terms (the build's documented
//    deviation); guard == 0 calls MultiChannel::AddTrainData as is;
//  * a FindBin of SIZE_MAX in dimension 0 would index before the histogram
//    (Integrand.hh:91-95); that single add is skipped and counted.
// Returns 0, or 6 (CHILI_ERR_LIMIT) if u runs out before ncalls are accepted.
int ref_mc_iterate(void *p, const double *u, int64_t n_u, int guard, chili_stats *stats,
                   chili_mc_iter_info *info) {
    auto *h = static_cast<MC *>(p);
    auto &func = h->integrand;
    auto &mc = h->mc;
    Quiet quiet;
    const size_t nch = func.NChannels();
    const size_t ndims = static_cast<size_t>(h->ndims);
    std::vector<double> rans(ndims);
    std::vector<FourVector> point(ndims);
    std::vector<double> densities(nch), train_data(nch);
    chili::StatsData results;
    func.InitializeTrain();
    std::memset(info, 0, sizeof(*info));
    const size_t ncalls = h->params.ncalls;
    int64_t k = 0;
    for (size_t i = 0; i < ncalls; ++i) {
        if (k >= n_u) return CHILI_ERR_LIMIT;
        const double *uk = u + k * (ndims + 1);
        ++k;
        // MultiChannel::GeneratePoint (MultiChannel.hh:141-150)
        for (size_t d = 0; d < ndims; ++d) rans[d] = replay_uniform(uk[d]);
        const size_t ichannel = nch < 2 ? 0 : replay_select(MCAccess::alpha(mc), uk[ndims]);
        func.GeneratePoint(ichannel, rans, point);
        if (!func.PreProcess()(point)) {
            --i;
            results += 0;
            info->rejected_pre++;
            continue;
        }
        double wgt = mc.GenerateWeight(func, point, ichannel, std::ref(densities), std::ref(rans));
        const double f = func(point);
        double val = wgt == 0 ? 0 : f * wgt;
        if (std::isnan(val)) {
            val = wgt = 0;
            i--;
            info->rejected_nan++;
        }
        if (h->params.should_optimize) {
            const auto &grid = func.GetChannel(ichannel).integrator.Grid();
            const bool dim0_bad = grid.FindBin(0, rans[0]) == std::numeric_limits<size_t>::max();
            const double val2 = val * val;
            if (!guard && !dim0_bad) {
                mc.AddTrainData(func, ichannel, val, wgt, train_data, rans, densities);
            } else {
                auto &td = func.GetChannel(ichannel).train_data;
                for (size_t j = 0; j < ndims; ++j) {
                    const size_t b = grid.FindBin(j, rans[j]);
                    if (j == 0 && b == std::numeric_limits<size_t>::max()) {
                        h->dropped_dim0++;
                        continue;
                    }
                    td[j * grid.Bins() + b] += val2;
                }
                for (size_t j = 0; j < nch; ++j) {
                    const double term = val2 * wgt / densities[j];
                    if (guard && !std::isfinite(term)) {
                        info->nonfinite_alpha_terms += 1;
                        continue;
                    }
                    train_data[j] += term;
                }
            }
        }
        if (!func.PostProcess()(point, val)) {
            i--;
            val = 0;
        }
        if (val > info->weight_max) info->weight_max = val;
        results += val;
    }
    info->points_tried = static_cast<uint64_t>(k);
    info->points_accepted = ncalls;
    info->points_weighted = ncalls + info->rejected_nan;
    h->last_hist.assign(nch * ndims * h->bins, 0.0);
    for (size_t c = 0; c < nch; ++c) {
        const auto &td = func.GetChannel(c).train_data;
        std::memcpy(h->last_hist.data() + c * ndims * h->bins, td.data(), sizeof(double) * td.size());
    }
    h->last_atrain = train_data;
    if (h->params.should_optimize && !h->defer) mc.Train(func, train_data);
    mc.UpdateResults(results);
    fill_stats(results, stats);
    return 0;
}

void ref_mc_set_defer(void *p, int defer) { static_cast<MC *>(p)->defer = defer; }

// MultiChannel::Train (MultiChannel.hh:182-194) on given training data: the
// step that follows the MPI all-reduce of the alpha-training sums and of
// every channel's histogram (MultiChannel.hh:184-190), with the sums of all
// ranks in place of the all-reduce.  The reference's own Train runs: Adapt,
// Integrand::Train, MaxDifference.
void ref_mc_train(void *p, const double *hist, const double *atrain) {
    auto *h = static_cast<MC *>(p);
    Quiet quiet;
    auto &func = h->integrand;
    const size_t nch = func.NChannels(), per = static_cast<size_t>(h->ndims) * h->bins;
    for (size_t c = 0; c < nch; ++c) {
        auto &td = func.GetChannel(c).train_data;
        td.assign(hist + c * per, hist + (c + 1) * per);
    }
    std::vector<double> train_data(atrain, atrain + nch);
    h->mc.Train(func, train_data);
}

// The reference's own uniform stream: Random::Instance() seeded with `seed`
// (Random.hh:15-21), then n draws of Generate, in the order Vegas::operator()
// consumes them (Vegas.cc:32).
void ref_random_uniforms(unsigned seed, int64_t n, double *out) {
    chili::Random::Instance().Seed(seed);
    std::vector<double> v(static_cast<size_t>(n));
    chili::Random::Instance().Generate(v);
    std::memcpy(out, v.data(), sizeof(double) * v.size());
}

// The reference's own Vegas::Optimize (Vegas.cc:54-69) on the camel, with its
// global generator seeded by `seed`: iterations until the pooled error meets
// atol or rtol and at least nitn iterations ran, Refine (grid split in two,
// ncalls doubled, Vegas.cc:79-82) every nrefine iterations.  Outputs: the
// number of iterations, each iteration's StatsData (at most max_iter), the
// final bins per dimension and ncalls, the pooled StatsData and the final
// grid edges (dims * (bins_out + 1), at most max_edges values).
int ref_vegas_optimize(int dims, int bins, double alpha, const double *params, int nparams, unsigned seed,
                       int64_t ncalls, int64_t nrefine, double atol, double rtol, int64_t nitn, int max_iter,
                       chili_stats *iters, int64_t *bins_out, int64_t *ncalls_out, chili_stats *pooled,
                       double *edges_out, int64_t max_edges) {
    Quiet quiet;
    std::streambuf *saved = std::cout.rdbuf(nullptr);  // PrintIteration (Vegas.cc:63)
    chili::Random::Instance().Seed(seed);
    chili::VegasParams vp;
    vp.ncalls = static_cast<size_t>(ncalls);
    vp.nrefine = static_cast<size_t>(nrefine);
    vp.atol = atol;
    vp.rtol = rtol;
    vp.alpha = alpha;
    vp.ninterations = static_cast<size_t>(nitn);
    chili::Vegas vegas(chili::AdaptiveMap(static_cast<size_t>(dims), static_cast<size_t>(bins)), vp);
    vegas.SetVerbosity(0);
    std::vector<double> p(params, params + nparams);
    chili::Func<double> f = [p](const std::vector<double> &x) { return camel(x, p); };
    vegas.Optimize(f);
    const auto grid = vegas.Grid();
    *bins_out = static_cast<int64_t>(grid.Bins());
    // ncalls after the last Refine: the reference keeps it in its private
    // params; every Refine doubles it
    const auto summary = vegas.Summary();  // prints "Final integral" (Vegas.cc:84-90)
    std::cout.rdbuf(saved);
    const int n_it = static_cast<int>(summary.results.size());
    const int64_t nref = nrefine > 0 ? n_it / nrefine : 0;
    *ncalls_out = ncalls << nref;
    for (int i = 0; i < n_it && i < max_iter; ++i) fill_stats(summary.results[i], iters + i);
    fill_stats(summary.sum_results, pooled);
    const int64_t ne = static_cast<int64_t>(grid.Dims()) * (*bins_out + 1);
    if (ne <= max_edges) std::memcpy(edges_out, grid.Hist().data(), sizeof(double) * ne);
    return n_it;
}

void ref_mc_get_training(void *p, double *hist, double *atrain) {
    auto *h = static_cast<MC *>(p);
    if (hist) std::memcpy(hist, h->last_hist.data(), sizeof(double) * h->last_hist.size());
    if (atrain) std::memcpy(atrain, h->last_atrain.data(), sizeof(double) * h->last_atrain.size());
}

uint64_t ref_mc_dropped_dim0(void *p) { return static_cast<MC *>(p)->dropped_dim0; }

// The reference's own loop: niter calls of MultiChannel::operator() with its
// global mt19937 seeded by `seed`.  Used as the timed CPU baseline.
void ref_mc_run_native(void *p, unsigned seed, int niter, chili_stats *out) {
    auto *h = static_cast<MC *>(p);
    Quiet quiet;
    chili::Random::Instance().Seed(seed);
    chili::StatsData total;
    for (int it = 0; it < niter; ++it) {
        h->mc(h->integrand);
    }
    (void)total;
    std::ostringstream sink;
    const auto summary = h->mc.Summary(sink);
    fill_stats(summary.sum_results, out);
}

// Interface::Evaluate (nanobind.hh:23-50): uniforms through channel ch's
// FSMapper alone, out = f * w (0 on PreProcess rejection or zero weight).
void ref_evaluate_batch(void *p, int ch, const double *u, int64_t n, double *out) {
    auto *h = static_cast<MC *>(p);
    Quiet quiet;
    auto &mapping = h->integrand.GetChannel(ch).mapping;
    std::vector<double> rans(h->ndims);
    for (int64_t i = 0; i < n; ++i) {
        for (int d = 0; d < h->ndims; ++d) rans[d] = u[i * h->ndims + d];
        std::vector<FourVector> point;
        mapping->GeneratePoint(point, rans);
        if (!h->integrand.PreProcess()(point)) {
            out[i] = 0;
            continue;
        }
        const double weight = mapping->GenerateWeight(point, rans);
        double val = weight == 0 ? 0 : h->integrand(point) * weight;
        if (!h->integrand.PostProcess()(point, val)) val = 0;
        out[i] = val;
    }
}

// ------------------------------------------------------ ConstructChannels
// The reference's ConstructChannels (ChannelNode.cc:74-291) with a Model
// whose Combinable reads a rule table: rows of 11 int32 {f1, f2, n, out[8]}.
// cuts == NULL: the first overload.  Every mapper's Mapper::Serialize bytes
// are appended to buf (cap bytes; *len = bytes needed); for the second
// overload the completed ptmin and etamax tables come back as (idx, value)
// pairs (capacity max_cut entries each).  Returns the number of channels, or
// -1 when the reference throws (e.g. a flavour missing from the masses).
int ref_construct_channels(double sqrts, const int32_t *flavs, int n, const int32_t *rules, int n_rules,
                           const chili_idx_value *masses, int nm, const chili_idx_value *widths, int nw,
                           const chili_cuts *cuts, int smax, char *buf, int64_t cap, int64_t *len,
                           chili_idx_value *ptmin_out, int *n_ptmin, chili_idx_value *etamax_out, int *n_etamax,
                           int max_cut) {
    try {
        std::vector<int32_t> table(rules, rules + 11 * n_rules);
        auto comb = [table, n_rules](int f1, int f2) {
            std::vector<int> out;
            for (int r = 0; r < n_rules; ++r) {
                const int32_t *row = table.data() + 11 * r;
                if (row[0] == f1 && row[1] == f2) out.insert(out.end(), row + 3, row + 3 + row[2]);
            }
            return out;
        };
        std::unordered_map<unsigned int, double> mm, ww;
        for (int i = 0; i < nm; ++i) mm[masses[i].idx] = masses[i].value;
        for (int i = 0; i < nw; ++i) ww[widths[i].idx] = widths[i].value;
        chili::Model model(comb, mm);
        model.SetWidths(ww);
        const std::vector<int> fl(flavs, flavs + n);
        std::vector<std::unique_ptr<chili::FSMapper>> maps;
        chili::Cuts c;
        if (cuts) {
            c = to_cuts(cuts);
            maps = chili::ConstructChannels(sqrts, fl, model, c, static_cast<size_t>(smax));
        } else {
            maps = chili::ConstructChannels(sqrts, fl, model, static_cast<size_t>(smax));
        }
        std::ostringstream os;
        for (const auto &m : maps) chili::Mapper<FourVector>::Serialize(os, *m);
        const std::string bytes = os.str();
        *len = static_cast<int64_t>(bytes.size());
        if (buf && static_cast<int64_t>(bytes.size()) <= cap) std::memcpy(buf, bytes.data(), bytes.size());
        int k = 0;
        for (const auto &kv : c.ptmin)
            if (k < max_cut) ptmin_out[k++] = chili_idx_value{kv.first, kv.second};
        *n_ptmin = k;
        k = 0;
        for (const auto &kv : c.etamax)
            if (k < max_cut) etamax_out[k++] = chili_idx_value{kv.first, kv.second};
        *n_etamax = k;
        return static_cast<int>(maps.size());
    } catch (...) {
        return -1;
    }
}

}  // extern "C"
