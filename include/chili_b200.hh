// chili_b200.hh -- C++ host adapters over the C ABI (chili_gpu.h) that keep
// the shapes and method names of Chili's integration classes, so that a
// driver written against the reference switches to the B200 path by changing
// types, not code structure:
//
//   reference (paths inside the Chili project)            this header
//   chili::AdaptiveMap        Integrator/AdaptiveMap.hh   chili::gpu::AdaptiveMap
//   chili::VegasParams/Vegas  Integrator/Vegas.hh         chili::gpu::VegasParams / Vegas
//   chili::StatsData          Integrator/Statistics.hh    chili::gpu::StatsData
//   chili::ChannelDescription Channel/ChannelNode.hh      chili::gpu::ChannelDescription
//   chili::Cuts               Tools/Cuts.hh               chili::gpu::Cuts
//   chili::FSMapper           Channel/Channel.hh          chili::gpu::FSMapper (batched)
//   chili::MultiChannelParams/MultiChannel                chili::gpu::MultiChannelParams / MultiChannel
//                             Channel/MultiChannel.hh
//
// Differences forced by the device: the integrand is a built-in device
// function chosen by id (chili_integrand_kind) instead of a std::function,
// and FSMapper/AdaptiveMap evaluate batches of points.  Errors from the C ABI
// are thrown as chili::gpu::Error (the reference throws std::runtime_error).
#pragma once

#include <cmath>
#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <ostream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "chili_gpu.h"

namespace chili {
namespace gpu {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc, const chili_ctx *ctx) {
    if (rc != CHILI_OK) throw Error(rc, std::string("chili_gpu: ") + chili_gpu_last_error(ctx));
}

// StatsData (Statistics.hh:62-142): same fields, Mean/Error/Efficiency.
struct StatsData {
    double n{}, min{1.7976931348623157e308}, max{2.2250738585072014e-308}, sum{}, sum2{}, n_finite{};
    StatsData() = default;
    explicit StatsData(const chili_stats &s)
        : n(s.n), min(s.min), max(s.max), sum(s.sum), sum2(s.sum2), n_finite(s.n_finite) {}
    StatsData &operator+=(const StatsData &x) {
        n += x.n;
        n_finite += x.n_finite;
        sum += x.sum;
        sum2 += x.sum2;
        min = (x.min < min) ? x.min : min;
        max = (max < x.max) ? x.max : max;
        return *this;
    }
    double Mean() const { return sum / n; }
    double Variance() const { return (sum2 / n - Mean() * Mean()) / (n - 1); }
    double Error() const { return std::sqrt(Variance()); }
    double Efficiency() const { return n_finite / n; }
    size_t Calls() const { return static_cast<size_t>(n); }
    size_t FiniteCalls() const { return static_cast<size_t>(n_finite); }
};

// A device context (one GPU, one stream).  Owned by Vegas / MultiChannel.
class Context {
  public:
    explicit Context(int device = 0) { check(chili_gpu_create(device, &ctx_), nullptr); }
    ~Context() { chili_gpu_destroy(ctx_); }
    Context(const Context &) = delete;
    Context &operator=(const Context &) = delete;
    chili_ctx *get() const { return ctx_; }
    void SetStream(void *stream) { check(chili_gpu_set_stream(ctx_, stream), ctx_); }
    void SetOption(const char *name, int64_t v) { check(chili_gpu_set_option(ctx_, name, v), ctx_); }

  private:
    chili_ctx *ctx_ = nullptr;
};

// AdaptiveMap (AdaptiveMap.hh:26-73): the host copy of a grid in the
// reference layout hist[dim*(bins+1)+k], initialised uniform.
class AdaptiveMap {
  public:
    AdaptiveMap() = default;
    AdaptiveMap(size_t dims, size_t bins) : dims_(dims), bins_(bins), hist_(dims * (bins + 1)) {
        for (size_t d = 0; d < dims; ++d)
            for (size_t k = 0; k <= bins; ++k)
                hist_[d * (bins + 1) + k] = static_cast<double>(k) / static_cast<double>(bins);
    }
    size_t Dims() const { return dims_; }
    size_t Bins() const { return bins_; }
    const std::vector<double> &Hist() const { return hist_; }
    std::vector<double> &Hist() { return hist_; }

  private:
    size_t dims_{}, bins_{};
    std::vector<double> hist_;
};

// VegasParams (Vegas.hh:30-38) and Vegas (Vegas.hh:47-95) on the camel
// integrand (CHILI_FUNC_CAMEL).
struct VegasParams {
    size_t ncalls{10000}, nrefine{5};
    double rtol{1e-4}, atol{1e-4}, alpha{1.};
    size_t ninterations{10};
};

struct VegasSummary {
    std::vector<StatsData> results;
    StatsData sum_results;
    StatsData Result() const { return sum_results; }
};

class Vegas {
  public:
    Vegas(AdaptiveMap map, VegasParams params, std::vector<double> camel_params, int device = 0,
          uint64_t seed = 42)
        : ctx_(device), grid_(std::move(map)), params_(params), seed_(seed) {
        check(chili_gpu_set_grids(ctx_.get(), grid_.Hist().data(), 1, static_cast<int>(grid_.Dims()),
                                  static_cast<int>(grid_.Bins())),
              ctx_.get());
        check(chili_gpu_set_integrand(ctx_.get(), CHILI_FUNC_CAMEL, camel_params.data(),
                                      static_cast<int>(camel_params.size())),
              ctx_.get());
    }
    // Uniforms from the caller instead of the device generator: before each
    // iteration source(n, out) writes the next n = ncalls * dims uniforms to
    // out, point after point (the order Vegas::operator() draws them from
    // Random::Generate, Vegas.cc:32), for instance a replay of a reference
    // run's stream.  An empty function restores the device generator.
    void SetUniformSource(std::function<void(size_t, double *)> source) { source_ = std::move(source); }
    // Vegas::operator() (Vegas.cc:18-52): one iteration, then Adapt.
    void operator()() {
        chili_stats st;
        const double *u = nullptr;
        if (source_) {
            uniforms_.resize(params_.ncalls * grid_.Dims());
            source_(uniforms_.size(), uniforms_.data());
            u = uniforms_.data();
        }
        check(chili_gpu_vegas_iterate(ctx_.get(), params_.ncalls, seed_, counter_, u, params_.alpha, 1, &st,
                                      nullptr),
              ctx_.get());
        counter_ += params_.ncalls;
        summary_.results.emplace_back(st);
        summary_.sum_results += summary_.results.back();
    }
    // Vegas::Optimize (Vegas.cc:54-69).
    void Optimize() {
        double abs_err = 1.7976931348623157e308, rel_err = abs_err;
        size_t irefine = 0;
        while ((abs_err > params_.atol && rel_err > params_.rtol) || summary_.results.size() < params_.ninterations) {
            (*this)();
            const StatsData cur = summary_.Result();
            abs_err = cur.Error();
            rel_err = abs_err / std::abs(cur.Mean());
            if (++irefine == params_.nrefine) {
                Refine();
                irefine = 0;
            }
        }
    }
    // Vegas::Refine (Vegas.cc:79-82): the device grid split in two
    // (AdaptiveMap::Split), ncalls doubled.  The host copy only takes the
    // new shape here; Grid() fills it from the device.
    void Refine() {
        check(chili_gpu_grid_split(ctx_.get(), 2), ctx_.get());
        params_.ncalls *= 2;
        grid_ = AdaptiveMap(grid_.Dims(), grid_.Bins() * 2);
    }
    const VegasParams &Params() const { return params_; }
    // Vegas::Grid (Vegas.hh:67-68): the device grid copied back.
    const AdaptiveMap &Grid() {
        check(chili_gpu_get_grids(ctx_.get(), grid_.Hist().data(), 1, static_cast<int>(grid_.Dims()),
                                  static_cast<int>(grid_.Bins())),
              ctx_.get());
        return grid_;
    }
    // Vegas::GenerateWeight (Vegas.cc:71-73), batched: x[n*dims] -> w[n].
    std::vector<double> GenerateWeight(const std::vector<double> &x) {
        const int64_t n = static_cast<int64_t>(x.size() / grid_.Dims());
        std::vector<double> w(static_cast<size_t>(n));
        check(chili_gpu_grid_weight(ctx_.get(), 0, x.data(), w.data(), nullptr, n), ctx_.get());
        return w;
    }
    VegasSummary Summary() const { return summary_; }

  private:
    Context ctx_;
    AdaptiveMap grid_;
    VegasParams params_;
    uint64_t seed_, counter_ = 0;
    VegasSummary summary_;
    std::function<void(size_t, double *)> source_;
    std::vector<double> uniforms_;
};

// ParticleInfo / ChannelDescription (ChannelNode.hh:26-51) and Cuts
// (Cuts.hh:13-19) in host form; converted to the C ABI's flat tables.
struct ParticleInfo {
    unsigned idx{};
    int pid{};
    double mass{}, width{};
};
struct ChannelDescription {
    std::vector<ParticleInfo> info;
    std::vector<std::pair<ParticleInfo, std::pair<ParticleInfo, ParticleInfo>>> decays;
};
struct Cuts {
    std::vector<double> sexternal;
    std::map<std::pair<int, int>, double> deltaR;
    std::map<unsigned, double> smin, ptmin, etamax;
};

// The flat C-ABI form of a channel set; keeps the arrays alive.
class ChannelSet {
  public:
    ChannelSet(const std::vector<ChannelDescription> &channels, const Cuts &cuts, double sqrts, int n_ext)
        : sqrts_(sqrts), n_ext_(n_ext) {
        infos_.resize(channels.size());
        decays_.resize(channels.size());
        for (size_t c = 0; c < channels.size(); ++c) {
            for (const auto &p : channels[c].info) infos_[c].push_back(conv(p));
            for (const auto &d : channels[c].decays)
                decays_[c].push_back(chili_decay{conv(d.first), conv(d.second.first), conv(d.second.second)});
        }
        for (size_t c = 0; c < channels.size(); ++c)
            descs_.push_back(chili_channel_desc{static_cast<int32_t>(infos_[c].size()), infos_[c].data(),
                                                static_cast<int32_t>(decays_[c].size()), decays_[c].data()});
        sext_ = cuts.sexternal;
        for (const auto &kv : cuts.deltaR) dr_.push_back({kv.first.first, kv.first.second, kv.second});
        for (const auto &kv : cuts.smin) smin_.push_back({kv.first, kv.second});
        for (const auto &kv : cuts.ptmin) ptmin_.push_back({kv.first, kv.second});
        for (const auto &kv : cuts.etamax) etamax_.push_back({kv.first, kv.second});
        cuts_ = chili_cuts{static_cast<int32_t>(sext_.size()), sext_.data(), static_cast<int32_t>(dr_.size()),
                           dr_.data(), static_cast<int32_t>(smin_.size()), smin_.data(),
                           static_cast<int32_t>(ptmin_.size()), ptmin_.data(), static_cast<int32_t>(etamax_.size()),
                           etamax_.data()};
    }
    const chili_channel_desc *descs() const { return descs_.data(); }
    int nch() const { return static_cast<int>(descs_.size()); }
    const chili_cuts *cuts() const { return &cuts_; }
    double sqrts() const { return sqrts_; }
    int n_ext() const { return n_ext_; }
    // NDims (Channel.hh:33)
    size_t NDims() const { return static_cast<size_t>(3 * (n_ext_ - 2) - 2); }
    // Host-only consistency check; empty when the set is usable.
    std::string Check() const {
        char buf[512];
        chili_gpu_check_channels(descs(), nch(), cuts(), sqrts_, n_ext_, buf, sizeof(buf));
        return buf;
    }

  private:
    static chili_particle_info conv(const ParticleInfo &p) { return chili_particle_info{p.idx, p.pid, p.mass, p.width}; }
    double sqrts_;
    int n_ext_;
    std::vector<std::vector<chili_particle_info>> infos_;
    std::vector<std::vector<chili_decay>> decays_;
    std::vector<chili_channel_desc> descs_;
    std::vector<double> sext_;
    std::vector<chili_pid_pair_value> dr_;
    std::vector<chili_idx_value> smin_, ptmin_, etamax_;
    chili_cuts cuts_{};
};

// Model (Model.hh:10-29): which flavours two currents combine into, and the
// masses and widths by |pid|.
class Model {
  public:
    Model(std::function<std::vector<int>(int, int)> func, std::unordered_map<unsigned, double> masses = {})
        : combinable_(std::move(func)), masses_(std::move(masses)) {}
    double &Mass(int flav) { return masses_[static_cast<unsigned>(std::abs(flav))]; }
    double &Width(int flav) { return widths_[static_cast<unsigned>(std::abs(flav))]; }
    void SetMasses(std::unordered_map<unsigned, double> m) { masses_ = std::move(m); }
    void SetWidths(std::unordered_map<unsigned, double> w) { widths_ = std::move(w); }
    std::vector<int> Combinable(int f1, int f2) const { return combinable_(f1, f2); }
    const std::unordered_map<unsigned, double> &Masses() const { return masses_; }
    const std::unordered_map<unsigned, double> &Widths() const { return widths_; }

  private:
    std::function<std::vector<int>(int, int)> combinable_;
    std::unordered_map<unsigned, double> masses_, widths_;
};

namespace detail {
inline int combinable_trampoline(int32_t f1, int32_t f2, int32_t *out, int32_t max_out, void *user) {
    try {
        const auto v = static_cast<const Model *>(user)->Combinable(f1, f2);
        if (static_cast<int32_t>(v.size()) > max_out) return -1;
        for (size_t i = 0; i < v.size(); ++i) out[i] = v[i];
        return static_cast<int>(v.size());
    } catch (...) {
        return -1;
    }
}

inline ParticleInfo from_c(const chili_particle_info &p) { return ParticleInfo{p.idx, p.pid, p.mass, p.width}; }

// The library's ConstructChannels; cuts == nullptr for the default cuts.
inline std::pair<std::vector<ChannelDescription>, Cuts> construct(double sqrts, const std::vector<int> &flavs,
                                                                  const Model &model, const Cuts *cuts,
                                                                  size_t smax) {
    std::vector<chili_idx_value> mt, wt;
    for (const auto &kv : model.Masses()) mt.push_back({kv.first, kv.second});
    for (const auto &kv : model.Widths()) wt.push_back({kv.first, kv.second});
    chili_model m{&combinable_trampoline, const_cast<Model *>(&model), static_cast<int32_t>(mt.size()), mt.data(),
                  static_cast<int32_t>(wt.size()), wt.data()};
    std::vector<int32_t> fl(flavs.begin(), flavs.end());
    std::unique_ptr<ChannelSet> cin;
    if (cuts) cin = std::make_unique<ChannelSet>(std::vector<ChannelDescription>{}, *cuts, sqrts, static_cast<int>(flavs.size()));
    chili_channel_list *list = nullptr;
    char err[512];
    const int rc = chili_construct_channels(sqrts, fl.data(), static_cast<int>(fl.size()), &m,
                                            cin ? cin->cuts() : nullptr, static_cast<int>(smax), &list, err,
                                            sizeof(err));
    if (rc != CHILI_OK) throw Error(rc, err);
    const chili_channel_desc *d = nullptr;
    const chili_cuts *c = nullptr;
    int n = 0;
    chili_channel_list_get(list, &d, &n, &c);
    std::vector<ChannelDescription> out(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) {
        for (int k = 0; k < d[i].n_info; ++k) out[i].info.push_back(from_c(d[i].info[k]));
        for (int k = 0; k < d[i].n_decays; ++k)
            out[i].decays.push_back({from_c(d[i].decays[k].parent),
                                     {from_c(d[i].decays[k].child1), from_c(d[i].decays[k].child2)}});
    }
    Cuts oc;
    oc.sexternal.assign(c->sexternal, c->sexternal + c->n_sexternal);
    for (int k = 0; k < c->n_deltaR; ++k) oc.deltaR[{c->deltaR[k].pid1, c->deltaR[k].pid2}] = c->deltaR[k].value;
    for (int k = 0; k < c->n_smin; ++k) oc.smin[c->smin[k].idx] = c->smin[k].value;
    for (int k = 0; k < c->n_ptmin; ++k) oc.ptmin[c->ptmin[k].idx] = c->ptmin[k].value;
    for (int k = 0; k < c->n_etamax; ++k) oc.etamax[c->etamax[k].idx] = c->etamax[k].value;
    chili_channel_list_free(list);
    return {std::move(out), std::move(oc)};
}
}  // namespace detail

// ConstructChannels (ChannelNode.cc:74-291): the channel set of a process
// (flavours: the two incoming, then the outgoing) with the default cuts
// (Delta R 0.4, pT > 30, |eta| < 99).  Where the reference returns one
// FSMapper per channel, this returns the set a MultiChannel is built on.
inline ChannelSet ConstructChannels(double sqrts, const std::vector<int> &flavs, const Model &model,
                                    size_t smax = 2) {
    auto r = detail::construct(sqrts, flavs, model, nullptr, smax);
    return ChannelSet(r.first, r.second, sqrts, static_cast<int>(flavs.size()));
}
// With given cuts, completed in place with the currents' pT and eta entries
// (ChannelNode.cc:161-162), as the reference's second overload does.
inline ChannelSet ConstructChannels(double sqrts, const std::vector<int> &flavs, const Model &model, Cuts &cuts,
                                    size_t smax = 2) {
    auto r = detail::construct(sqrts, flavs, model, &cuts, smax);
    cuts = r.second;
    return ChannelSet(r.first, r.second, sqrts, static_cast<int>(flavs.size()));
}

// MultiChannelParams (MultiChannel.hh:29-49).
struct MultiChannelParams {
    size_t ncalls{10000}, niterations{10};
    double rtol{1e-5};
    size_t nrefine{1};
    double beta{0.25}, min_alpha{1e-5}, refine_size{1.5};
    size_t max_bins{200}, iteration{};
    bool should_optimize{true};
    double grid_alpha{1.};  // VegasParams::alpha of the channel grids
};

struct MultiChannelSummary {
    std::vector<StatsData> results;
    std::vector<double> best_weights;
    StatsData sum_results;
    StatsData Result() const { return sum_results; }
};

// MultiChannel (MultiChannel.hh:51-139) over a ChannelSet with one VEGAS grid
// of `bins` bins per channel (Integrand::AddChannel, Integrand.hh:67-72).
class MultiChannel {
  public:
    MultiChannel(const ChannelSet &channels, size_t bins, MultiChannelParams params, int integrand_kind,
                 std::vector<double> integrand_params, int device = 0, uint64_t seed = 7,
                 bool guard_alpha = true)
        : ctx_(device), params_(params), bins_(bins), seed_(seed), guard_(guard_alpha) {
        chili_ctx *c = ctx_.get();
        check(chili_gpu_set_channels(c, channels.descs(), channels.nch(), channels.cuts(), channels.sqrts(),
                                     channels.n_ext()),
              c);
        ndims_ = static_cast<size_t>(chili_gpu_ndims(c));
        nch_ = static_cast<size_t>(channels.nch());
        std::vector<double> edges;
        for (size_t ch = 0; ch < nch_; ++ch) {
            const AdaptiveMap m(ndims_, bins);
            edges.insert(edges.end(), m.Hist().begin(), m.Hist().end());
        }
        check(chili_gpu_set_grids(c, edges.data(), static_cast<int>(nch_), static_cast<int>(ndims_),
                                  static_cast<int>(bins)),
              c);
        check(chili_gpu_set_integrand(c, integrand_kind, integrand_params.data(),
                                      static_cast<int>(integrand_params.size())),
              c);
        check(chili_gpu_set_preprocess(c, CHILI_PRE_FINITE), c);
    }
    size_t Dimensions() const { return ndims_; }
    size_t NChannels() const { return nch_; }
    MultiChannelParams &Parameters() { return params_; }

    // MultiChannel::operator() (MultiChannel.hh:196-251).
    void operator()() {
        chili_multichannel_params p = to_c(params_);
        chili_stats st;
        chili_mc_iter_info info;
        check(chili_gpu_multichannel_iterate(ctx_.get(), &p, seed_, counter_, nullptr, 0, guard_ ? 1 : 0, &st,
                                             &info),
              ctx_.get());
        counter_ += info.points_tried;
        last_ = info;
        summary_.results.emplace_back(st);  // UpdateResults (MultiChannel.cc:69-77)
        summary_.sum_results += summary_.results.back();
    }
    // MultiChannel::Optimize (MultiChannel.hh:253-268), RefineChannels (:121-130).
    void Optimize(std::ostream *os = nullptr) {
        double rel_err = 1.7976931348623157e308;
        while (rel_err > params_.rtol && summary_.results.size() < params_.niterations) {
            (*this)();
            const StatsData cur = summary_.sum_results;
            rel_err = cur.Error() / std::abs(cur.Mean());
            if (os)
                *os << "XS: " << summary_.results.size() << "   " << cur.Mean() << " +/- " << cur.Error() << "\n";
            if (++params_.iteration == params_.nrefine) RefineChannels();
        }
    }
    // MultiChannel::Summary (MultiChannel.cc:156-168).
    MultiChannelSummary Summary(std::ostream &os) {
        std::vector<double> a(nch_), best(nch_);
        double md;
        check(chili_gpu_get_alpha(ctx_.get(), a.data(), best.data(), &md, static_cast<int>(nch_)), ctx_.get());
        summary_.best_weights = best;
        const StatsData r = summary_.Result();
        os << "Final integral = " << r.Mean() << " +/- " << r.Error() << " (" << r.Error() / r.Mean() * 100
           << " %)\nCut Efficiency: " << r.Efficiency() << "\nChannel weights:\n";
        for (size_t i = 0; i < nch_; ++i) os << "  alpha(" << i << ") = " << best[i] << "\n";
        return summary_;
    }
    std::vector<double> ChannelWeights() {
        std::vector<double> a(nch_);
        check(chili_gpu_get_alpha(ctx_.get(), a.data(), nullptr, nullptr, static_cast<int>(nch_)), ctx_.get());
        return a;
    }
    const chili_mc_iter_info &LastIteration() const { return last_; }
    chili_ctx *context() { return ctx_.get(); }

  private:
    void RefineChannels() {
        params_.iteration = 0;
        params_.ncalls = static_cast<size_t>(static_cast<double>(params_.ncalls) * params_.refine_size);
        if (bins_ < params_.max_bins) {
            check(chili_gpu_grid_split(ctx_.get(), 2), ctx_.get());
            bins_ *= 2;
        }
    }
    static chili_multichannel_params to_c(const MultiChannelParams &p) {
        return chili_multichannel_params{p.ncalls, p.niterations, p.rtol, p.nrefine, p.beta, p.min_alpha,
                                         p.refine_size, p.max_bins, p.iteration, p.should_optimize ? 1 : 0,
                                         p.grid_alpha};
    }
    Context ctx_;
    MultiChannelParams params_;
    size_t bins_, ndims_{}, nch_{};
    uint64_t seed_, counter_ = 0;
    bool guard_;
    chili_mc_iter_info last_{};
    MultiChannelSummary summary_;
};

// FSMapper (Channel.hh:15-77), batched over one channel of a context.
class FSMapper {
  public:
    FSMapper(chili_ctx *ctx, int channel, size_t ndims, int n_ext)
        : ctx_(ctx), ch_(channel), ndims_(ndims), n_ext_(n_ext) {}
    size_t NDims() const { return ndims_; }
    // GeneratePoint (Channel.cc:22-38): x[n*ndims] -> mom[n*n_ext*4]
    std::vector<double> GeneratePoint(const std::vector<double> &x) const {
        const int64_t n = static_cast<int64_t>(x.size() / ndims_);
        std::vector<double> mom(static_cast<size_t>(n) * n_ext_ * 4);
        check(chili_gpu_fsmapper_generate(ctx_, ch_, x.data(), mom.data(), n), ctx_);
        return mom;
    }
    // GenerateWeight (Channel.cc:40-61): mom -> weights, x_out[n*ndims]
    std::vector<double> GenerateWeight(const std::vector<double> &mom, std::vector<double> &x_out) const {
        const int64_t n = static_cast<int64_t>(mom.size() / (n_ext_ * 4));
        std::vector<double> w(static_cast<size_t>(n));
        x_out.resize(static_cast<size_t>(n) * ndims_);
        check(chili_gpu_fsmapper_weight(ctx_, ch_, mom.data(), x_out.data(), w.data(), n), ctx_);
        return w;
    }

  private:
    chili_ctx *ctx_;
    int ch_;
    size_t ndims_;
    int n_ext_;
};

}  // namespace gpu
}  // namespace chili
