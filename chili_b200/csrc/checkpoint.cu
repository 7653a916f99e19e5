// checkpoint.cu -- the reference's results.chili format, read and written
// by the library so that a grid trained on the CPU resumes on the GPU and
// vice versa. Layout (little-endian, size_t = 8 bytes), restated from the
// reference's Serialize methods:
//   Integrand::Serialize (Integrand.hh:48-55): size_t nch, then per channel
//     AdaptiveMap::Serialize (AdaptiveMap.cc:23-32): size_t bins, size_t dims,
//       double edges[(bins+1)*dims]
//     Mapper::Serialize (Mapper.hh:49-56): size_t len, char name[len] ("FSMapper"),
//     FSMapper::_Serialize (Channel.cc:7-20): ChannelDescription::Serialize
//       (ChannelNode.cc:33-47: size_t n_info, ParticleInfo info[n_info],
//       size_t n_decays, (parent, child1, child2) ParticleInfo each, std::map
//       order), double sqrts, double ptmax, size_t ntot, size_t nout,
//       size_t n_ptmin, double ptmin[n_ptmin]
//     ParticleInfo::Serialize (ChannelNode.cc:19-25): uint32 idx, int32 pid,
//       double mass, double width
//   MultiChannel::Serialize (MultiChannel.cc:95-106): size_t ndims,
//     MultiChannelParams::Serialize (MultiChannel.cc:49-59: size_t ncalls,
//     size_t niterations, double rtol, size_t nrefine, double beta,
//     double min_alpha, double refine_size, size_t max_bins), size_t n,
//     double best_weights[n], double min_diff, MultiChannelSummary::Serialize
//     (MultiChannel.cc:21-34: size_t n_results, StatsData results[] as
//     6 doubles n, min, max, sum, sum2, n_finite (Statistics.hh:80-87),
//     size_t n, double best_weights[n]).
// Loading sets channel weights = best weights, as the reference does
// (MultiChannel.cc:85).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "context.h"

namespace {

struct Writer {
    std::ofstream out;
    template <class T> void put(const T &v) { out.write(reinterpret_cast<const char *>(&v), sizeof(T)); }
    void put_size(size_t v) { put<uint64_t>(static_cast<uint64_t>(v)); }
    void particle(const chili_particle_info &p) {
        put<uint32_t>(p.idx);
        put<int32_t>(p.pid);
        put<double>(p.mass);
        put<double>(p.width);
    }
};

struct Reader {
    std::ifstream in;
    bool ok = true;
    template <class T> T get() {
        T v{};
        if (!in.read(reinterpret_cast<char *>(&v), sizeof(T))) ok = false;
        return v;
    }
    size_t get_size(size_t limit) {
        const uint64_t v = get<uint64_t>();
        if (v > limit) ok = false;
        return ok ? static_cast<size_t>(v) : 0;
    }
    chili_particle_info particle() {
        chili_particle_info p;
        p.idx = get<uint32_t>();
        p.pid = get<int32_t>();
        p.mass = get<double>();
        p.width = get<double>();
        return p;
    }
};

// std::map<ParticleInfo, ...> order (ChannelNode.cc:293-301)
bool info_less(const chili_particle_info &a, const chili_particle_info &b) {
    if (a.idx == b.idx) {
        if (a.mass == b.mass) return a.width < b.width;
        return a.mass < b.mass;
    }
    return a.idx < b.idx;
}

bool same_particle(const chili_particle_info &a, const chili_particle_info &b) {
    return a.idx == b.idx && a.pid == b.pid && a.mass == b.mass && a.width == b.width;
}

}  // namespace

extern "C" {

int chili_gpu_save_checkpoint(chili_ctx *ctx, const char *path, const chili_multichannel_params *params,
                              const chili_stats *results, int64_t nresults) {
    if (!ctx || !path || !params || (nresults > 0 && !results) || nresults < 0)
        return fail(ctx, CHILI_ERR_INVALID_ARG, "NULL argument or nresults < 0");
    if (int rc = set_device(ctx)) return rc;
    if (int rc = need_channels(ctx)) return rc;
    if (int rc = need_grids(ctx)) return rc;
    if (ctx->g_nch != ctx->nch || ctx->dims != ctx->ndims)
        return fail(ctx, CHILI_ERR_STATE, "grids do not match the channel set");
    const int nch = ctx->nch, D = ctx->dims, B = ctx->bins;
    const size_t per = static_cast<size_t>(D) * (B + 1);
    std::vector<double> edges(per * nch), best(nch), md(1);
    CK(cudaMemcpyAsync(edges.data(), ctx->edges.p, sizeof(double) * edges.size(), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(best.data(), best_ptr(ctx), sizeof(double) * nch, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(md.data(), mindiff_ptr(ctx), sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    Writer w;
    w.out.open(path, std::ios::binary | std::ios::trunc);
    if (!w.out) return fail(ctx, CHILI_ERR_INVALID_ARG, std::string("cannot open ") + path);
    w.put_size(nch);
    const std::string name = "FSMapper";
    for (int c = 0; c < nch; ++c) {
        w.put_size(B);
        w.put_size(D);
        for (size_t q = 0; q < per; ++q) w.put<double>(edges[c * per + q]);
        w.put_size(name.size());
        w.out.write(name.data(), static_cast<std::streamsize>(name.size()));
        w.put_size(ctx->ch_info[c].size());
        for (const auto &p : ctx->ch_info[c]) w.particle(p);
        std::vector<chili_decay> dec = ctx->ch_decays[c];
        std::stable_sort(dec.begin(), dec.end(),
                         [](const chili_decay &a, const chili_decay &b) { return info_less(a.parent, b.parent); });
        w.put_size(dec.size());
        for (const auto &d : dec) {
            w.particle(d.parent);
            w.particle(d.child1);
            w.particle(d.child2);
        }
        w.put<double>(ctx->sqrts);
        w.put<double>(ctx->sqrts / 2.0);
        w.put_size(ctx->n_ext);
        w.put_size(ctx->n_ext - 2);
        w.put_size(ctx->ch_ptmin[c].size());
        for (double v : ctx->ch_ptmin[c]) w.put<double>(v);
    }
    w.put_size(D);
    w.put_size(params->ncalls);
    w.put_size(params->niterations);
    w.put<double>(params->rtol);
    w.put_size(params->nrefine);
    w.put<double>(params->beta);
    w.put<double>(params->min_alpha);
    w.put<double>(params->refine_size);
    w.put_size(params->max_bins);
    // best weights: empty until the first MaxDifference update (NaN here)
    const bool have_best = !std::isnan(best[0]);
    w.put_size(have_best ? nch : 0);
    if (have_best)
        for (double v : best) w.put<double>(v);
    w.put<double>(md[0]);
    w.put_size(static_cast<size_t>(nresults));
    for (int64_t k = 0; k < nresults; ++k) {
        w.put<double>(results[k].n);
        w.put<double>(results[k].min);
        w.put<double>(results[k].max);
        w.put<double>(results[k].sum);
        w.put<double>(results[k].sum2);
        w.put<double>(results[k].n_finite);
    }
    w.put_size(ctx->summary_best.size());
    for (double v : ctx->summary_best) w.put<double>(v);
    w.out.flush();
    if (!w.out) return fail(ctx, CHILI_ERR_INVALID_ARG, std::string("write failed: ") + path);
    return CHILI_OK;
}

int chili_gpu_load_checkpoint(chili_ctx *ctx, const char *path, chili_multichannel_params *params,
                              chili_stats *results, int64_t max_results, int64_t *nresults) {
    if (!ctx || !path) return fail(ctx, CHILI_ERR_INVALID_ARG, "NULL argument");
    if (int rc = set_device(ctx)) return rc;
    if (int rc = need_channels(ctx)) return rc;
    Reader r;
    r.in.open(path, std::ios::binary);
    if (!r.in) return fail(ctx, CHILI_ERR_INVALID_ARG, std::string("cannot open ") + path);
    const int nch = ctx->nch;
    if (r.get_size(CHILI_MAX_CHANNELS) != static_cast<size_t>(nch) || !r.ok)
        return fail(ctx, CHILI_ERR_INVALID_ARG, "checkpoint: channel count differs from the channel set");
    std::vector<double> edges;
    int bins = 0, dims = 0;
    for (int c = 0; c < nch; ++c) {
        const size_t B = r.get_size(CHILI_MAX_BINS), D = r.get_size(CHILI_MAX_DIMS);
        if (!r.ok || B < 2 || static_cast<int>(D) != ctx->ndims || (c > 0 && static_cast<int>(B) != bins))
            return fail(ctx, CHILI_ERR_INVALID_ARG, "checkpoint: grid sizes do not match the channel set");
        bins = static_cast<int>(B);
        dims = static_cast<int>(D);
        for (size_t q = 0; q < (B + 1) * D; ++q) edges.push_back(r.get<double>());
        const size_t len = r.get_size(256);
        std::string name(len, '\0');
        if (len) r.in.read(&name[0], static_cast<std::streamsize>(len));
        if (!r.ok || name != "FSMapper") return fail(ctx, CHILI_ERR_INVALID_ARG, "checkpoint: mapper is not FSMapper");
        const size_t ni = r.get_size(CHILI_MAX_EXT);
        bool same = ni == ctx->ch_info[c].size();
        for (size_t i = 0; i < ni; ++i) {
            const chili_particle_info p = r.particle();
            same = same && same_particle(p, ctx->ch_info[c][i]);
        }
        std::vector<chili_decay> dec = ctx->ch_decays[c];
        std::stable_sort(dec.begin(), dec.end(),
                         [](const chili_decay &a, const chili_decay &b) { return info_less(a.parent, b.parent); });
        const size_t nd = r.get_size(CHILI_MAX_EXT);
        same = same && nd == dec.size();
        for (size_t i = 0; i < nd; ++i) {
            const chili_particle_info p = r.particle(), c1 = r.particle(), c2 = r.particle();
            same = same && i < dec.size() && same_particle(p, dec[i].parent) && same_particle(c1, dec[i].child1) &&
                   same_particle(c2, dec[i].child2);
        }
        const double sq = r.get<double>();
        r.get<double>();  // ptmax
        const size_t ntot = r.get_size(CHILI_MAX_EXT), nout = r.get_size(CHILI_MAX_EXT);
        const size_t np = r.get_size(CHILI_MAX_EXT);
        for (size_t i = 0; i < np; ++i) r.get<double>();
        same = same && sq == ctx->sqrts && ntot == static_cast<size_t>(ctx->n_ext) && nout + 2 == ntot;
        if (!r.ok) return fail(ctx, CHILI_ERR_INVALID_ARG, "checkpoint: truncated channel section");
        if (!same)
            return fail(ctx, CHILI_ERR_INVALID_ARG,
                        "checkpoint: channel " + std::to_string(c) + " differs from the channel set");
    }
    if (static_cast<int>(r.get_size(CHILI_MAX_DIMS)) != dims || !r.ok)
        return fail(ctx, CHILI_ERR_INVALID_ARG, "checkpoint: dimension mismatch");
    chili_multichannel_params p{};
    p.ncalls = r.get<uint64_t>();
    p.niterations = r.get<uint64_t>();
    p.rtol = r.get<double>();
    p.nrefine = r.get<uint64_t>();
    p.beta = r.get<double>();
    p.min_alpha = r.get<double>();
    p.refine_size = r.get<double>();
    p.max_bins = r.get<uint64_t>();
    p.should_optimize = 1;
    p.grid_alpha = params ? params->grid_alpha : 1.0;
    const size_t nb = r.get_size(CHILI_MAX_CHANNELS);
    std::vector<double> best(nb);
    for (auto &v : best) v = r.get<double>();
    const double md = r.get<double>();
    const size_t nr = r.get_size(1ull << 32);
    std::vector<chili_stats> res(nr);
    for (auto &s : res) {
        s.n = r.get<double>();
        s.min = r.get<double>();
        s.max = r.get<double>();
        s.sum = r.get<double>();
        s.sum2 = r.get<double>();
        s.n_finite = r.get<double>();
    }
    const size_t ns = r.get_size(CHILI_MAX_CHANNELS);
    std::vector<double> sbest(ns);
    for (auto &v : sbest) v = r.get<double>();
    if (!r.ok) return fail(ctx, CHILI_ERR_INVALID_ARG, "checkpoint: truncated");
    if (nb != 0 && nb != static_cast<size_t>(nch))
        return fail(ctx, CHILI_ERR_INVALID_ARG, "checkpoint: best weights do not match the channel count");
    // grids, then channel weights = best weights (MultiChannel.cc:85), min_diff
    if (int rc = chili_gpu_set_grids(ctx, edges.data(), nch, dims, bins)) return rc;
    if (nb == static_cast<size_t>(nch)) {
        if (int rc = chili_gpu_set_alpha(ctx, best.data(), nch)) return rc;
        CK(cudaMemcpyAsync(best_ptr(ctx), best.data(), sizeof(double) * nch, cudaMemcpyHostToDevice, ctx->stream));
    }
    CK(cudaMemcpyAsync(mindiff_ptr(ctx), &md, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->summary_best = sbest;
    if (params) {
        p.iteration = params->iteration;
        *params = p;
    }
    if (nresults) *nresults = static_cast<int64_t>(nr);
    if (results)
        for (size_t k = 0; k < nr && static_cast<int64_t>(k) < max_results; ++k) results[k] = res[k];
    return CHILI_OK;
}

}  // extern "C"
