// mapper_driver.cc -- TEST INFRASTRUCTURE ONLY (built by oracle/Makefile into
// oracle/_ref/mapper_driver, run by tests/test_gpu_mapper.py).
//
// Puts chili::gpu::GpuFSMapper (include/chili_b200_mapper.hh) where the
// reference's own code expects a Mapper<FourVector>: in Channel<FourVector>
// objects of a reference Integrand driven by the reference's MultiChannel
// (MultiChannel.hh:141-251, compiled here from the unmodified headers and
// linked against the unmodified sources in libchili_ref.so), beside the same
// channels with the stock FSMapper.
//
//   mapper_driver <points> <ncalls> <iterations>
//
// Output lines:
//   MAP ch npts gen_max gen_p99 wgt_max wgt_p99 rans_max nan_mismatch
//       differences GPU vs FSMapper per channel: GeneratePoint momenta
//       (relative to each leg's energy), GenerateWeight weights (relative)
//       and its in/out uniform buffers (relative)
//   ITER k n mean_stock mean_gpu var_stock var_gpu
//       one MultiChannel::operator() each (same seed, no adaptation)
//   SAVE ok            the GPU mappers' MultiChannel::SaveAs loads back
//                      into stock FSMappers (LoadFrom)
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <memory>
#include <random>
#include <sstream>
#include <vector>

#include "Channel/Channel.hh"
#include "Channel/Integrand.hh"
#include "Channel/MultiChannel.hh"
#include "Integrator/Random.hh"
#include "chili_b200_mapper.hh"

using chili::ChannelDescription;
using chili::FourVector;
using chili::ParticleInfo;

namespace {

// The 2->4 channels of the example: six Z -> pair channels and three pure
// multi-peripheral chains, at sqrt(S) = 1 TeV with ConstructChannels' default
// cuts (ChannelNode.cc:69-95).
std::vector<ChannelDescription> channels(chili::Cuts &cuts) {
    const int flavs[6] = {1, -1, 11, -11, 13, -13};
    for (int f1 : flavs)
        for (int f2 : flavs) cuts.deltaR[{f1, f2}] = 0.4;
    for (int i = 0; i < 6; ++i) {
        cuts.smin[1u << i] = 0;
        cuts.ptmin[1u << i] = 30;
        cuts.etamax[1u << i] = 99;
        if (i > 1) cuts.sexternal.push_back(0);
    }
    auto leg = [&](int i) {
        ParticleInfo p;
        p.idx = 1u << i;
        p.pid = flavs[i];
        return p;
    };
    std::vector<ChannelDescription> out;
    for (int a = 2; a < 6; ++a)
        for (int b = a + 1; b < 6; ++b) {
            ParticleInfo z;
            z.idx = (1u << a) | (1u << b);
            z.pid = 23;
            z.mass = 91.1876;
            z.width = 2.4952;
            cuts.ptmin[z.idx] = 0;
            cuts.etamax[z.idx] = 99;
            ChannelDescription d;
            std::vector<ParticleInfo> t{z};
            for (int k = 2; k < 6; ++k)
                if (k != a && k != b) t.push_back(leg(k));
            std::sort(t.begin(), t.end(), [](const ParticleInfo &x, const ParticleInfo &y) { return x.idx > y.idx; });
            d.info = t;
            d.decays[z] = {leg(a), leg(b)};
            out.push_back(d);
        }
    for (int last = 2; last < 5; ++last) {
        ChannelDescription d;
        for (int k = 5; k >= 2; --k)
            if (k != last) d.info.push_back(leg(k));
        d.info.push_back(leg(last));
        out.push_back(d);
    }
    return out;
}

double rel(double a, double b) {
    if (a == b || (std::isnan(a) && std::isnan(b))) return 0;
    return std::abs(a - b) / std::max(std::abs(b), 1e-300);
}

double p99(std::vector<double> v) {
    if (v.empty()) return 0;
    std::sort(v.begin(), v.end());
    return v[static_cast<size_t>(0.99 * static_cast<double>(v.size() - 1))];
}

// The 2->4 propagator integrand (the same user function as the tests'):
// sum over outgoing pairs of a Z Breit-Wigner times t-channel factors.
double propagator(const std::vector<FourVector> &mom) {
    const double m2 = 91.1876 * 91.1876, mw2 = m2 * 2.4952 * 2.4952, mt2 = 100.0;
    double sum = 0;
    for (size_t i = 2; i < mom.size(); ++i)
        for (size_t j = i + 1; j < mom.size(); ++j) {
            const double d = (mom[i] + mom[j]).Mass2() - m2;
            sum += 1.0 / (d * d + mw2);
        }
    double t = 1;
    for (size_t j = 2; j < mom.size(); ++j) t *= 1.0 / (std::abs((mom[0] + mom[j]).Mass2()) + mt2);
    return sum * t;
}

template <class M>
chili::Integrand<FourVector> integrand(const std::vector<ChannelDescription> &descs, const chili::Cuts &cuts,
                                       size_t bins) {
    chili::Integrand<FourVector> f;
    for (const auto &d : descs) {
        chili::Channel<FourVector> ch;
        ch.mapping = std::make_unique<M>(1000.0, 6, d, cuts);
        ch.integrator = chili::Vegas(chili::AdaptiveMap(ch.mapping->NDims(), bins), chili::VegasParams{});
        f.AddChannel(std::move(ch));
    }
    f.Function() = propagator;
    f.PreProcess() = [](const std::vector<FourVector> &m) { return !std::isnan(m[0][0]); };
    f.PostProcess() = [](const std::vector<FourVector> &, double) { return true; };
    return f;
}

}  // namespace

int main(int argc, char **argv) {
    const int npts = argc > 1 ? std::atoi(argv[1]) : 200;
    const size_t ncalls = argc > 2 ? std::strtoul(argv[2], nullptr, 10) : 200;
    const int iters = argc > 3 ? std::atoi(argv[3]) : 2;
    spdlog::set_level(spdlog::level::off);
    std::cerr.rdbuf(nullptr);  // the reference's NaN retries print to std::cerr
    chili::Cuts cuts;
    const auto descs = channels(cuts);
    try {
        // 1. the mapper alone, channel by channel
        std::mt19937_64 gen(2026);
        std::uniform_real_distribution<double> U(0.0, 1.0);
        for (size_t c = 0; c < descs.size(); ++c) {
            chili::FSMapper stock(1000.0, 6, descs[c], cuts);
            chili::gpu::GpuFSMapper gpu(1000.0, 6, descs[c], cuts);
            if (gpu.NDims() != stock.NDims()) {
                std::printf("NDIMS mismatch %zu %zu\n", gpu.NDims(), stock.NDims());
                return 1;
            }
            std::vector<double> dg, dw;
            double rmax = 0;
            int nan_mismatch = 0;
            for (int i = 0; i < npts; ++i) {
                std::vector<double> x(stock.NDims());
                for (auto &v : x) v = U(gen);
                std::vector<FourVector> ms, mg;
                stock.GeneratePoint(ms, x);
                gpu.GeneratePoint(mg, x);
                // component differences relative to the leg's energy (a
                // component near zero has no relative precision of its own)
                for (size_t k = 0; k < ms.size(); ++k) {
                    const bool e_ok = !std::isnan(ms[k][0]);
                    const double scale = e_ok ? std::max(std::abs(ms[k][0]), 1e-300) : 1.0;
                    for (size_t q = 0; q < 4; ++q) {
                        if (std::isnan(ms[k][q]) != std::isnan(mg[k][q])) ++nan_mismatch;
                        else if (e_ok && !std::isnan(ms[k][q])) dg.push_back(std::abs(mg[k][q] - ms[k][q]) / scale);
                    }
                }
                if (std::isnan(ms[0][0])) continue;
                // in/out uniform buffers that start alike with values the map may leave
                std::vector<double> rs(stock.NDims()), rg;
                for (auto &v : rs) v = U(gen);
                rg = rs;
                const double ws = stock.GenerateWeight(ms, rs);
                const double wg = gpu.GenerateWeight(ms, rg);
                if (std::isnan(ws) != std::isnan(wg)) ++nan_mismatch;
                else dw.push_back(rel(wg, ws));
                for (size_t k = 0; k < rs.size(); ++k) rmax = std::max(rmax, rel(rg[k], rs[k]));
            }
            std::printf("MAP %zu %d %.3e %.3e %.3e %.3e %.3e %d\n", c, npts,
                        dg.empty() ? 0 : *std::max_element(dg.begin(), dg.end()), p99(dg),
                        dw.empty() ? 0 : *std::max_element(dw.begin(), dw.end()), p99(dw), rmax, nan_mismatch);
        }
        // 2. the reference's MultiChannel over the two integrands
        chili::MultiChannelParams params;
        params.ncalls = ncalls;
        params.niterations = static_cast<size_t>(iters);
        params.should_optimize = false;  // no adaptation: the same grids and weights on both sides
        auto fs = integrand<chili::FSMapper>(descs, cuts, 50);
        auto fg = integrand<chili::gpu::GpuFSMapper>(descs, cuts, 50);
        chili::MultiChannel ms(fs.NDims(), fs.NChannels(), params), mg(fg.NDims(), fg.NChannels(), params);
        std::vector<chili::StatsData> rs, rg;
        chili::Random::Instance().Seed(7);
        for (int k = 0; k < iters; ++k) ms(fs);
        chili::Random::Instance().Seed(7);
        for (int k = 0; k < iters; ++k) mg(fg);
        std::ostringstream sink;
        const auto ss = ms.Summary(sink), sg = mg.Summary(sink);
        for (int k = 0; k < iters; ++k)
            std::printf("ITER %d %.0f %.17e %.17e %.17e %.17e\n", k, ss.results[k].Calls() * 1.0,
                        ss.results[k].Mean(), sg.results[k].Mean(),
                        ss.results[k].Variance(), sg.results[k].Variance());
        // 3. a checkpoint written with the GPU mappers loads into stock FSMappers
        const std::string path = std::string(argc > 4 ? argv[4] : "mapper_driver.chili");
        if (!mg.SaveAs(fg, path)) {
            std::printf("SAVE failed\n");
            return 1;
        }
        chili::Integrand<FourVector> back;
        chili::MultiChannel mb(fs.NDims(), fs.NChannels(), params);
        const bool ok = mb.LoadFrom(back, path) && back.NChannels() == fs.NChannels() &&
                        back.GetChannel(0).mapping->NDims() == fs.NDims();
        std::printf("SAVE %s\n", ok ? "ok" : "mismatch");
    } catch (const std::exception &e) {
        std::printf("ERROR %s\n", e.what());
        return 1;
    }
    return 0;
}
