// A driver in the style of the reference's src/example.cc, written against
// the C++ adapters of include/chili_b200.hh: the 2->4 propagator integrand on
// nine channels (six Z -> pair channels and three pure multi-peripheral
// chains), optimised on the GPU.
//
//   g++ -std=c++17 -O2 -I include examples/multichannel_2to4.cc \
//       -L chili_b200 -lchili_b200 -Wl,-rpath,$PWD/chili_b200 -o mc2to4
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <iostream>

#include "chili_b200.hh"

using chili::gpu::ChannelDescription;
using chili::gpu::ParticleInfo;

int main(int argc, char **argv) {
    const int iterations = argc > 1 ? std::atoi(argv[1]) : 5;
    const int flavs[6] = {1, -1, 11, -11, 13, -13};
    chili::gpu::Cuts cuts;  // the defaults of ConstructChannels (ChannelNode.cc:69-95)
    for (int f1 : flavs)
        for (int f2 : flavs) cuts.deltaR[{f1, f2}] = 0.4;
    for (int i = 0; i < 6; ++i) {
        cuts.smin[1u << i] = 0;
        cuts.ptmin[1u << i] = 30;
        cuts.etamax[1u << i] = 99;
        if (i > 1) cuts.sexternal.push_back(0);
    }
    auto leg = [&](int i) { return ParticleInfo{1u << i, flavs[i], 0, 0}; };
    std::vector<ChannelDescription> channels;
    for (int a = 2; a < 6; ++a)
        for (int b = a + 1; b < 6; ++b) {  // Z -> (a, b)
            ParticleInfo z{(1u << a) | (1u << b), 23, 91.1876, 2.4952};
            cuts.ptmin[z.idx] = 0;
            cuts.etamax[z.idx] = 99;
            ChannelDescription d;
            std::vector<ParticleInfo> t{z};
            for (int k = 2; k < 6; ++k)
                if (k != a && k != b) t.push_back(leg(k));
            std::sort(t.begin(), t.end(), [](const ParticleInfo &x, const ParticleInfo &y) { return x.idx > y.idx; });
            d.info = t;
            d.decays.push_back({z, {leg(a), leg(b)}});
            channels.push_back(d);
        }
    for (int last = 2; last < 5; ++last) {  // multi-peripheral chains
        ChannelDescription d;
        for (int k = 5; k >= 2; --k)
            if (k != last) d.info.push_back(leg(k));
        d.info.push_back(leg(last));
        channels.push_back(d);
    }
    chili::gpu::ChannelSet set(channels, cuts, 1000.0, 6);
    const std::string why = set.Check();
    if (!why.empty()) {
        std::cerr << "invalid channels: " << why << "\n";
        return 2;
    }
    chili::gpu::MultiChannelParams params;
    params.ncalls = 200000;
    params.niterations = static_cast<size_t>(iterations);
    params.nrefine = params.niterations + 1;  // no refinement
    params.rtol = 0;
    try {
        chili::gpu::MultiChannel mc(set, 100, params, CHILI_FUNC_PROPAGATOR, {91.1876, 2.4952, 10.0});
        mc.Optimize(&std::cout);
        auto summary = mc.Summary(std::cout);
        const auto r = summary.Result();
        std::printf("RESULT %.10e %.10e %zu\n", r.Mean(), r.Error(), r.Calls());
    } catch (const chili::gpu::Error &e) {
        std::cerr << e.what() << "\n";
        return 1;
    }
    return 0;
}
