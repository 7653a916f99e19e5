// Channels of a process from a model, as src/example.cc would build them with
// chili::ConstructChannels (ChannelNode.cc:74-291), through the C++ adapters:
// prints the number of channels and one line per description.
//   construct_channels [smax]
#include <cstdio>
#include <cstdlib>

#include "chili_b200.hh"

int main(int argc, char **argv) {
    const size_t smax = argc > 1 ? static_cast<size_t>(std::atoi(argv[1])) : 2;
    // a Z / photon model: f f~ -> gamma, Z; f V -> f
    chili::gpu::Model model([](int a, int b) -> std::vector<int> {
        if (a == -b && a != 0 && std::abs(a) != 22 && std::abs(a) != 23) return {22, 23};
        if (b == 22 || b == 23) return {a};
        if (a == 22 || a == 23) return {b};
        return {};
    });
    for (int f : {11, 13, 22}) model.Mass(f) = 0, model.Width(f) = 0;
    model.Mass(23) = 91.1876;
    model.Width(23) = 2.4952;
    const std::vector<int> flavs{11, -11, 13, -13, 22};
    try {
        auto set = chili::gpu::ConstructChannels(1000.0, flavs, model, smax);
        std::printf("CHANNELS %d\n", set.nch());
        const std::string why = set.Check();
        std::printf("CHECK %s\n", why.empty() ? "ok" : why.c_str());
        for (int c = 0; c < set.nch(); ++c) {
            const auto &d = set.descs()[c];
            std::printf("channel %d:", c);
            for (int k = 0; k < d.n_info; ++k) std::printf(" (%u,%d)", d.info[k].idx, d.info[k].pid);
            for (int k = 0; k < d.n_decays; ++k)
                std::printf(" [%u->%u+%u]", d.decays[k].parent.idx, d.decays[k].child1.idx, d.decays[k].child2.idx);
            std::printf("\n");
        }
    } catch (const chili::gpu::Error &e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
