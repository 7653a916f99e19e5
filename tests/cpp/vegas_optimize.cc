// Test driver: chili::gpu::Vegas::Optimize (include/chili_b200.hh) on the
// camel, with the uniforms replayed from a file (the reference's own stream,
// written by the test) so that its iterations can be compared with the
// reference's Vegas::Optimize (Vegas.cc:54-69) on the same uniforms.
//
//   vegas_optimize <uniforms.bin> <params.bin> <edges_out.bin> dims bins ncalls nrefine atol rtol nitn alpha
//
// Prints one "ITER n sum sum2" line per iteration, then
// "RESULT iterations bins ncalls mean error"; writes the final grid edges.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <vector>

#include "chili_b200.hh"

static std::vector<double> read_doubles(const char *path) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    const std::streamsize n = f.tellg();
    f.seekg(0);
    std::vector<double> v(static_cast<size_t>(n) / sizeof(double));
    f.read(reinterpret_cast<char *>(v.data()), static_cast<std::streamsize>(v.size() * sizeof(double)));
    return v;
}

int main(int argc, char **argv) {
    if (argc != 12) {
        std::cerr << "usage: vegas_optimize uniforms params edges_out dims bins ncalls nrefine atol rtol nitn alpha\n";
        return 2;
    }
    const std::vector<double> u = read_doubles(argv[1]);
    const std::vector<double> camel = read_doubles(argv[2]);
    const size_t dims = std::strtoul(argv[4], nullptr, 10), bins = std::strtoul(argv[5], nullptr, 10);
    chili::gpu::VegasParams params;
    params.ncalls = std::strtoul(argv[6], nullptr, 10);
    params.nrefine = std::strtoul(argv[7], nullptr, 10);
    params.atol = std::atof(argv[8]);
    params.rtol = std::atof(argv[9]);
    params.ninterations = std::strtoul(argv[10], nullptr, 10);
    params.alpha = std::atof(argv[11]);
    size_t pos = 0;
    try {
        chili::gpu::Vegas vegas(chili::gpu::AdaptiveMap(dims, bins), params, camel);
        vegas.SetUniformSource([&](size_t n, double *out) {
            if (pos + n > u.size()) throw std::runtime_error("the uniform file ran out");
            for (size_t i = 0; i < n; ++i) out[i] = u[pos + i];
            pos += n;
        });
        vegas.Optimize();
        const auto summary = vegas.Summary();
        for (const auto &r : summary.results) std::printf("ITER %zu %.17e %.17e\n", r.Calls(), r.sum, r.sum2);
        const auto &grid = vegas.Grid();
        std::ofstream out(argv[3], std::ios::binary);
        out.write(reinterpret_cast<const char *>(grid.Hist().data()),
                  static_cast<std::streamsize>(grid.Hist().size() * sizeof(double)));
        const auto res = summary.Result();
        std::printf("RESULT %zu %zu %zu %.17e %.17e %zu\n", summary.results.size(), grid.Bins(),
                    vegas.Params().ncalls, res.Mean(), res.Error(), pos);
    } catch (const std::exception &e) {
        std::cerr << e.what() << "\n";
        return 1;
    }
    return 0;
}
