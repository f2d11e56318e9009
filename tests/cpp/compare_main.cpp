// A Compare-mode driver in the shape of the reference's src/Parareal/main.cpp
// (lines 183-255), written against include/sp_convection.hpp: analytic initial
// field (exactQ), DoSerial, DoParallel, max-norm relative error of the
// Parareal result against the serial one (computeErrorReference).
// usage: compare_main P [--gridSize N --endTime T --timeStepsFine F --timeStepsCoarse G --kmax K --nu0 ...]
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "sp_convection.hpp"

static double exactQ(double nu0, double nufreq, double cx, double cy, double cz, double x, double y, double z,
                     double t) {
    const double pi = 3.14159265358979;
    const double a = nufreq > 0 ? nu0 * t - (nu0 / (2. * nufreq)) * (std::cos(nufreq * t) - 1.) : nu0 * t;
    return std::sin(2. * pi * (x - cx * t)) * std::sin(2. * pi * (y - cy * t)) * std::sin(2. * pi * (z - cz * t)) *
           std::exp(-12. * pi * pi * a);
}

int main(int argc, char** argv) {
    if (argc < 2) { std::fprintf(stderr, "usage: %s P [options]\n", argv[0]); return 2; }
    const int P = std::atoi(argv[1]);
    try {
        sp::RuntimeConfiguration conf(P, argc - 1, argv + 1);
        const int N = conf.gridSize();
        sp::ConvectionField q, qinitial, qreference;
        q.Init("q", N, N, N);
        qinitial.Init("qinitial", N, N, N);
        qreference.Init("qreference", N, N, N);
        sp::Convection convection(N, N, N, conf.dx(), conf.nu0(), conf.nufreq(), conf.cx(), conf.cy(), conf.cz());
        sp::Parareal<sp::Convection, sp::ConvectionField> parareal(convection, qinitial, q, 0., conf);
        std::vector<double> init((size_t)N * N * N);
        for (int k = 0; k < N; ++k)
            for (int j = 0; j < N; ++j)
                for (int i = 0; i < N; ++i)
                    init[((size_t)k * N + j) * N + i] = exactQ(conf.nu0(), conf.nufreq(), conf.cx(), conf.cy(),
                                                               conf.cz(), (i + .5) / N, (j + .5) / N, (k + .5) / N, 0.);
        convection.fill(qinitial, init);
        parareal.DoSerial();
        convection.synchronize();
        cudaMemcpy(qreference.data(), q.data(), q.layout().total * sizeof(double), cudaMemcpyDeviceToDevice);
        convection.fill(qinitial, init);
        parareal.DoParallel(&qreference);
        const sp_parareal_report& r = parareal.report();
        std::printf("timesteps per slice fine propagator: %d\n", r.tsFine);
        std::printf("timesteps per slice coarse propagator: %d\n", r.tsCoarse);
        for (int k = 0; k < r.iterations; ++k) std::printf("Error after iteration %d: %.7e\n", k + 1, r.err_max[k]);
        std::printf("Error at end: %.7e\n", r.err_max[r.iterations - 1]);
        std::printf("Parallel run time: %.6f\n", r.seconds);
    } catch (const sp::Error& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
