// The reference's benchmark driver (src/Test.cpp:50-74, its Base block) with `Base::` swapped
// for `GPU::`: the same case — M = 2 freestream, gamma 1.4, dt = 1e-3, 1000 steps, BC map
// by colour tag — on the B200 solver through the C++ drop-in of hcfd_gpu.hpp.
//
//   hcfd_wedge_driver <mesh.hmsh> <output prefix> [niter]
//
// writes <prefix>_0.hsln (t = 0) and <prefix>_1.hsln (t = niter dt), like the reference's
// ../sols/Base_{0,1}.hsln, and prints the device-loop time.
#include "hcfd_gpu.hpp"

#include <chrono>
#include <cstdio>
#include <cstdlib>

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s mesh.hmsh out_prefix [niter]\n", argv[0]);
        return 2;
    }
    try {
        const int nvars = 4;
        const double gma = 1.4;
        double M = 2.0;
        double p = 1.0 / (gma * M * M);
        const double QIC[] = {1, 1, 0, p};
        const double QBC[][4] = {{1, 1, 0, p}, {1, 1, 0, p}, {1, 1, 0, p}, {1, 1, 0, p}};
        double dt = 1e-3;
        GPU::Mesh mesh(argv[1]);
        int niter = argc > 3 ? std::atoi(argv[3]) : 1000;

        const GPU::BCtype BCmap[] = {GPU::SYMMETRY, GPU::SYMMETRY, GPU::SYMMETRY, GPU::SUPINLET, GPU::SUPOUTLET};
        GPU::Domain domain(mesh);
        GPU::GaussGreen grads(domain);
        GPU::Limiter limiter(domain);
        GPU::Flux flux(nvars, gma, domain);
        GPU::Euler intg(nvars, domain, flux, grads, limiter);
        intg.set_output(argv[2]);
        intg.gather_BCs(BCmap, QBC);
        intg.initialise(QIC);
        auto t1 = std::chrono::steady_clock::now();
        intg.run(niter * dt, dt, niter * dt);
        auto t2 = std::chrono::steady_clock::now();
        std::printf("GPU Base-equivalent run: %d steps, %.3f ms\n", niter,
                    std::chrono::duration<double, std::milli>(t2 - t1).count());
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
