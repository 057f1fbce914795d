// The reference's npt_lj_mtk regression written against the C++ mirror:
// 6^3 simple-cubic LJ at rho = 0.8, eps = sigma = 1, r_c = 2.5, MTK NPT at
// T* = 1 (T = 1/k_B K with eps = 1 eV), tau_T = 0.1, P = 0, tau_P = 1,
// dt = 0.005, 80 steps.  Prints the final cell volume and the conserved
// extended Hamiltonian.
#include <atomiverse_b200/md.hpp>

#include <cmath>
#include <cstdio>
#include <cstdlib>

int main(int argc, char** argv) {
    using namespace atvb_cpp;
    const int ns = 6, n = ns * ns * ns;
    const double L = std::cbrt(n / 0.8), a = L / ns;
    Frame f;
    f.resize(n);
    int k = 0;
    for (int ix = 0; ix < ns; ++ix)
        for (int iy = 0; iy < ns; ++iy)
            for (int iz = 0; iz < ns; ++iz, ++k) {
                f.x[k] = (ix + 0.5) * a;
                f.y[k] = (iy + 0.5) * a;
                f.z[k] = (iz + 0.5) * a;
                f.vx[k] = 0.02 * ((ix + iy + iz) % 3 - 1);
                f.vy[k] = 0.02 * ((ix + 2 * iy) % 3 - 1);
                f.vz[k] = 0.02 * ((2 * ix + iz) % 3 - 1);
            }
    f.box[0] = f.box[1] = f.box[2] = L;
    try {
        const double T = 1.0 / 8.617333262e-5;
        md::MD sim(0, argc > 1 ? std::atoi(argv[1]) : ATVB_FP64);
        sim.set_neighbor(NeighborList(2.5, 0.3))
            .set_evaluator(PairLJCut(1.0, 1.0, 2.5))
            .set_integrator(md::NoseHooverNPT(T, 0.1, 0.0, 1.0, 0.005));
        atvb_scalars s = sim.run(f, 80);
        std::printf("%.12f %.12e %d\n", f.box[0] * f.box[1] * f.box[2], s.conserved, s.status);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "md_npt: %s\n", e.what());
        return 1;
    }
    return 0;
}
