// A caller written against the reference-shaped C++ API: an NVE Lennard-Jones
// lattice driven through md::MD (the pattern of the reference's
// regressions/md/lj_argon case).  Prints the energies of two run() chunks.
// With arguments `every [file]`, thermo rows every `every` steps come first.
#include <atomiverse_b200/md.hpp>

#include <cmath>
#include <cstdio>
#include <cstdlib>

int main(int argc, char** argv) {
    using namespace atvb_cpp;
    const int nc = 6;
    const double rho = 0.8442, a = std::cbrt(4.0 / rho);
    Frame f;
    f.resize(4 * nc * nc * nc);
    const double b[4][3] = {{0, 0, 0}, {0.5, 0.5, 0}, {0.5, 0, 0.5}, {0, 0.5, 0.5}};
    int k = 0;
    for (int i = 0; i < nc; ++i)
        for (int j = 0; j < nc; ++j)
            for (int l = 0; l < nc; ++l)
                for (int m = 0; m < 4; ++m, ++k) {
                    f.x[k] = (i + b[m][0]) * a;
                    f.y[k] = (j + b[m][1]) * a;
                    f.z[k] = (l + b[m][2]) * a + 0.01 * std::sin(k);
                    f.vx[k] = 0.01 * std::cos(3.0 * k);
                }
    f.box[0] = f.box[1] = f.box[2] = nc * a;
    md::MD sim;
    sim.set_neighbor(NeighborList(2.5, 0.3))
        .set_evaluator(PairLJCut(1.0, 1.0, 2.5))
        .set_integrator(md::VelocityVerlet(0.05));
    if (argc > 1)
        sim.set_thermo(std::atoi(argv[1]), argc > 2 ? argv[2] : "");
    atvb_scalars s1 = sim.run(f, 50);
    atvb_scalars s2 = sim.run(f, 50);
    std::printf("%lld %.10f %.10f %.10f\n", (long long)s2.step, s1.energy + s1.kinetic,
                s2.energy + s2.kinetic, s2.kinetic);
    return 0;
}
