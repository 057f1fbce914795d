// Checkpoint and resume through the C++ mirror: an MTK NPT LJ run stopped
// after 40 steps, checkpointed, resumed in a fresh md::MD and continued for
// 40 more steps ends bit for bit where an uninterrupted 80-step run ends.
// Also reads trajectory snapshots (every 20 steps).  Prints "OK <frames>" or
// the first mismatch.
#include <atomiverse_b200/md.hpp>

#include <cmath>
#include <cstdio>
#include <cstdlib>

using namespace atvb_cpp;

static Frame lattice() {
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
    return f;
}

static void configure(md::MD& sim) {
    const double T = 1.0 / 8.617333262e-5;
    sim.set_neighbor(NeighborList(2.5, 0.3))
        .set_evaluator(PairLJCut(1.0, 1.0, 2.5))
        .set_integrator(md::NoseHooverNPT(T, 0.1, 0.0, 1.0, 0.005));
}

int main() {
    try {
        Frame a = lattice();
        md::MD sa;
        configure(sa);
        sa.set_snapshots(20, 8);
        sa.run(a, 80);
        std::vector<int64_t> steps;
        std::vector<double> xyz;
        const int frames = sa.poll_snapshots(steps, xyz);

        Frame b = lattice();
        std::vector<char> blob;
        {
            md::MD sb;
            configure(sb);
            sb.run(b, 40);
            blob = sb.checkpoint();
        }
        Frame c = lattice();
        md::MD sc;
        configure(sc);
        sc.restore(c, blob);
        sc.run(c, 40);
        for (int i = 0; i < a.n(); ++i)
            if (a.x[i] != c.x[i] || a.y[i] != c.y[i] || a.z[i] != c.z[i] || a.vx[i] != c.vx[i]) {
                std::printf("MISMATCH %d\n", i);
                return 1;
            }
        if (a.box[0] != c.box[0]) {
            std::printf("MISMATCH box\n");
            return 1;
        }
        std::printf("OK %d\n", frames);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "md_resume: %s\n", e.what());
        return 1;
    }
    return 0;
}
