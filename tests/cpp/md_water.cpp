// A caller of the reference-shaped C++ API with a molecular system: per-type
// PairLJCut coefficients (LJ on oxygen only), CoulLong + KSpacePME, and
// special bonds excluding the intramolecular 1-2/1-3 pairs (the pattern of
// the reference's SPC/E water setups).  Reads the frame from a binary file
// written by the test, runs n steps and prints the energies and a position
// checksum so the test can compare against the Python layer bit for bit.
//
// File layout (little endian): int64 n, int64 nbonds, double box[3],
// double alpha, double rc, int64 grid, then per atom x, y, z, q, mass
// (double) and type (int32), then nbonds pairs of int64 tags.
#include <atomiverse_b200/md.hpp>

#include <cstdio>
#include <cstdlib>

int main(int argc, char** argv) {
    using namespace atvb_cpp;
    if (argc < 4) {
        std::fprintf(stderr, "usage: md_water FRAME N_STEPS PRECISION\n");
        return 2;
    }
    FILE* fp = std::fopen(argv[1], "rb");
    if (!fp)
        return 2;
    int64_t n = 0, nb = 0, grid = 0;
    double box[3], alpha = 0, rc = 0;
    bool ok = std::fread(&n, 8, 1, fp) == 1 && std::fread(&nb, 8, 1, fp) == 1 &&
              std::fread(box, 8, 3, fp) == 3 && std::fread(&alpha, 8, 1, fp) == 1 &&
              std::fread(&rc, 8, 1, fp) == 1 && std::fread(&grid, 8, 1, fp) == 1;
    if (!ok || n <= 0 || nb < 0)
        return 2;
    Frame f;
    f.resize((int)n);
    f.type.resize(n);
    for (auto* v : {&f.x, &f.y, &f.z, &f.charge, &f.mass})
        ok = ok && std::fread(v->data(), 8, (size_t)n, fp) == (size_t)n;
    ok = ok && std::fread(f.type.data(), 4, (size_t)n, fp) == (size_t)n;
    f.bonds.resize(nb);
    for (auto& b : f.bonds)
        ok = ok && std::fread(&b.first, 8, 1, fp) == 1 && std::fread(&b.second, 8, 1, fp) == 1;
    std::fclose(fp);
    if (!ok)
        return 2;
    for (int k = 0; k < 3; ++k)
        f.box[k] = box[k];

    try {
        KSpacePME pme(alpha, 1.0, 4);
        pme.grid[0] = pme.grid[1] = pme.grid[2] = (int)grid;
        md::MD sim(0, std::atoi(argv[3]));
        sim.set_neighbor(NeighborList(rc, 1.0))
            .set_evaluator(PairLJCut({{0, 0, 0.0067, 3.166}}, rc).set_special_bonds(0.0, 0.0, 0.0))
            .set_evaluator(CoulLong(alpha, rc).set_special_bonds(0.0, 0.0, 0.0))
            .set_evaluator(pme)
            .set_integrator(md::VelocityVerlet(0.5));
        atvb_scalars s = sim.run(f, std::atoi(argv[2]));
        double sum = 0.0;
        for (int i = 0; i < f.n(); ++i)
            sum += f.x[i] + 2.0 * f.y[i] + 3.0 * f.z[i];
        std::printf("%lld %.17g %.17g %.17g %.17g\n", (long long)s.step, s.energy_lj,
                    s.energy_coul, s.energy_recip, sum);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "md_water: %s\n", e.what());
        return 1;
    }
    return 0;
}
