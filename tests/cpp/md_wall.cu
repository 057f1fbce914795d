// A user component in the reference's plugin form (cuda::Component with
// build / launch / destroy, registered by MD::on(md::Phase::force).add):
// a harmonic wall E = k d^2, F_z = -2 k d for atoms whose z lies d above
// the plane z = zw, written as this program's own CUDA kernel and run by
// the library at the force phase of every step.  A second component at
// end_of_step records the step indices it sees and whether the plan asked
// for the virial.
//
// Usage: md_wall FRAME N1 N2 OUT -- runs N1 steps, then N2 more (run() is
// continuable), writes x y z vx vy vz fx fy fz (n doubles each) to OUT and
// prints "energy kinetic builds destroys last_step stress_required".
// FRAME (little endian): int64 n, then double box[3], dt, cutoff, skin, zw,
// k, then per atom x, y, z, vx, vy, vz, mass (double).
#include <atomiverse_b200/md.hpp>

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>

using namespace atvb_cpp;

__global__ void k_wall(int64_t n, const double* __restrict__ z, double* __restrict__ fz,
                       double* energy, double zw, double k) {
    __shared__ double sh[256];
    double e = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double d = z[i] - zw;
        if (d > 0.0) {
            fz[i] += -2.0 * k * d;
            e += k * d * d;
        }
    }
    sh[threadIdx.x] = e;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        atomicAdd(energy, sh[0]);
}

static int g_builds = 0, g_destroys = 0;

class HarmonicWall : public Component {
  public:
    HarmonicWall(double zw, double k) : zw_(zw), k_(k) {}
    std::string name() const override { return "HarmonicWall"; }
    bool provides_force() const override { return true; }
    bool provides_energy() const override { return true; }
    void build(const BuildContext&) override { ++g_builds; }
    void launch(const LaunchContext& ctx) override {
        const atvb_device_frame& f = ctx.frame;
        k_wall<<<32, 256, 0, (cudaStream_t)ctx.stream>>>(f.n_atoms, f.z, f.fz, f.energy, zw_, k_);
    }
    void destroy(const DestroyContext&) override { ++g_destroys; }

  private:
    double zw_, k_;
};

// Observes the plan: the cumulative step index and the stress verdict.
class StepProbe : public Component {
  public:
    StepProbe(long long* last, int* stress) : last_(last), stress_(stress) {}
    std::string name() const override { return "StepProbe"; }
    bool requires_system_stress() const override { return true; }
    void set_stress_required(bool on) override { *stress_ = on ? 1 : 0; }
    void launch(const LaunchContext& ctx) override {
        if (ctx.at(md::Phase::end_of_step))
            *last_ = ctx.step;
    }

  private:
    long long* last_;
    int* stress_;
};

int main(int argc, char** argv) {
    if (argc < 5) {
        std::fprintf(stderr, "usage: md_wall FRAME N1 N2 OUT\n");
        return 2;
    }
    FILE* fp = std::fopen(argv[1], "rb");
    if (!fp)
        return 2;
    int64_t n = 0;
    double hdr[8];
    bool ok = std::fread(&n, 8, 1, fp) == 1 && std::fread(hdr, 8, 8, fp) == 8 && n > 0;
    Frame f;
    if (ok) {
        f.resize((int)n);
        for (auto* v : {&f.x, &f.y, &f.z, &f.vx, &f.vy, &f.vz, &f.mass})
            ok = ok && std::fread(v->data(), 8, (size_t)n, fp) == (size_t)n;
    }
    std::fclose(fp);
    if (!ok)
        return 2;
    for (int k = 0; k < 3; ++k)
        f.box[k] = hdr[k];
    const double dt = hdr[3], rc = hdr[4], skin = hdr[5], zw = hdr[6], kw = hdr[7];
    long long last = -1;
    int stress = -1;
    atvb_scalars sc{};
    try {
        md::MD sim(0, ATVB_FP64);
        sim.set_neighbor(NeighborList{rc, skin});
        sim.set_evaluator(PairLJCut{1.0, 1.0, rc});
        sim.set_integrator(md::VelocityVerlet{dt});
        sim.on(md::Phase::force).add(HarmonicWall{zw, kw}, 0);
        sim.on(md::Phase::end_of_step).add(StepProbe{&last, &stress}, 10);
        sim.run(f, std::atoi(argv[2]));
        sc = sim.run(f, std::atoi(argv[3]));
    } catch (const std::exception& e) {
        std::fprintf(stderr, "md_wall: %s\n", e.what());
        return 1;
    }
    FILE* out = std::fopen(argv[4], "wb");
    if (!out)
        return 2;
    for (auto* v : {&f.x, &f.y, &f.z, &f.vx, &f.vy, &f.vz, &f.fx, &f.fy, &f.fz})
        std::fwrite(v->data(), 8, (size_t)n, out);
    std::fclose(out);
    std::printf("%.17g %.17g %d %d %lld %d\n", sc.energy, sc.kinetic, g_builds, g_destroys, last,
                stress);
    return 0;
}
