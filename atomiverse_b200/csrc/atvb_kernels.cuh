// atvb_kernels.cuh -- launch configuration shared by the kernel launchers
// and the engine that captures them into the per-step CUDA graph.
#pragma once

#include <vector>

#include "atvb_common.cuh"

namespace atvb {

constexpr int kChunk = 256;     // atoms per item of the per-atom kernels
constexpr int kRebuildKernels = 6; // launches of one list build (cell sort + rows)
constexpr long long kCondMinAtoms = 100000; // engines from this size skip them by
                                            // conditional graph nodes
constexpr int kListChunk = 8;   // cells per item of the list build (warp/cell)
constexpr int kGridChunk = 4096; // grid points per item of the PME grid kernels
constexpr int kLaneClasses = 6;  // pair lanes per atom: 1, 2, 4, 8, 16, 32
constexpr int kGenLanes = 8;      // lanes per atom of k_pair_general
constexpr int kPairBlock = 256;  // pair-kernel threads per block (atoms per item = this / lanes)

struct ItemList {
    const Item* d = nullptr; // device array
    int n = 0;               // number of items
    int grid = 0;            // blocks to launch (persistent loop covers n)
};

// The PME transforms of a launch (fft.cu): per pass, one group of items
// per line length (the z passes: first line of a group of lines; the y
// passes: k0 x column block; the x pass: m1 x column block), so that each
// system's transform depends on its own mesh alone, whatever it is batched
// with.
constexpr int kFftBlock = 256;          // threads per FFT block
constexpr int kFftSmem = 56 * 1024;     // shared memory an FFT block may use
constexpr int kFftMaxLines = 16;        // lines per FFT block
struct FftGroup {
    ItemList items;
    int n = 0;    // line length (z: K2 / 2 for an even K2, else K2)
    int k = 0;    // roots of unity of the axis (z: K2)
    int reg = -1; // register form (fft_reg*.cu), -1 for the generic kernels
    int c = 1;    // lines (z) or columns (y, x) per item
};
struct FftCfg {
    std::vector<FftGroup> z, y, x;
    int launches() const { return (int)(2 * z.size() + 2 * y.size() + x.size()); }
};

struct LaunchCfg {
    const SysParams* sp = nullptr; // device table of every system
    ItemList atoms;     // kChunk atoms per item (original or sorted order)
    ItemList list;      // kListChunk cells per item
    // pair work by [precision][log2 lanes]: each system has its own lane
    // count, chosen from that system alone, so its forces and energies do
    // not depend on which other systems share the engine
    ItemList pair[2][kLaneClasses];
    ItemList pair_gen[2]; // [precision]: systems with types or special pairs
                          // (kChunk / kGenLanes atoms per item)
    ItemList cells;     // kChunk cells per item
    ItemList pme_atoms; // kChunk atoms of PME systems
    ItemList pme_grid;  // kGridChunk half-complex grid points per item
    ItemList pme_real;  // kGridChunk real grid points per item
    const int* sys_list = nullptr; // device list of system indices
    int nsys = 0;
    int pair_G = 4;     // lanes per atom of the largest system (reported)
    int any_mixed = 0, any_fp64 = 0;
    int any_snap = 0;   // a system publishes trajectory snapshots
    int any_baro = 0;   // a system runs the Berendsen barostat (k_baro_scale)
    int any_near = 0;   // a mixed system settles near-cutoff LJ pairs (k_pair_fix)
    FftCfg fft;         // the PME grid transforms
    int pme_order = 4;  // common PME order (the PME kernels are templated)
    int pme_mixed = 0;
};

// neighbor.cu
void launch_rebuild(const LaunchCfg& lc, cudaStream_t s);
void launch_sort_cells(const LaunchCfg& lc, cudaStream_t s);
void launch_build_list(const LaunchCfg& lc, cudaStream_t s);
// pair.cu
void launch_pair(const LaunchCfg& lc, cudaStream_t s);
void launch_pair_fix(const LaunchCfg& lc, cudaStream_t s);
// pair_general.cu
void launch_pair_general(const LaunchCfg& lc, cudaStream_t s);
void cuda_check(cudaError_t e, const char* what); // engine.cu: throws on error

// pme.cu
void launch_pme_spread(const LaunchCfg& lc, cudaStream_t s);
void launch_pme_gather(const LaunchCfg& lc, cudaStream_t s);
// fft.cu
void launch_pme_fft(const LaunchCfg& lc, cudaStream_t s);
void fft_smem_optin(int bytes);
int fft_lines_per_block(int n, int K, bool mixed);
// Register forms of the line transforms (fft_reg.cu): the form of a line
// length (-1: none), z lines per item, y / x columns per item, and a launch
// of one pass (0 z forward, 1 y forward, 2 x with the influence function,
// 3 y inverse, 4 z inverse).
int fft_reg_index(int n);
int fft_reg_lines(int idx, bool mixed);
int fft_reg_cols(bool mixed);
void launch_fft_reg(int pass, int idx, bool mixed, const ItemList& il, const SysParams* sp,
                    cudaStream_t s);
// integrate.cu
void launch_integrate_a(const LaunchCfg& lc, cudaStream_t s);
// cond_sort / cond_rows / use_cond: the step graph's conditional handles of
// the list build (set when a system rebuilds), only while the step is being
// captured
void launch_sys_a(const LaunchCfg& lc, cudaStream_t s, cudaGraphConditionalHandle cond_sort = 0,
                  cudaGraphConditionalHandle cond_rows = 0, bool use_cond = false);
void launch_integrate_b(const LaunchCfg& lc, cudaStream_t s);
void launch_sys_b(const LaunchCfg& lc, cudaStream_t s);
void launch_sys_energy(const LaunchCfg& lc, cudaStream_t s);
void launch_force_rebuild(const LaunchCfg& lc, cudaStream_t s);
void launch_state_in(const LaunchCfg& lc, cudaStream_t s);
void launch_wrap_in(const LaunchCfg& lc, cudaStream_t s);
void launch_state_out(const LaunchCfg& lc, int what, cudaStream_t s);
void launch_npt_prep(const LaunchCfg& lc, cudaStream_t s);
void launch_repack(const LaunchCfg& lc, cudaStream_t s);
void launch_snapshots(const LaunchCfg& lc, cudaStream_t s);
void launch_force_combine(const LaunchCfg& lc, cudaStream_t s);
void launch_kinetic(const LaunchCfg& lc, cudaStream_t s);

} // namespace atvb
