// static_forces.cu -- atvb_pair_forces_static: the short-range pair term
// (shifted LJ 12-6 + real-space Ewald erfc Coulomb) for caller-owned device
// arrays, with no device or host allocation.
//
// Every intermediate (cell counts and starts, per-atom cell and slot, the
// cell-sorted positions, two fixed-point energy sums) lives in one file-scope
// __device__ array of fixed size, so the call needs no cudaMalloc, no
// cudaFree and no allocating library routine.  That array is one per device:
// calls on the same device must not overlap (issue them on one stream, or
// order their streams); two calls in flight at once corrupt each other's
// scratch.  The first call on a device looks the array's address up with
// cudaGetSymbolAddress; make that first call outside any stream capture.
// The address is kept per device together with the id of the context it
// belongs to, and looked up again when that context changes (after a
// cudaDeviceReset the array lives at a new address).
//
// Method: cells of edge >= the larger cutoff, count / scan / scatter of
// atom indices, then each atom's place in its cell from the number of
// smaller indices in that cell (so every cell is in index order, sums run
// in a fixed order and repeat bit for bit; one thread per atom, no serial
// per-cell sort), then one thread per atom walks the
// 27 neighbouring cells (every cell along an axis with fewer than 3 cells).
// Physics as the library's main pair kernel: shifted LJ
// (src/cpu/potentials/pair_lj_cut.cpp:723-800, shift
// cuda/potentials/lj_kernel.cuh:59-65) and Coulomb
// k_e q_i q_j erfc(alpha r)/r (src/cpu/potentials/coul_long.cpp:146-222),
// minimum image in an orthorhombic box, energy halved per visit.
#include <cuda.h> // CUcontext / CUresult types only: no libcuda link
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "atvb.h"
#include "atvb_common.cuh"
#include "atvb_engine.h"

namespace atvb {
namespace {

constexpr int kStaticMaxAtoms = 65536;
constexpr int kStaticMaxCells = 65536;
constexpr int kStaticMaxDevices = 64;

// scratch layout (byte offsets, each a multiple of 256)
constexpr size_t kOffCount = 0;                                     // int[cells]
constexpr size_t kOffStart = kOffCount + 4 * (size_t)kStaticMaxCells; // int[cells + 64]
constexpr size_t kOffCell = kOffStart + 4 * ((size_t)kStaticMaxCells + 64); // int[atoms]
constexpr size_t kOffSlot = kOffCell + 4 * (size_t)kStaticMaxAtoms;  // int[atoms]
constexpr size_t kOffIdx = kOffSlot + 4 * (size_t)kStaticMaxAtoms;   // int[atoms]
constexpr size_t kOffPos = kOffIdx + 4 * (size_t)kStaticMaxAtoms;    // double4[atoms]
constexpr size_t kOffEnergy = kOffPos + 32 * (size_t)kStaticMaxAtoms; // u64[2]
constexpr size_t kOffTmp = kOffEnergy + 256;                        // int[atoms]
constexpr size_t kStaticBytes = kOffTmp + 4 * (size_t)kStaticMaxAtoms;
static_assert(kOffStart % 256 == 0 && kOffCell % 256 == 0 && kOffSlot % 256 == 0 &&
                  kOffIdx % 256 == 0 && kOffPos % 256 == 0 && kOffEnergy % 256 == 0 &&
                  kOffTmp % 256 == 0,
              "scratch regions must stay 256-byte aligned");

__device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

struct StaticArgs {
    int n;
    int nc[3];
    int ncell;
    double L[3], halfL[3], cinv[3];
    int has_lj, has_coul;
    double lj_rc2, lj_sig6, lj_eps4, lj_eps24, lj_shift;
    double c_rc2, c_alpha, c_alpha2;
    const double *x, *y, *z, *q;
    double *fx, *fy, *fz, *energy;
    int* count;
    int* start;
    int* cell;
    int* slot;
    int* sidx;
    int* tmp; // atom indices of each cell in arrival order
    double4* pos;
    unsigned long long* esum;
};

ATVB_DEV double wrap_static(double v, double L) {
    double w = v - L * floor(v / L);
    return w;
}

ATVB_DEV int cell_coord(double w, double cinv, int nc) {
    int c = (int)floor(w * cinv); // NaN -> INT_MIN, clamped below
    return c < 0 ? 0 : (c > nc - 1 ? nc - 1 : c);
}

__global__ void k_static_zero(StaticArgs a) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < a.ncell;
         c += gridDim.x * blockDim.x)
        a.count[c] = 0;
    if (blockIdx.x == 0 && threadIdx.x < 2)
        a.esum[threadIdx.x] = 0ull;
}

__global__ void k_static_bin(StaticArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n)
        return;
    const int cx = cell_coord(wrap_static(a.x[i], a.L[0]), a.cinv[0], a.nc[0]);
    const int cy = cell_coord(wrap_static(a.y[i], a.L[1]), a.cinv[1], a.nc[1]);
    const int cz = cell_coord(wrap_static(a.z[i], a.L[2]), a.cinv[2], a.nc[2]);
    const int c = (cx * a.nc[1] + cy) * a.nc[2] + cz;
    a.cell[i] = c;
    a.slot[i] = atomicAdd(&a.count[c], 1);
}

// Exclusive scan of the cell counts: one block of 1024 threads, each owning
// a contiguous run of at most 64 cells.
__global__ void __launch_bounds__(1024) k_static_scan(StaticArgs a) {
    __shared__ int warp_tot[32];
    const int t = threadIdx.x;
    const int per = (a.ncell + 1023) / 1024;
    const int b = t * per;
    const int e = min(b + per, a.ncell);
    int local = 0;
    for (int c = b; c < e; ++c)
        local += a.count[c];
    // inclusive warp scan, then across warps
    int v = local;
    const int lane = t & 31, w = t >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o)
            v += u;
    }
    if (lane == 31)
        warp_tot[w] = v;
    __syncthreads();
    if (w == 0) {
        int s = warp_tot[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o)
                s += u;
        }
        warp_tot[lane] = s;
    }
    __syncthreads();
    int run = v - local + (w > 0 ? warp_tot[w - 1] : 0);
    for (int c = b; c < e; ++c) {
        a.start[c] = run;
        run += a.count[c];
    }
    if (t == 1023)
        a.start[a.ncell] = run;
}

// Atom indices into their cells, in arrival order (which varies from call
// to call with the atomic slots).
__global__ void k_static_scatter(StaticArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n)
        return;
    a.tmp[a.start[a.cell[i]] + a.slot[i]] = i;
}

// Each atom's place in its cell = the number of smaller indices in that cell,
// so every cell ends up in original-index order whatever the arrival order.
// One thread per atom, O(atoms in the cell) each: a cell holding many atoms
// costs a longer scan per thread, never a serial sort.
__global__ void k_static_rank(StaticArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n)
        return;
    const int c = a.cell[i];
    const int b = a.start[c], e = a.start[c + 1];
    int r = 0;
    for (int k = b; k < e; ++k)
        r += a.tmp[k] < i ? 1 : 0;
    const int s = b + r;
    a.pos[s] = make_double4(wrap_static(a.x[i], a.L[0]), wrap_static(a.y[i], a.L[1]),
                            wrap_static(a.z[i], a.L[2]), a.has_coul ? a.q[i] : 0.0);
    a.sidx[s] = i;
}

ATVB_DEV double img(double d, double L, double halfL) {
    // both coordinates are in [0, L], so one fold suffices
    if (d > halfL)
        d -= L;
    else if (d < -halfL)
        d += L;
    return d;
}

__global__ void __launch_bounds__(256) k_static_forces(StaticArgs a) {
    __shared__ double sh[64];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double elj = 0.0, ec = 0.0;
    if (i < a.n) {
        const double xi = wrap_static(a.x[i], a.L[0]);
        const double yi = wrap_static(a.y[i], a.L[1]);
        const double zi = wrap_static(a.z[i], a.L[2]);
        const double kqi = a.has_coul ? kQqr2e * a.q[i] : 0.0;
        const int ci[3] = {cell_coord(xi, a.cinv[0], a.nc[0]),
                           cell_coord(yi, a.cinv[1], a.nc[1]),
                           cell_coord(zi, a.cinv[2], a.nc[2])};
        int lo[3], cnt[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (a.nc[d] >= 3) {
                lo[d] = ci[d] - 1;
                cnt[d] = 3;
            } else {
                lo[d] = 0;
                cnt[d] = a.nc[d];
            }
        }
        double fx = 0.0, fy = 0.0, fz = 0.0;
        for (int ox = 0; ox < cnt[0]; ++ox) {
            int cx = lo[0] + ox;
            cx += cx < 0 ? a.nc[0] : (cx >= a.nc[0] ? -a.nc[0] : 0);
            for (int oy = 0; oy < cnt[1]; ++oy) {
                int cy = lo[1] + oy;
                cy += cy < 0 ? a.nc[1] : (cy >= a.nc[1] ? -a.nc[1] : 0);
                for (int oz = 0; oz < cnt[2]; ++oz) {
                    int cz = lo[2] + oz;
                    cz += cz < 0 ? a.nc[2] : (cz >= a.nc[2] ? -a.nc[2] : 0);
                    const int c = (cx * a.nc[1] + cy) * a.nc[2] + cz;
                    const int e = a.start[c + 1];
                    for (int s = a.start[c]; s < e; ++s) {
                        if (a.sidx[s] == i)
                            continue;
                        const double4 pj = a.pos[s];
                        const double dx = img(xi - pj.x, a.L[0], a.halfL[0]);
                        const double dy = img(yi - pj.y, a.L[1], a.halfL[1]);
                        const double dz = img(zi - pj.z, a.L[2], a.halfL[2]);
                        const double r2 = dx * dx + dy * dy + dz * dz;
                        if (r2 < 1e-20)
                            continue;
                        const double r2inv = 1.0 / r2;
                        double fpair = 0.0;
                        if (a.has_lj && r2 < a.lj_rc2) {
                            const double r6inv = r2inv * r2inv * r2inv * a.lj_sig6;
                            fpair = a.lj_eps24 * r2inv * (2.0 * r6inv * r6inv - r6inv);
                            elj += a.lj_eps4 * (r6inv * r6inv - r6inv) - a.lj_shift;
                        }
                        if (a.has_coul && r2 < a.c_rc2) {
                            const double qq = kqi * pj.w;
                            if (qq != 0.0) {
                                const double r = sqrt(r2);
                                const double ar = a.c_alpha * r;
                                const double erfc_ar = erfc(ar);
                                const double g = kEwaldF * ar * exp(-a.c_alpha2 * r2);
                                fpair += qq * (erfc_ar + g) * r2inv / r;
                                ec += qq * erfc_ar / r;
                            }
                        }
                        fx += fpair * dx;
                        fy += fpair * dy;
                        fz += fpair * dz;
                    }
                }
            }
        }
        a.fx[i] = fx;
        a.fy[i] = fy;
        a.fz[i] = fz;
    }
    if (a.energy == nullptr)
        return;
    // each pair is visited from both ends: half the energy per visit
    double v[2] = {0.5 * elj, 0.5 * ec};
    block_sum_vec<2>(v, sh);
    if (threadIdx.x == 0) {
        fix_add(&a.esum[0], v[0]);
        fix_add(&a.esum[1], v[1]);
    }
}

__global__ void k_static_energy(StaticArgs a) {
    if (threadIdx.x < 2)
        a.energy[threadIdx.x] = (double)(long long)a.esum[threadIdx.x] * kEFixInv;
}

std::mutex g_scratch_mu;
void* g_scratch_addr[kStaticMaxDevices] = {};
unsigned long long g_scratch_ctx[kStaticMaxDevices] = {};

// Unique id of the calling thread's current context (cuCtxGetId), 0 if there
// is none yet.  The driver calls come through the runtime's entry-point
// lookup, so the library does not link libcuda itself.
unsigned long long current_ctx_id() {
    using GetCur = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCur get_cur = nullptr;
    static GetId get_id = nullptr;
    if (!get_cur || !get_id) {
        void* p = nullptr;
        void* q = nullptr;
        cudaDriverEntryPointQueryResult r1, r2;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault,
                                             &r1) != cudaSuccess ||
            cudaGetDriverEntryPointByVersion("cuCtxGetId", &q, 12000, cudaEnableDefault,
                                             &r2) != cudaSuccess ||
            !p || !q)
            return 0;
        get_cur = reinterpret_cast<GetCur>(p);
        get_id = reinterpret_cast<GetId>(q);
    }
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (get_cur(&c) != CUDA_SUCCESS || c == nullptr || get_id(c, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

unsigned char* static_scratch(int dev) {
    if (dev < 0 || dev >= kStaticMaxDevices)
        throw Error(ATVB_ERR_INVALID, "device ordinal out of range for the static scratch");
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    const unsigned long long ctx = current_ctx_id();
    if (g_scratch_addr[dev] == nullptr || ctx == 0 || ctx != g_scratch_ctx[dev]) {
        // first call on this device, or a new context (a device reset)
        void* p = nullptr;
        const cudaError_t rc = cudaGetSymbolAddress(&p, g_static_scratch);
        if (rc != cudaSuccess || p == nullptr)
            throw Error(ATVB_ERR_CUDA, std::string("cudaGetSymbolAddress(static scratch): ") +
                                           cudaGetErrorString(rc));
        g_scratch_addr[dev] = p;
        g_scratch_ctx[dev] = current_ctx_id(); // the context now exists
    }
    return static_cast<unsigned char*>(g_scratch_addr[dev]);
}

void run_static(const atvb_system_desc& d, const double* x, const double* y,
                const double* z, const double* q, double* fx, double* fy, double* fz,
                double* energy, cudaStream_t stream) {
    const int n = d.n_atoms;
    if (n < 1 || n > kStaticMaxAtoms)
        throw Error(ATVB_ERR_INVALID, "atvb_pair_forces_static: n_atoms must be in [1, " +
                                          std::to_string(kStaticMaxAtoms) + "]");
    if (d.box[1] != 0.0 || d.box[2] != 0.0 || d.box[3] != 0.0 || d.box[5] != 0.0 ||
        d.box[6] != 0.0 || d.box[7] != 0.0)
        throw Error(ATVB_ERR_INVALID, "atvb_pair_forces_static: box must be orthorhombic");
    if (d.precision != ATVB_FP64)
        throw Error(ATVB_ERR_INVALID, "atvb_pair_forces_static: FP64 only");
    if (d.pme_enabled)
        throw Error(ATVB_ERR_INVALID,
                    "atvb_pair_forces_static: short-range pair term only (pme_enabled must be 0)");
    if (!d.lj_enabled && !d.coul_enabled)
        throw Error(ATVB_ERR_INVALID, "atvb_pair_forces_static: no pair term enabled");
    StaticArgs a{};
    a.n = n;
    double rc = 0.0;
    a.has_lj = d.lj_enabled ? 1 : 0;
    if (a.has_lj) {
        if (!(d.lj_cutoff > 0.0))
            throw Error(ATVB_ERR_INVALID, "PairLJCut: cutoff must be positive");
        rc = d.lj_cutoff;
        const double s2 = d.lj_sigma * d.lj_sigma;
        a.lj_sig6 = s2 * s2 * s2;
        a.lj_rc2 = d.lj_cutoff * d.lj_cutoff;
        a.lj_eps4 = 4.0 * d.lj_epsilon;
        a.lj_eps24 = 24.0 * d.lj_epsilon;
        const double r2inv = 1.0 / a.lj_rc2;
        const double r6inv = r2inv * r2inv * r2inv * a.lj_sig6;
        a.lj_shift = 4.0 * d.lj_epsilon * (r6inv * r6inv - r6inv);
    }
    a.has_coul = d.coul_enabled ? 1 : 0;
    if (a.has_coul) {
        if (!(d.coul_alpha > 0.0) || !(d.coul_cutoff > 0.0))
            throw Error(ATVB_ERR_INVALID, "CoulLong: alpha and cutoff must be positive");
        rc = d.coul_cutoff > rc ? d.coul_cutoff : rc;
        a.c_rc2 = d.coul_cutoff * d.coul_cutoff;
        a.c_alpha = d.coul_alpha;
        a.c_alpha2 = d.coul_alpha * d.coul_alpha;
    }
    long long cells = 1;
    const double L[3] = {d.box[0], d.box[4], d.box[8]};
    for (int k = 0; k < 3; ++k) {
        if (!(L[k] > 2.0 * rc))
            throw Error(ATVB_ERR_INVALID,
                        "atvb_pair_forces_static: every box edge must exceed twice the cutoff");
        const double ncd = L[k] / rc;
        a.nc[k] = ncd > (double)kStaticMaxCells ? kStaticMaxCells : (int)ncd;
        a.L[k] = L[k];
        a.halfL[k] = 0.5 * L[k];
        a.cinv[k] = a.nc[k] / L[k];
        cells *= a.nc[k];
    }
    if (cells > kStaticMaxCells)
        throw Error(ATVB_ERR_INVALID, "atvb_pair_forces_static: more than " +
                                          std::to_string(kStaticMaxCells) +
                                          " cells (box too large for the cutoff)");
    a.ncell = (int)cells;
    if (!x || !y || !z || !fx || !fy || !fz || (d.coul_enabled && !q))
        throw Error(ATVB_ERR_INVALID, "atvb_pair_forces_static: NULL array");
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    unsigned char* base = static_scratch(dev);
    a.count = reinterpret_cast<int*>(base + kOffCount);
    a.start = reinterpret_cast<int*>(base + kOffStart);
    a.cell = reinterpret_cast<int*>(base + kOffCell);
    a.slot = reinterpret_cast<int*>(base + kOffSlot);
    a.sidx = reinterpret_cast<int*>(base + kOffIdx);
    a.pos = reinterpret_cast<double4*>(base + kOffPos);
    a.esum = reinterpret_cast<unsigned long long*>(base + kOffEnergy);
    a.tmp = reinterpret_cast<int*>(base + kOffTmp);
    a.x = x;
    a.y = y;
    a.z = z;
    a.q = q;
    a.fx = fx;
    a.fy = fy;
    a.fz = fz;
    a.energy = energy;
    const int ab = (n + 255) / 256;
    const int cb = (a.ncell + 255) / 256;
    k_static_zero<<<cb, 256, 0, stream>>>(a);
    k_static_bin<<<ab, 256, 0, stream>>>(a);
    k_static_scan<<<1, 1024, 0, stream>>>(a);
    k_static_scatter<<<ab, 256, 0, stream>>>(a);
    k_static_rank<<<ab, 256, 0, stream>>>(a);
    k_static_forces<<<ab, 256, 0, stream>>>(a);
    if (energy)
        k_static_energy<<<1, 32, 0, stream>>>(a);
    cuda_check(cudaGetLastError(), "atvb_pair_forces_static launch");
}

} // namespace
} // namespace atvb

extern "C" int atvb_pair_forces_static(const atvb_system_desc* desc, const double* x,
                                       const double* y, const double* z, const double* q,
                                       double* fx, double* fy, double* fz,
                                       double* energy, void* stream) {
    try {
        if (!desc)
            throw atvb::Error(ATVB_ERR_INVALID, "desc is NULL");
        atvb::run_static(*desc, x, y, z, q, fx, fy, fz, energy,
                         static_cast<cudaStream_t>(stream));
        atvb::g_last_error.clear();
        return ATVB_OK;
    } catch (const atvb::Error& e) {
        atvb::g_last_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        atvb::g_last_error = e.what();
        return ATVB_ERR_INVALID;
    }
}
