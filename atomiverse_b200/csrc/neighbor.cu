// neighbor.cu -- cell binning, cell-ordered permutation and the Verlet list.
//
// Semantics follow the reference CPU cell list
// (src/cpu/neighbor/cell_list.cpp:83-314 grid/stencil/binning and :743-895
// list): a pair {i, j} is listed iff its minimum-image separation, computed
// in FP64 on the rebuild-time coordinates, satisfies r^2 < (cutoff+skin)^2.
// Every product and sum of that test is rounded separately (__dmul_rn /
// __dadd_rn), which is exactly the arithmetic of the FP64 oracle, so the
// pair set equals the oracle's bit for bit.  The list itself is a FULL list
// (each pair stored in both rows) in row-major ELL form with a fixed row
// capacity, so the force kernel needs no atomics and sums every row in a
// fixed order.
#include "atvb_common.cuh"
#include "atvb_kernels.cuh"

namespace atvb {

// Stage 1: cell of every atom (original order) and its arrival slot.
__global__ void k_cell_count(const Item* items, int nitems,
                             const SysParams* sp) {
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        if (!P.st->rebuild)
            continue;
        const int i = item.begin + threadIdx.x;
        if (i >= P.n)
            continue;
        const double p[3] = {P.x[i], P.y[i], P.z[i]};
        int c[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            int cd = (int)floor(p[d] * P.cs_inv[d]);
            cd = cd < 0 ? 0 : (cd > P.nc[d] - 1 ? P.nc[d] - 1 : cd);
            c[d] = cd;
        }
        const int cell = (c[0] * P.nc[1] + c[1]) * P.nc[2] + c[2];
        P.cell_of[i] = cell;
        P.slot[i] = atomicAdd(&P.cell_count[cell], 1);
    }
}

// Stage 2: exclusive scan of the cell counts, one block per system.
__global__ void k_cell_scan(const int* sys_list, const SysParams* sp) {
    const SysParams& P = sp[sys_list[blockIdx.x]];
    if (!P.st->rebuild)
        return;
    __shared__ int warp_tot[32];
    __shared__ int carry;
    if (threadIdx.x == 0)
        carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int base = 0; base < P.ncell; base += blockDim.x) {
        const int c = base + threadIdx.x;
        const int v = c < P.ncell ? P.cell_count[c] : 0;
        int incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o)
                incl += t;
        }
        if (lane == 31)
            warp_tot[w] = incl;
        __syncthreads();
        if (w == 0) {
            const int nw = blockDim.x >> 5;
            int t = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o)
                    t += u;
            }
            if (lane < nw)
                warp_tot[lane] = t; // inclusive over warps
        }
        __syncthreads();
        const int before = (w > 0 ? warp_tot[w - 1] : 0) + carry;
        if (c < P.ncell) {
            P.cell_start[c] = before + incl - v;
            P.cell_count[c] = 0; // ready for the next rebuild
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1)
            carry = before + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0)
        P.cell_start[P.ncell] = carry;
}

// Stage 3: scatter atom ids into their cells.
__global__ void k_cell_scatter(const Item* items, int nitems,
                               const SysParams* sp) {
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        if (!P.st->rebuild)
            continue;
        const int i = item.begin + threadIdx.x;
        if (i >= P.n)
            continue;
        P.perm[P.cell_start[P.cell_of[i]] + P.slot[i]] = i;
    }
}

// Stage 4: order each cell by original index, so the permutation (and with
// it every later summation order) is independent of atomic arrival order.
__global__ void k_cell_sort(const Item* citems, int nitems,
                            const SysParams* sp) {
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = citems[it];
        const SysParams& P = sp[item.sys];
        if (!P.st->rebuild)
            continue;
        const int c = item.begin + threadIdx.x;
        if (c >= P.ncell)
            continue;
        const int a = P.cell_start[c], b = P.cell_start[c + 1];
        for (int k = a + 1; k < b; ++k) {
            const int v = P.perm[k];
            int m = k - 1;
            while (m >= a && P.perm[m] > v) {
                P.perm[m + 1] = P.perm[m];
                --m;
            }
            P.perm[m + 1] = v;
        }
    }
}

// Stage 5: inverse permutation, sorted positions, reference positions.
__global__ void k_permute(const Item* items, int nitems, const SysParams* sp) {
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        if (!P.st->rebuild)
            continue;
        const int s = item.begin + threadIdx.x;
        if (s >= P.n)
            continue;
        const int i = P.perm[s];
        P.rank[i] = s;
        P.cellS[s] = P.cell_of[i];
        const double x = P.x[i], y = P.y[i], z = P.z[i], q = P.q[i];
        P.posd4[s] = make_double4(x, y, z, q);
        int4 v;
        v.x = (int)pos_fix(x, P.fix_scale[0]);
        v.y = (int)pos_fix(y, P.fix_scale[1]);
        v.z = (int)pos_fix(z, P.fix_scale[2]);
        v.w = 0;
        P.lpos[s] = v;
        if (P.prec == kMixed) {
            v.w = __float_as_int((float)q);
            reinterpret_cast<int4*>(P.pos4)[s] = v;
        }
        else {
            const double xx[3] = {x, y, z};
            reinterpret_cast<double4*>(P.pos4)[s] = pack_pos64(xx, P.fix64_scale, q);
        }
        if (P.ntypes)
            P.stype[s] = (unsigned char)P.type[i];
        P.xr[i] = x;
        P.yr[i] = y;
        P.zr[i] = z;
    }
}

// Exact FP64 pair-set test (same rounding as the oracle built with
// -ffp-contract=off): branchy single-wrap minimum image
// (cell_list.h:214-227), then ((dx*dx + dy*dy) + dz*dz).
ATVB_DEV double exact_r2(const double4& a, const double4& b, const double* L,
                         const double* halfL) {
    double d[3] = {__dadd_rn(a.x, -b.x), __dadd_rn(a.y, -b.y),
                   __dadd_rn(a.z, -b.z)};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (d[k] > halfL[k])
            d[k] = __dadd_rn(d[k], -L[k]);
        else if (d[k] < -halfL[k])
            d[k] = __dadd_rn(d[k], L[k]);
    }
    return __dadd_rn(__dadd_rn(__dmul_rn(d[0], d[0]), __dmul_rn(d[1], d[1])),
                     __dmul_rn(d[2], d[2]));
}

// The sorted atoms of stencil column `col` around cell (cx, cy, cz): at most
// two contiguous runs [a0, a0 + l0) and [a1, a1 + l1) (two when the z range
// wraps).  Offsets along an axis stay within one period of the cell index,
// so one conditional add or subtract wraps them (also on an aliased axis,
// whose offsets are absolute cell indices).
ATVB_DEV void column_runs(int nc0, int nc1, int nc2, const int* __restrict__ cstart, int4 col,
                          int cx, int cy, int cz, int& a0, int& l0, int& a1, int& l1) {
    int xx = cx + col.x;
    xx += xx < 0 ? nc0 : (xx >= nc0 ? -nc0 : 0);
    int yy = cy + col.y;
    yy += yy < 0 ? nc1 : (yy >= nc1 ? -nc1 : 0);
    const int base = (xx * nc1 + yy) * nc2;
    int lo0, hi0, lo1 = 0, hi1 = -1;
    if (col.z < 0) {
        lo0 = base;
        hi0 = base + nc2 - 1;
    } else {
        const int z0 = cz - col.z, z1 = cz + col.z;
        if (z0 < 0) {
            lo0 = base + z0 + nc2;
            hi0 = base + nc2 - 1;
            lo1 = base;
            hi1 = base + z1;
        } else if (z1 >= nc2) {
            lo0 = base + z0;
            hi0 = base + nc2 - 1;
            lo1 = base;
            hi1 = base + z1 - nc2;
        } else {
            lo0 = base + z0;
            hi0 = base + z1;
        }
    }
    a0 = cstart[lo0];
    l0 = cstart[hi0 + 1] - a0;
    if (hi1 >= lo1) {
        a1 = cstart[lo1];
        l1 = cstart[hi1 + 1] - a1;
    } else {
        a1 = 0;
        l1 = 0;
    }
}

// Special class (1: 1-2, 2: 1-3, 3: 1-4, 0: none) of sorted pair (i, j):
// a scan of i's few special partners, by original index.
ATVB_DEV unsigned special_class(const SysParams& P, int i, int j) {
    const int io = P.perm[i], jo = P.perm[j];
    for (int q = P.sp_first[io]; q < P.sp_first[io + 1]; ++q)
        if (P.sp_j[q] == jo)
            return P.sp_cls[q];
    return 0u;
}

// Stage 6 (items of kListChunk cells): one warp per cell.  Every atom of a
// cell has the same stencil, so the warp resolves the stencil columns once
// (up to 32 at a time, one per lane, into runs of sorted atoms laid end to
// end by a warp prefix sum), loads each window of 32 consecutive candidates
// once, and tests that window against every atom of the cell in turn,
// appending hits to that atom's row with a ballot.  Rows list candidates in
// column order.  Candidates are screened in FP32 on the fixed-point
// positions (16 bytes per candidate, exact integer minimum image); only
// those whose FP32 distance lies within the error band of
// r^2 = (cutoff + skin)^2 take the exact FP64 test, so the listed set is
// exactly the FP64 one.
constexpr int kCellAtomsWarp = 32; // atoms of one cell handled per pass

__global__ void __launch_bounds__(256)
    k_build_list(const Item* items, int nitems, const SysParams* sp) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    __shared__ int4 sq[8][kCellAtomsWarp];
    __shared__ float4 sr[8][kCellAtomsWarp];
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Item item = items[it];
        const SysParams& P = sp[item.sys];
        if (!P.st->rebuild)
            continue;
        const int c = item.begin + warp;
        if (c >= P.ncell)
            continue; // warp-uniform
        // every field the loops use, read once: the row stores below could
        // alias SysParams as far as the compiler knows, and would force a
        // reload of any field read after them
        const int nc0 = P.nc[0], nc1 = P.nc[1], nc2 = P.nc[2];
        int* __restrict__ nbr = P.nbr;
        const bool has_sp = P.has_special != 0;
        const double L[3] = {P.L[0], P.L[1], P.L[2]};
        const double hL[3] = {P.halfL[0], P.halfL[1], P.halfL[2]};
        const double rl2 = P.rlist2;
        const int cap = P.cap, ncol = P.ncol;
        const int4* __restrict__ cols = P.cols;
        const int* __restrict__ cstart = P.cell_start;
        const double4* __restrict__ pos = P.posd4;
        const int4* __restrict__ lp = P.lpos;
        const float sx = P.Lf_fix[0], sy = P.Lf_fix[1], sz = P.Lf_fix[2];
        const float blo = P.lband_lo, bhi = P.lband_hi;
        const float flo = P.fband_lo, fhi = P.fband_hi;
        const bool local = P.lframe_ok != 0;
        const int cz = c % nc2, cy = (c / nc2) % nc1, cx = c / (nc1 * nc2);
        const int cs = cstart[c], ce = cstart[c + 1];
        for (int i0 = cs; i0 < ce; i0 += kCellAtomsWarp) {
            const int ni = min(kCellAtomsWarp, ce - i0);
            const int4 org = lp[i0];
            __syncwarp();
            if (lane < ni) {
                const int4 q = lp[i0 + lane];
                sq[warp][lane] = q;
                sr[warp][lane] = make_float4((float)(int)((unsigned)q.x - (unsigned)org.x) * sx,
                                             (float)(int)((unsigned)q.y - (unsigned)org.y) * sy,
                                             (float)(int)((unsigned)q.z - (unsigned)org.z) * sz,
                                             0.0f);
            }
            __syncwarp();
            int cnt = 0; // row length of atom i0 + lane
            for (int c0 = 0; c0 < ncol; c0 += 32) {
                int a0 = 0, l0 = 0, a1 = 0, l1 = 0;
                if (c0 + lane < ncol)
                    column_runs(nc0, nc1, nc2, cstart, cols[c0 + lane], cx, cy, cz, a0, l0,
                                a1, l1);
                const int tot = l0 + l1;
                int incl = tot;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(full, incl, o);
                    if (lane >= o)
                        incl += t;
                }
                const int excl = incl - tot;
                const int total = __shfl_sync(full, incl, 31);
                for (int b = 0; b < total; b += 32) {
                    const int t = b + lane;
                    // owner column: the first lane whose inclusive sum exceeds t
                    int own = 0;
#pragma unroll
                    for (int step = 16; step > 0; step >>= 1) {
                        const int probe = __shfl_sync(full, incl, own + step - 1);
                        if (probe <= t)
                            own += step;
                    }
                    own &= 31;
                    const int o = t - __shfl_sync(full, excl, own);
                    const int oa0 = __shfl_sync(full, a0, own);
                    const int ol0 = __shfl_sync(full, l0, own);
                    const int oa1 = __shfl_sync(full, a1, own);
                    const bool live = t < total;
                    const int j = live ? (o < ol0 ? oa0 + o : oa1 + (o - ol0)) : -1;
                    int4 qj = make_int4(0, 0, 0, 0);
                    if (live)
                        qj = lp[j];
                    if (local) {
                        // candidate in the cell-local frame (see lframe_ok)
                        const float rx = (float)(int)((unsigned)qj.x - (unsigned)org.x) * sx;
                        const float ry = (float)(int)((unsigned)qj.y - (unsigned)org.y) * sy;
                        const float rz = (float)(int)((unsigned)qj.z - (unsigned)org.z) * sz;
                        // two atoms of the cell per pass: their screens,
                        // votes and appends are independent, so their
                        // latencies overlap; an odd last atom takes the
                        // one-atom pass (sparse cells hold one atom or two)
                        int ii = 0;
                        for (; ii + 1 < ni; ii += 2) {
                            const int i1 = ii + 1;
                            const float4 ra = sr[warp][ii], rb = sr[warp][i1];
                            const float ax = ra.x - rx, ay = ra.y - ry, az = ra.z - rz;
                            const float bx = rb.x - rx, by = rb.y - ry, bz = rb.z - rz;
                            const float r2a = ax * ax + ay * ay + az * az;
                            const float r2b = bx * bx + by * by + bz * bz;
                            const bool va = live && j != i0 + ii;
                            const bool vb = live && j != i0 + i1;
                            bool ha = va && r2a < flo, hb = vb && r2b < flo;
                            const bool aa = va && !(r2a < flo) && r2a < fhi;
                            const bool ab = vb && !(r2b < flo) && r2b < fhi;
                            if (__any_sync(full, aa || ab)) { // rare: exact FP64 test
                                if (aa)
                                    ha = exact_r2(pos[i0 + ii], pos[j], L, hL) < rl2;
                                if (ab)
                                    hb = exact_r2(pos[i0 + i1], pos[j], L, hL) < rl2;
                            }
                            const unsigned ma = __ballot_sync(full, ha);
                            const unsigned mb = __ballot_sync(full, hb);
                            if (ma | mb) {
                                const int basea = __shfl_sync(full, cnt, ii);
                                const int baseb = __shfl_sync(full, cnt, i1);
                                if (ha) {
                                    const int wpos = basea + __popc(ma & lt);
                                    unsigned e = (unsigned)j;
                                    if (has_sp)
                                        e |= special_class(P, i0 + ii, j) << 30;
                                    if (wpos < cap)
                                        nbr[(size_t)(i0 + ii) * cap + wpos] = (int)e;
                                }
                                if (hb) {
                                    const int wpos = baseb + __popc(mb & lt);
                                    unsigned e = (unsigned)j;
                                    if (has_sp)
                                        e |= special_class(P, i0 + i1, j) << 30;
                                    if (wpos < cap)
                                        nbr[(size_t)(i0 + i1) * cap + wpos] = (int)e;
                                }
                                if (lane == ii)
                                    cnt += __popc(ma);
                                if (lane == i1)
                                    cnt += __popc(mb);
                            }
                        }
                        if (ii < ni) {
                            const float4 ri = sr[warp][ii];
                            const float dx = ri.x - rx, dy = ri.y - ry, dz = ri.z - rz;
                            const float r2f = dx * dx + dy * dy + dz * dz;
                            const bool valid = live && j != i0 + ii;
                            bool hit = valid && r2f < flo;
                            const bool amb = valid && !(r2f < flo) && r2f < fhi;
                            if (__any_sync(full, amb)) {
                                if (amb)
                                    hit = exact_r2(pos[i0 + ii], pos[j], L, hL) < rl2;
                            }
                            const unsigned m = __ballot_sync(full, hit);
                            if (m) {
                                const int base = __shfl_sync(full, cnt, ii);
                                if (hit) {
                                    const int wpos = base + __popc(m & lt);
                                    unsigned e = (unsigned)j;
                                    if (has_sp)
                                        e |= special_class(P, i0 + ii, j) << 30;
                                    if (wpos < cap)
                                        nbr[(size_t)(i0 + ii) * cap + wpos] = (int)e;
                                }
                                if (lane == ii)
                                    cnt += __popc(m);
                            }
                        }
                    } else {
                        // exact integer minimum image (small boxes)
                        for (int ii = 0; ii < ni; ++ii) {
                            const int4 qi = sq[warp][ii];
                            const float dx = (float)(int)((unsigned)qi.x - (unsigned)qj.x) * sx;
                            const float dy = (float)(int)((unsigned)qi.y - (unsigned)qj.y) * sy;
                            const float dz = (float)(int)((unsigned)qi.z - (unsigned)qj.z) * sz;
                            const float r2f = dx * dx + dy * dy + dz * dz;
                            const bool valid = live && j != i0 + ii;
                            bool hit = valid && r2f < blo;
                            const bool amb = valid && !(r2f < blo) && r2f < bhi;
                            if (__any_sync(full, amb)) {
                                if (amb)
                                    hit = exact_r2(pos[i0 + ii], pos[j], L, hL) < rl2;
                            }
                            const unsigned m = __ballot_sync(full, hit);
                            if (m) {
                                const int base = __shfl_sync(full, cnt, ii);
                                if (hit) {
                                    const int wpos = base + __popc(m & lt);
                                    unsigned e = (unsigned)j;
                                    if (has_sp)
                                        e |= special_class(P, i0 + ii, j) << 30;
                                    if (wpos < cap)
                                        nbr[(size_t)(i0 + ii) * cap + wpos] = (int)e;
                                }
                                if (lane == ii)
                                    cnt += __popc(m);
                            }
                        }
                    }
                }
            }
            if (lane < ni) {
                const int i = i0 + lane;
                P.nnbr[i] = cnt < cap ? cnt : cap;
                atomicMax(&P.st->max_nnbr, cnt);
                atomicAdd(&P.st->list_entries, (unsigned long long)cnt);
                if (cnt > cap) {
                    // the row is cut: pairs are missing until rows are widened
                    atomicOr(&P.st->overflow, 1);
                    atomicOr(&P.st->status, kStatusRowOverflow);
                }
            }
        }
    }
}

// Binning and the sorted repack: after these the sorted positions (pos4)
// that the PME chain reads are final, so that chain may start beside the
// list build.
void launch_sort_cells(const LaunchCfg& lc, cudaStream_t s) {
    k_cell_count<<<lc.atoms.grid, kChunk, 0, s>>>(lc.atoms.d, lc.atoms.n,
                                                   lc.sp);
    k_cell_scan<<<lc.nsys, 1024, 0, s>>>(lc.sys_list, lc.sp);
    k_cell_scatter<<<lc.atoms.grid, kChunk, 0, s>>>(lc.atoms.d, lc.atoms.n,
                                                     lc.sp);
    k_cell_sort<<<lc.cells.grid, kChunk, 0, s>>>(lc.cells.d, lc.cells.n,
                                                  lc.sp);
    k_permute<<<lc.atoms.grid, kChunk, 0, s>>>(lc.atoms.d, lc.atoms.n, lc.sp);
}

void launch_build_list(const LaunchCfg& lc, cudaStream_t s) {
    k_build_list<<<lc.list.grid, 32 * kListChunk, 0, s>>>(lc.list.d,
                                                           lc.list.n, lc.sp);
}

void launch_rebuild(const LaunchCfg& lc, cudaStream_t s) {
    launch_sort_cells(lc, s);
    launch_build_list(lc, s);
}

} // namespace atvb
