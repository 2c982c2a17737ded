// K1: cell list by integer cell sort, one CTA per system (sm_100a).
//
// Replaces the brute-force O(N^2) minimum-image search of the reference force loops
// (potentials/metal/Field.cpp:381-414, potentials/pair/Field.cpp:730-760) with a cell
// list whose neighbour set is the reference criterion: j != i, minimum image,
// rsq <= rc^2 (potentials/metal/NbrListPBC.cpp:41-125).
//
// Per system (one CTA):
//   1. wrap positions into the minimum-image cell in place, in FP64
//      (Field::resetSimulationCellMinImage, metal/Field.cpp:1894-1920);
//   2. integer cell key per atom, counts by shared-memory atomics;
//   3. exclusive scan -> cell_start;
//   4. scatter, then a rank sort inside every cell by original atom index, so the
//      sorted order (and every FP64 sum that follows it) is deterministic;
//   5. sorted double4 positions (w = charge or species label) and the work items
//      (<= kHomeChunk home atoms of one cell) of the pair kernels.
#include "akmc_internal.h"

namespace akmc {

AKMC_CHECKS_FILE(cells)

namespace {

// Longest cell whose atom list the in-cell rank sort keeps in shared memory.
constexpr int kSegCap = 256;

__device__ __forceinline__ void set_status(int* st, int code)
{
    atomicCAS(st, 0, code);
}

// In-place exclusive scan of v[0..len) by a whole CTA; returns the total.
__device__ int block_exclusive_scan(int* v, int len, int* warp_sums)
{
    const int tid = threadIdx.x, nt = blockDim.x;
    const int per = (len + nt - 1) / nt;
    const int b = tid * per;
    const int e = min(b + per, len);
    int local = 0;
    for (int k = b; k < e; k++) local += v[k];
    // warp inclusive scan of the per-thread sums
    int x = local;
    const int lane = tid & 31, warp = tid >> 5;
    #pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int nw = (nt + 31) >> 5;
        int w = lane < nw ? warp_sums[lane] : 0;
        #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        warp_sums[lane] = w;          // inclusive warp prefix
    }
    __syncthreads();
    int run = x - local + (warp > 0 ? warp_sums[warp - 1] : 0);
    for (int k = b; k < e; k++) {
        int c = v[k];
        v[k] = run;
        run += c;
    }
    int total = warp_sums[((nt + 31) >> 5) - 1];
    __syncthreads();
    return total;
}

// Shared memory of one cell-sort CTA.
struct CellShared {
    int* cnt;                         // [ncell] counts, offsets, item counts (dynamic)
    int* warp_sums;                   // [32]
    int (*seg)[kSegCap];              // [warps][kSegCap] in-cell rank sort
    int* items;                       // work items of the system just ordered
    int* base;                        // queue offset (chunks, then items)
    double* move;                     // [warps] displacement maxima
};

// Queue the atom chunks of system s (n atoms) for the list kernels.
__device__ void queue_chunks(const BatchDev& b, int s, int n, const CellShared& sh)
{
    if (!b.chunks) return;
    const int nch = (n + kChunkAtoms - 1) / kChunkAtoms;
    if (threadIdx.x == 0) *sh.base = atomicAdd(&b.counters[1], nch);
    __syncthreads();
    for (int k = threadIdx.x; k < nch; k += blockDim.x) b.chunks[*sh.base + k] = make_int2(s, k * kChunkAtoms);
    __syncthreads();
}

// Steps 1-2 for the atoms [a0, a0 + n) of a system of geometry g: wrap in place in FP64 (a
// non-finite coordinate sets *st and becomes 0); with keys, the integer cell key, the slot
// inside the cell and the cell counts in sh.cnt (zeroed by the caller); with ref, the
// largest squared minimum-image displacement of this thread's atoms from ref ([n][3],
// original order).  Returns this thread's displacement maximum.
__device__ double wrap_system(const BatchDev& b, double* pos, int* st, const SysGeom& g, int a0, int n,
                              bool keys, const double* ref, const CellShared& sh)
{
    const int nc0 = g.nc[0], nc1 = g.nc[1], nc2 = g.nc[2];
    double move2 = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double* p = pos + 3 * (size_t)(a0 + i);
        double x = p[0], y = p[1], z = p[2];
        if (!(isfinite(x) && isfinite(y) && isfinite(z))) {
            set_status(st, AKMC_ERR_NONFINITE);
            x = y = z = 0.0;
        }
        double u = x * g.invL[0], v = y * g.invL[1], w = z * g.invL[2];
        u -= rint(u);
        v -= rint(v);
        w -= rint(w);
        x = u * g.L[0];
        y = v * g.L[1];
        z = w * g.L[2];
        p[0] = x;
        p[1] = y;
        p[2] = z;
        if (ref) {
            const double* r = ref + 3 * (size_t)i;
            double dx = x - r[0], dy = y - r[1], dz = z - r[2];
            dx -= g.L[0] * rint(dx * g.invL[0]);
            dy -= g.L[1] * rint(dy * g.invL[1]);
            dz -= g.L[2] * rint(dz * g.invL[2]);
            move2 = fmax(move2, dx * dx + dy * dy + dz * dz);
        }
        if (keys) {
            int cx = (int)floor((u + 0.5) * nc0);
            int cy = (int)floor((v + 0.5) * nc1);
            int cz = (int)floor((w + 0.5) * nc2);
            cx = min(max(cx, 0), nc0 - 1);
            cy = min(max(cy, 0), nc1 - 1);
            cz = min(max(cz, 0), nc2 - 1);
            const int key = (cz * nc1 + cy) * nc0 + cx;
            b.keys[a0 + i] = key;
            b.slots[a0 + i] = atomicAdd(&sh.cnt[key], 1);
        }
    }
    return move2;
}

// The CTA's maximum of a per-thread value >= 0, in every thread.
__device__ double cta_max(double v, const CellShared& sh)
{
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) sh.move[threadIdx.x >> 5] = v;
    __syncthreads();
    double m = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = fmax(m, sh.move[w]);
    __syncthreads();
    return m;
}

// Sorted positions of a system whose order is kept (EAM list reuse: w = species label).
__device__ void refresh_sorted(const BatchDev& b, const double* pos, int a0, int n)
{
    for (int d = threadIdx.x; d < n; d += blockDim.x) {
        const int orig = b.perm[a0 + d];
        if (AKMC_BAD(orig < a0 || orig >= a0 + n, 1, orig)) continue;
        const double* p = pos + 3 * (size_t)orig;
        b.spos[a0 + d] = make_double4(p[0], p[1], p[2], (double)b.label[orig]);
    }
}

// Steps 3-5 for system s from the keys, slots and counts of wrap_system: cell offsets,
// scatter, rank sort inside cells, perm / sorted positions / labels, the work items of the
// cell-scan passes and their queue entries.
__device__ void order_system(const BatchDev& b, const double* pos, int family, int s, const SysGeom& g,
                             const CellShared& sh, int* st_sys)
{
    const int n = g.n_atoms, a0 = g.atom_begin;
    const int ncell = g.nc[0] * g.nc[1] * g.nc[2];
    const int tid = threadIdx.x, nt = blockDim.x;
    int* sh_cnt = sh.cnt;
    __syncthreads();                  // every count is in

    // 3. cell offsets
    block_exclusive_scan(sh_cnt, ncell, sh.warp_sums);
    for (int c = tid; c < ncell; c += nt) b.cell_start[g.cell_begin + c] = a0 + sh_cnt[c];
    __syncthreads();

    // 4a. scatter (slot order is arbitrary: atomics)
    for (int i = tid; i < n; i += nt) {
        const int key = b.keys[a0 + i];
        if (AKMC_BAD(key < 0 || key >= ncell, 4, key)) continue;
        const int at = sh_cnt[key] + b.slots[a0 + i];
        if (AKMC_BAD(at < 0 || at >= n, 5, at)) continue;
        b.order[a0 + at] = i;
    }
    __syncthreads();

    // 4b-5. rank sort inside each cell (warp per cell), sorted positions
    const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    for (int c = warp; c < ncell; c += nw) {
        const int st = sh_cnt[c];
        const int en = (c + 1 < ncell) ? sh_cnt[c + 1] : n;
        const int len = en - st;
        const int* seg = b.order + a0 + st;
        // cells up to kSegCap atoms rank against a shared-memory copy of their list
        const bool in_smem = len <= kSegCap;
        if (in_smem) {
            for (int e = lane; e < len; e += 32) sh.seg[warp][e] = seg[e];
            __syncwarp();
        }
        const int* sg = in_smem ? sh.seg[warp] : seg;
        for (int e = lane; e < len; e += 32) {
            const int me = sg[e];
            int rank = 0;
            for (int m = 0; m < len; m++) rank += (sg[m] < me);
            const int dst = a0 + st + rank;
            if (AKMC_BAD(rank >= len || me < 0 || me >= n, 3, me)) continue;
            const int orig = a0 + me;
            b.perm[dst] = orig;
            const double* p = pos + 3 * (size_t)orig;
            int lab = b.label[orig];
            if (b.label_check > 0 && (unsigned)lab >= (unsigned)b.label_check) {
                set_status(st_sys, AKMC_ERR_ARG);    // never index a table with it
                lab = 0;
            }
            const double wv = (family == AKMC_FAMILY_IONIC) ? b.charge[orig] : (double)lab;
            b.spos[dst] = make_double4(p[0], p[1], p[2], wv);
            b.slabel[dst] = lab;
        }
        __syncwarp();
    }
    __syncthreads();

    // 5b. work items: ceil(len / home_chunk) per cell, scanned into this system's
    // window.  Cell lengths come from cell_start in global memory (written above by
    // this CTA), so the shared array can be overwritten with item counts.
    const int hc = g.home_chunk > 0 ? g.home_chunk : (b.home_chunk > 0 ? b.home_chunk : kHomeChunk);
    for (int c = tid; c < ncell; c += nt) {
        const int st = b.cell_start[g.cell_begin + c];
        const int en = (c + 1 < ncell) ? b.cell_start[g.cell_begin + c + 1] : a0 + n;
        sh_cnt[c] = (en - st + hc - 1) / hc;
    }
    __syncthreads();
    const int total_items = block_exclusive_scan(sh_cnt, ncell, sh.warp_sums);
    if (tid == 0) *sh.items = total_items;
    __syncthreads();
    for (int c = tid; c < ncell; c += nt) {
        const int st = b.cell_start[g.cell_begin + c];
        const int en = (c + 1 < ncell) ? b.cell_start[g.cell_begin + c + 1] : a0 + n;
        int k = sh_cnt[c];
        for (int f = st; f < en; f += hc, k++) {
            WorkItem it;
            it.cell = g.cell_begin + c;
            it.first = f;
            it.count = min(hc, en - f);
            it.sys = s;
            b.items[g.item_base + k] = it;
        }
    }
    if (tid == 0) {
        b.n_items[s] = *sh.items;
        if (b.work) *sh.base = atomicAdd(&b.counters[0], *sh.items);      // queue this system's items
    }
    __syncthreads();
    if (b.work)
        for (int k = tid; k < *sh.items; k += nt) b.work[*sh.base + k] = g.item_base + k;
    __syncthreads();
}

// One system of a call (status already reset): chunks, wrap, then either the kept order
// (list reuse) or a full sort with its work items.
__device__ void sort_system(const BatchDev& b, double* pos, int* status, int family, int s,
                            const CellShared& sh)
{
    const SysGeom g = b.geom[s];
    const int n = g.n_atoms, a0 = g.atom_begin;
    const int ncell = g.nc[0] * g.nc[1] * g.nc[2];
    const int tid = threadIdx.x, nt = blockDim.x;
    if (!system_active(b, s)) {            // skipped system: no items for the pair kernels
        if (tid == 0) b.n_items[s] = 0;
        return;
    }
    queue_chunks(b, s, n, sh);
    for (int c = tid; c < ncell; c += nt) sh.cnt[c] = 0;
    __syncthreads();
    // with a skin and a list from an earlier call: largest displacement since its build
    const bool check_list = b.skin > 0.0 && b.list_ok[s] != 0;
    const double move2 = wrap_system(b, pos, &status[s], g, a0, n, true,
                                     check_list ? b.ref_pos + 3 * (size_t)a0 : nullptr, sh);
    __syncthreads();
    if (check_list && cta_max(move2, sh) <= 0.25 * b.skin * b.skin) {
        // every atom within skin/2 of its build position: keep the sorted order and the
        // list, refresh the sorted positions; no work items for the cell-scan pass
        refresh_sorted(b, pos, a0, n);
        if (tid == 0) {
            b.n_items[s] = 0;
            b.list_mode[s] = 2;
        }
        return;
    }
    order_system(b, pos, family, s, g, sh, &status[s]);
    if (b.skin > 0.0) {
        // this call builds the list: remember the positions it is built at
        for (int i = tid; i < n; i += nt) {
            const double* p = pos + 3 * (size_t)(a0 + i);
            double* r = b.ref_pos + 3 * (size_t)(a0 + i);
            r[0] = p[0];
            r[1] = p[1];
            r[2] = p[2];
        }
        if (tid == 0) {
            b.list_mode[s] = 1;
            b.list_ok[s] = 1;
        }
    } else if (b.list_mode && tid == 0) {
        b.list_mode[s] = 0;
    }
    __syncthreads();
}

#define CELL_SHARED_DECL                                                        \
    extern __shared__ int sh_cnt[];                                             \
    __shared__ int warp_sums[32];                                               \
    __shared__ int s_seg[kCellThreads / 32][kSegCap];                           \
    __shared__ int s_items, s_base;                                             \
    __shared__ double s_move[kCellThreads / 32];                                \
    const CellShared sh{sh_cnt, warp_sums, s_seg, &s_items, &s_base, s_move}

__global__ void __launch_bounds__(kCellThreads)
cell_sort_kernel(BatchDev b, double* __restrict__ pos, int* __restrict__ status, int family)
{
    CELL_SHARED_DECL;
    pdl_wait();            // the caller's positions and the previous call's readers
    pdl_release();
    const int s = blockIdx.x;
    if (threadIdx.x == 0) status[s] = AKMC_OK;     // each call starts from a clean status
    sort_system(b, pos, status, family, s, sh);
}

// One CTA per image group k (systems m * n_groups + k).  With an EAM list and a skin the
// images that run share one order and one list: the largest displacement of any of them
// from the group's build positions decides between keeping both (every running image
// refreshes its sorted positions) and a rebuild from the first running image (the
// "builder": sorted and given the cell-scan work items that write the list at image 0's
// rows; the other images take its order).  Without a list every running image is sorted on
// its own.
__global__ void __launch_bounds__(kCellThreads)
cell_sort_images_kernel(BatchDev b, double* __restrict__ pos, int* __restrict__ status, int family)
{
    CELL_SHARED_DECL;
    pdl_wait();
    pdl_release();
    const int k = blockIdx.x, W = b.n_groups, NI = b.n_images;
    const int tid = threadIdx.x, nt = blockDim.x;
    int builder = -1;
    for (int m = NI - 1; m >= 0; m--) {
        const int s = m * W + k;
        if (tid == 0) {
            status[s] = AKMC_OK;
            b.n_items[s] = 0;
        }
        if (system_active(b, s)) builder = m;
    }
    if (builder < 0) return;
    if (!(b.skin > 0.0 && b.nbr)) {
        for (int m = 0; m < NI; m++) sort_system(b, pos, status, family, m * W + k, sh);
        return;
    }
    const SysGeom g0 = b.geom[k];
    const int n = g0.n_atoms;
    const int ncell = g0.nc[0] * g0.nc[1] * g0.nc[2];
    for (int m = 0; m < NI; m++)
        if (system_active(b, m * W + k)) queue_chunks(b, m * W + k, n, sh);
    for (int c = tid; c < ncell; c += nt) sh.cnt[c] = 0;
    __syncthreads();
    const bool have = b.list_ok[k] != 0;
    const double* ref = have ? b.ref_pos + 3 * (size_t)g0.atom_begin : nullptr;
    double move2 = 0.0;
    for (int m = 0; m < NI; m++) {
        const int s = m * W + k;
        if (!system_active(b, s)) continue;
        const int am = b.geom[s].atom_begin;
        move2 = fmax(move2, wrap_system(b, pos, &status[s], g0, am, n, m == builder, ref, sh));
    }
    __syncthreads();
    const double mx = cta_max(move2, sh);
    if (have && mx <= 0.25 * b.skin * b.skin) {
        for (int m = 0; m < NI; m++) {
            const int s = m * W + k;
            if (!system_active(b, s)) continue;
            refresh_sorted(b, pos, b.geom[s].atom_begin, n);
            if (tid == 0) b.list_mode[s] = 2;
        }
        return;
    }
    const int sb = builder * W + k;
    const SysGeom gb = b.geom[sb];
    order_system(b, pos, family, sb, gb, sh, &status[sb]);
    // the other images take the builder's order (their sorted positions if they run)
    for (int m = 0; m < NI; m++) {
        if (m == builder) continue;
        const int s = m * W + k;
        const int am = b.geom[s].atom_begin, shift = am - gb.atom_begin;
        const bool run = system_active(b, s);
        for (int d = tid; d < n; d += nt) {
            const int orig = b.perm[gb.atom_begin + d] + shift;
            if (AKMC_BAD(orig < am || orig >= am + n, 2, orig)) continue;
            b.perm[am + d] = orig;
            b.slabel[am + d] = b.slabel[gb.atom_begin + d];
            if (run) {
                const double* p = pos + 3 * (size_t)orig;
                b.spos[am + d] = make_double4(p[0], p[1], p[2], (double)b.label[orig]);
            }
        }
        if (run && tid == 0) b.list_mode[s] = 2;
    }
    // the build positions (original order) at image 0's rows
    for (int i = tid; i < n; i += nt) {
        const double* p = pos + 3 * (size_t)(gb.atom_begin + i);
        double* r = b.ref_pos + 3 * (size_t)(g0.atom_begin + i);
        r[0] = p[0];
        r[1] = p[1];
        r[2] = p[2];
    }
    if (tid == 0) {
        b.list_mode[sb] = 1;
        b.list_ok[k] = 1;
    }
}

}  // namespace

// Whole-cell ionic batches (mixed precision): the pair kernel takes every atom of a system as
// a candidate of every other, so no cell order is needed -- one CTA per system wraps the
// positions in place (as wrap_system, the reference's s -= rint(s)) and writes the
// "sorted" arrays in the caller's order (perm = identity).
__global__ void __launch_bounds__(kCellThreads)
wrap_whole_cell_kernel(BatchDev b, double* __restrict__ pos, int* __restrict__ status)
{
    pdl_wait();            // the caller's positions and the previous call's readers
    pdl_release();
    const int s = blockIdx.x;
    if (threadIdx.x == 0) status[s] = AKMC_OK;     // each call starts from a clean status
    __syncthreads();
    if (!system_active(b, s)) return;
    const SysGeom g = b.geom[s];
    for (int i = threadIdx.x; i < g.n_atoms; i += blockDim.x) {
        const int a = g.atom_begin + i;
        double* p = pos + 3 * (size_t)a;
        double x = p[0], y = p[1], z = p[2];
        if (!(isfinite(x) && isfinite(y) && isfinite(z))) {
            set_status(&status[s], AKMC_ERR_NONFINITE);
            x = y = z = 0.0;
        }
        double u = x * g.invL[0], v = y * g.invL[1], w = z * g.invL[2];
        u -= rint(u);
        v -= rint(v);
        w -= rint(w);
        x = u * g.L[0];
        y = v * g.L[1];
        z = w * g.L[2];
        p[0] = x;
        p[1] = y;
        p[2] = z;
        b.spos[a] = make_double4(x, y, z, b.charge[a]);
        b.slabel[a] = b.label[a];
        b.perm[a] = a;
    }
}

cudaError_t launch_cell_sort(const BatchDev& b, double* pos, int* status, int family,
                             int smem_cells, cudaStream_t st)
{
    const size_t smem = sizeof(int) * (size_t)smem_cells;
    if (b.n_images > 1)
        return launch_pdl(cell_sort_images_kernel, dim3(b.n_groups), dim3(kCellThreads), smem, st, b, pos, status,
                          family);
    return launch_pdl(cell_sort_kernel, dim3(b.nsys), dim3(kCellThreads), smem, st, b, pos, status, family);
}

cudaError_t launch_wrap_whole_cell(const BatchDev& b, double* pos, int* status, cudaStream_t st)
{
    return launch_pdl(wrap_whole_cell_kernel, dim3(b.nsys), dim3(kCellThreads), 0, st, b, pos, status);
}

cudaError_t configure_cell_kernels()
{
    cudaError_t e = cudaFuncSetAttribute(cell_sort_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(sizeof(int) * kMaxCellsPerSystem));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(cell_sort_images_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(sizeof(int) * kMaxCellsPerSystem));
}

}  // namespace akmc
