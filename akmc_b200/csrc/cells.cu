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

__global__ void __launch_bounds__(kCellThreads)
cell_sort_kernel(BatchDev b, double* __restrict__ pos, int* __restrict__ status, int family)
{
    extern __shared__ int sh_cnt[];
    __shared__ int warp_sums[32];
    __shared__ int s_seg[kCellThreads / 32][kSegCap];
    __shared__ int s_items, s_base;
    __shared__ double s_move[kCellThreads / 32];

    pdl_wait();            // the caller's positions and the previous call's readers
    pdl_release();
    const int s = blockIdx.x;
    const SysGeom g = b.geom[s];
    const int n = g.n_atoms, a0 = g.atom_begin;
    const int nc0 = g.nc[0], nc1 = g.nc[1], nc2 = g.nc[2];
    const int ncell = nc0 * nc1 * nc2;
    const int tid = threadIdx.x, nt = blockDim.x;

    if (tid == 0) status[s] = AKMC_OK;     // each call starts from a clean status
    if (!system_active(b, s)) {            // skipped system: no items for the pair kernels
        if (tid == 0) b.n_items[s] = 0;
        return;
    }
    const int nch = (n + kChunkAtoms - 1) / kChunkAtoms;
    if (b.chunks && tid == 0) s_base = atomicAdd(&b.counters[1], nch);   // this system's atom chunks
    for (int c = tid; c < ncell; c += nt) sh_cnt[c] = 0;
    __syncthreads();
    if (b.chunks)
        for (int k = tid; k < nch; k += nt) b.chunks[s_base + k] = make_int2(s, k * kChunkAtoms);

    // with a skin and a list from an earlier call: largest displacement since its build
    const bool check_list = b.skin > 0.0 && b.list_ok[s] != 0;
    double move2 = 0.0;

    // 1-2. wrap in place, cell keys, counts
    for (int i = tid; i < n; i += nt) {
        double* p = pos + 3 * (size_t)(a0 + i);
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
        if (check_list) {
            const double* r = b.ref_pos + 3 * (size_t)(a0 + i);
            double dx = x - r[0], dy = y - r[1], dz = z - r[2];
            dx -= g.L[0] * rint(dx * g.invL[0]);
            dy -= g.L[1] * rint(dy * g.invL[1]);
            dz -= g.L[2] * rint(dz * g.invL[2]);
            move2 = fmax(move2, dx * dx + dy * dy + dz * dz);
        }
        int cx = (int)floor((u + 0.5) * nc0);
        int cy = (int)floor((v + 0.5) * nc1);
        int cz = (int)floor((w + 0.5) * nc2);
        cx = min(max(cx, 0), nc0 - 1);
        cy = min(max(cy, 0), nc1 - 1);
        cz = min(max(cz, 0), nc2 - 1);
        const int key = (cz * nc1 + cy) * nc0 + cx;
        b.keys[a0 + i] = key;
        b.slots[a0 + i] = atomicAdd(&sh_cnt[key], 1);
    }
    __syncthreads();

    if (check_list) {
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) move2 = fmax(move2, __shfl_xor_sync(0xffffffffu, move2, o));
        if ((tid & 31) == 0) s_move[tid >> 5] = move2;
        __syncthreads();
        double m = 0.0;
        for (int w = 0; w < (nt >> 5); w++) m = fmax(m, s_move[w]);
        if (m <= 0.25 * b.skin * b.skin) {
            // every atom within skin/2 of its build position: keep the sorted order and the
            // list, refresh the sorted positions; no work items for the cell-scan pass
            for (int d = tid; d < n; d += nt) {
                const int orig = b.perm[a0 + d];
                const double* p = pos + 3 * (size_t)orig;
                b.spos[a0 + d] = make_double4(p[0], p[1], p[2], (double)b.label[orig]);
            }
            if (tid == 0) {
                b.n_items[s] = 0;
                b.list_mode[s] = 2;
            }
            return;
        }
    }

    // 3. cell offsets
    block_exclusive_scan(sh_cnt, ncell, warp_sums);
    for (int c = tid; c < ncell; c += nt) b.cell_start[g.cell_begin + c] = a0 + sh_cnt[c];
    __syncthreads();

    // 4a. scatter (slot order is arbitrary: atomics)
    for (int i = tid; i < n; i += nt) {
        const int key = b.keys[a0 + i];
        b.order[a0 + sh_cnt[key] + b.slots[a0 + i]] = i;
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
            for (int e = lane; e < len; e += 32) s_seg[warp][e] = seg[e];
            __syncwarp();
        }
        const int* sg = in_smem ? s_seg[warp] : seg;
        for (int e = lane; e < len; e += 32) {
            const int me = sg[e];
            int rank = 0;
            for (int m = 0; m < len; m++) rank += (sg[m] < me);
            const int dst = a0 + st + rank;
            const int orig = a0 + me;
            b.perm[dst] = orig;
            const double* p = pos + 3 * (size_t)orig;
            const double wv = (family == AKMC_FAMILY_IONIC) ? b.charge[orig] : (double)b.label[orig];
            b.spos[dst] = make_double4(p[0], p[1], p[2], wv);
            b.slabel[dst] = b.label[orig];
        }
        __syncwarp();
    }
    __syncthreads();

    // 5b. work items: ceil(len / home_chunk) per cell, scanned into this system's
    // window.  Cell lengths come from cell_start in global memory (written above by
    // this CTA), so the shared array can be overwritten with item counts.
    const int hc = b.home_chunk > 0 ? b.home_chunk : kHomeChunk;
    for (int c = tid; c < ncell; c += nt) {
        const int st = b.cell_start[g.cell_begin + c];
        const int en = (c + 1 < ncell) ? b.cell_start[g.cell_begin + c + 1] : a0 + n;
        sh_cnt[c] = (en - st + hc - 1) / hc;
    }
    __syncthreads();
    const int total_items = block_exclusive_scan(sh_cnt, ncell, warp_sums);
    if (tid == 0) s_items = total_items;
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
        b.n_items[s] = s_items;
        if (b.work) s_base = atomicAdd(&b.counters[0], s_items);        // queue this system's items
    }
    if (b.work) {
        __syncthreads();
        for (int k = tid; k < s_items; k += nt) b.work[s_base + k] = g.item_base + k;
    }
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
}

}  // namespace

cudaError_t launch_cell_sort(const BatchDev& b, double* pos, int* status, int family,
                             int smem_cells, cudaStream_t st)
{
    const size_t smem = sizeof(int) * (size_t)smem_cells;
    return launch_pdl(cell_sort_kernel, dim3(b.nsys), dim3(kCellThreads), smem, st, b, pos, status, family);
}

cudaError_t configure_cell_kernels()
{
    return cudaFuncSetAttribute(cell_sort_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(sizeof(int) * kMaxCellsPerSystem));
}

}  // namespace akmc
