// Internal structures shared by the host side (capi.cu, potentials.cpp) and the
// sm_100a kernels (cells.cu, pair_kernels.cu).  Not part of the public ABI.
#pragma once

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "akmc.h"

namespace akmc {

// Bounds checks of the self-checking build (python -m akmc_b200.build --checks defines
// AKMC_CHECKS and writes libakmc_b200_checks.so).  AKMC_BAD(cond, code, value) is true when
// the index condition `cond` holds (an access would leave its buffer): the build counts the
// hit under `code` in a per-file device array, keeps the first offending value, and the
// caller skips the access; nothing traps.  akmc_checks_read (capi.cu) returns the counts.  In
// the default build every check is the constant false and compiles away.
constexpr int kCheckCodes = 32;
#ifdef AKMC_CHECKS
#define AKMC_CHECKS_FILE(name)                                                               \
    __device__ int g_checks_##name[2 * kCheckCodes];                                         \
    __device__ __forceinline__ bool check_hit(int code, long long v)                         \
    {                                                                                        \
        if (atomicAdd(&g_checks_##name[code], 1) == 0) g_checks_##name[kCheckCodes + code] = (int)v; \
        return true;                                                                         \
    }                                                                                        \
    cudaError_t checks_read_##name(int* out)                                                 \
    {                                                                                        \
        return cudaMemcpyFromSymbol(out, g_checks_##name, sizeof(int) * 2 * kCheckCodes);    \
    }                                                                                        \
    cudaError_t checks_clear_##name()                                                        \
    {                                                                                        \
        static const int zero[2 * kCheckCodes] = {0};                                        \
        return cudaMemcpyToSymbol(g_checks_##name, zero, sizeof(zero));                      \
    }
#define AKMC_BAD(cond, code, v) ((cond) && check_hit((code), (long long)(v)))
#else
#define AKMC_CHECKS_FILE(name)
#define AKMC_BAD(cond, code, v) false
#endif
// the check arrays of the files that carry checks (AKMC_CHECKS build only)
cudaError_t checks_read_cells(int* out);
cudaError_t checks_clear_cells();
cudaError_t checks_read_pair(int* out);
cudaError_t checks_clear_pair();
cudaError_t checks_read_walkers(int* out);
cudaError_t checks_clear_walkers();

constexpr int kMaxSpecies = 8;
constexpr int kMaxEamPots = 4;
constexpr double kPi = 3.14159265358979323846;
constexpr double kTwoPi = 6.28318530717958647692;
constexpr double kCtoev = 14.3996454784;          // e^2/(4 pi eps0), eV*Angstrom
constexpr double kTwoOverRootPi = 1.128379167095512;  // pair/Field.cpp:2223

// Threads per CTA of the pair kernels and the number of home atoms one CTA owns.
constexpr int kPairThreads = 128;
constexpr int kPairWarps = kPairThreads / 32;
constexpr int kHomeChunk = 32;
constexpr int kMinHomeChunk = 8;
// Neighbour candidates staged in shared memory per round.
constexpr int kStageCap = 1024;
// Threads of the per-system cell-sort kernel.
constexpr int kCellThreads = 1024;
// Largest cell grid one system may have (cell counters live in shared memory).
constexpr int kMaxCellsPerSystem = 12288;
// Structure-factor kernel tiling: k-vectors per CTA and atoms per chunk.
constexpr int kSkThreads = 64;
constexpr int kSkAtomChunk = 64;
constexpr int kSkGroup = 4;

// ---------------------------------------------------------------------------------
// host-side potential description
// ---------------------------------------------------------------------------------
struct SpeciesRec {
    std::string name;
    double mass = 0.0, charge = 0.0;
};

struct EamTable {           // MetalPotential as readLEAM leaves it (MetalPotential.cpp:276-361)
    std::string atA, atB, file;
    int n_embed = 0, n_r = 0;
    double step_embed = 0.0, step_r = 0.0, pot_cutoff = 0.0;
    std::vector<double> F, dF, rho, drho, phi, dphi;
};

struct BuckRec {            // TwoBody Buckingham entry (TwoBody.cpp:96-116)
    std::string a, b;
    double A = 0.0, rho = 1.0, C = 0.0;
};

// ---------------------------------------------------------------------------------
// device parameter blocks (passed by value)
// ---------------------------------------------------------------------------------
// The tabulated EAM potentials of a field on the device, one per entry of the potentials
// file (all on one grid), chosen as the reference's ManyBody does (ManyBody.cpp:937-1000,
// 539-549, 598-615, 700-708, 790-826): the density of a neighbour of species b from table
// meshTable[b*ns+b], the embedding of species a from meshTable[a*ns+a], and the pair term of
// species (a, b) -- phi, phi', rho' and the embedding derivative at both densities -- from
// meshTable[a*ns+b].  Species pairs without a potential contribute nothing (meshTable = -1).
struct EamDev {
    int ns, ntab;
    signed char mesh[kMaxSpecies * kMaxSpecies];       // meshTable[a*ns+b]: table index or -1
    unsigned char pair_ok[kMaxSpecies * kMaxSpecies];  // meshTable[a*ns+b] >= 0
    unsigned char dens_ok[kMaxSpecies];                // meshTable[b*ns+b] >= 0
    unsigned char embed_ok[kMaxSpecies];               // meshTable[a*ns+a] >= 0
    // FP32 packed rows of table k at rows + 2 n_r k, two float4 per r bin i:
    //   rows[2i]   = {phi_i, phi_{i+1}-phi_i, dphi_i, dphi_{i+1}-dphi_i}
    //   rows[2i+1] = {drho_i, drho_{i+1}-drho_i, rho_i, rho_{i+1}-rho_i}
    const float4* rows;
    const double *phi, *dphi, *rho, *drho;   // FP64 tables, [ntab][n_r]
    const double *F, *dF;                    // [ntab][n_embed]
    int n_r, n_embed;
    double step_r, inv_step_r, step_embed, inv_step_embed, pot_cutoff;
};

struct IonicDev {
    int ns;
    double buckA[kMaxSpecies * kMaxSpecies];
    double buckInvRho[kMaxSpecies * kMaxSpecies];
    double buckC[kMaxSpecies * kMaxSpecies];
    float buckAf[kMaxSpecies * kMaxSpecies];      // FP32 copies for the far-pair terms
    float buckInvRhof[kMaxSpecies * kMaxSpecies];
    float buckCf[kMaxSpecies * kMaxSpecies];
    double cfact, eta, inv_eta, r_split2;
    float etaf, eta3f, inv_etaf;
    int nk;
    const int4* kint;        // nx, ny, nz per k-vector
    const double* g0;        // energy prefactor incl. half-space weight
    const double4* kd;       // {nx, ny, nz, g0} as doubles (phase in FP64)
    const float4* kf;        // {nx, ny, nz, g0} as floats (force terms in FP32)
    // 1-D phase-factor table of one atom: X[0..gx], Y[-gy..gy], Z[-gz..gz] at offsets
    // 0, gx+1, gx+1+2gy+1; kt[k] = the three table slots of k-vector k
    const int4* kt;
    int gx, gy, gz, ntab;
    // k-vectors in groups of at most kSkGroup that share (nx, ny) and have consecutive nz
    // (the k-set is ordered nx, ny, nz): {first k, count, X slot | Y slot << 16, Z slot of the first}
    const int4* kgrp;
    int ngrp;
    // erfc(x) exp(x^2) on the far-pair range x = eta r, r in [r_split, cutoff], as a
    // polynomial of degree kErfcxDeg in t = x * erfcx_t1 + erfcx_t0 (t in [-1, 1]): the
    // Chebyshev interpolant of the function, fitted in FP64 at setup and written in monomial
    // form (erfcx_c[k] multiplies t^k).  erfcx_on = 0 where the fit misses 1e-9 relative on
    // the range: the far pairs then call erfcf.
    float erfcx_c[12];
    float erfcx_c0lo;        // erfcx_c[0]'s FP32 rounding error (kept, so the sum carries no bias)
    float erfcx_t0, erfcx_t1;
    int erfcx_on;
};

constexpr int kErfcxDeg = 11;

// Largest phase table a warp keeps in shared memory (entries).
constexpr int kMaxPhaseTable = 128;

// Per-system geometry of one batch (device array, one entry per system).
struct SysGeom {
    int atom_begin, n_atoms;
    int cell_begin, nc[3];
    int item_base, item_cap;          // work-item window of this system
    int home_chunk;                   // home atoms per work item of this system (8, 16 or 32)
    int mi_mask;                      // bit d set: dimension d uses per-pair minimum image
    double L[3], invL[3], cell_w_inv[3];
};

struct WorkItem {                     // one CTA of the pair kernels
    int cell;                         // global cell index
    int first;                        // first sorted atom (global index)
    int count;                        // home atoms of this item (<= kHomeChunk)
    int sys;
};

// Batch view passed to kernels.
struct BatchDev {
    int nsys, n_total, total_cells, total_items;
    const SysGeom* geom;
    int* cell_start;                  // [total_cells + 1] global sorted offsets
    int* perm;                        // sorted -> original (global index)
    int* keys;                        // per original atom: local cell
    int* slots;                       // per original atom: slot inside cell
    int* order;                       // per system scratch for the segment sort
    double4* spos;                    // sorted wrapped positions, w = charge or label
    double2* sextra;                  // EAM: {F'(rho), rho} per sorted atom
    double2* eatom;                   // per sorted atom partial energies
    WorkItem* items;
    int* n_items;                     // per system
    const int* label;                 // per original atom
    const double* charge;             // per original atom
    int* slabel;                      // species label per sorted atom
    double2* skpart;                  // [nsys][nchunk][nk] partial structure factors
    double2* sk;                      // [nsys][nk] structure factors C_k, S_k
    float2* skf;                      // [nsys][nk] the same in FP32 (force terms)
    int* sk_counter;                  // [nsys][ktiles] arrival counters (self-resetting)
    int sk_chunks;                    // atom chunks of the structure-factor kernel
    int stage_cap;                    // candidates staged per round (<= kStageCap)
    int home_chunk;                   // home atoms per work item (8, 16 or 32); 0 = kHomeChunk
    // EAM neighbour list written by the density pass (null: the force pass rescans cells)
    unsigned short* nbr;              // [nbr_cap][n_total], index within the atom's system
    int* nbr_count;                   // [n_total]
    int nbr_cap;
    // with a list: the force pass's neighbour record per sorted atom, {x, y, z, F'(rho)},
    // F' NaN where rho < 1e-8 (no many-body term for its pairs); written by the density pass
    double4* frec;
    // per-system switch of one call (null: every system): a system whose entry is 0 is
    // skipped by every kernel, its positions, forces and energies left untouched
    const int* active;
    // EAM neighbour-list reuse.  With skin > 0 a system's list holds every pair within
    // cutoff + skin at the positions of its last build (ref_pos, original atom order) and
    // is reused, without re-sorting, while no atom has moved more than skin/2 since; the
    // pair terms still apply the exact test rsq <= cutoff^2.  skin 0: every call sorts and
    // scans the cells (list_mode 0).
    double skin;
    double* ref_pos;                  // [n_total][3]
    int* list_mode;                   // per system, this call: 0 no skin, 1 built, 2 reused
    int* list_ok;                     // per system: a list for the current plan exists
    // Work queues of one call, filled by the cell kernel for the systems that run (null
    // work: the pair kernels take one CTA per planned item and the list kernels one thread
    // per atom of the batch).  Persistent CTAs then take queued items by ticket and atom
    // chunks by stride, so a call where few systems run costs few CTAs.
    int* work;                        // [total_items at home chunk 8] queued item indices
    int2* chunks;                     // [chunk_cap] {system, first atom within it}
    int* counters;                    // [kCounters]: queued items, queued chunks, tickets
    int* ticket;                      // the ticket counter of this pair-kernel launch
    int chunk_cap;
    // Image groups (n_images > 1): systems m * n_groups + k, m < n_images, are images of
    // one group k -- the same atoms, box and labels at positions within a fraction of the
    // skin of one another (the ends of a dimer and its rotation trial).  They share one
    // sorted order and one neighbour list, kept at image 0's rows with image 0's build
    // positions and rebuilt from the first image that runs in a call whenever an image that
    // runs has moved skin/2 from them.  0 or 1: every system on its own.
    int n_images, n_groups;
    // Species count against which the cell kernel checks every label (an out-of-range label
    // sets AKMC_ERR_ARG and is read as species 0); 0: the labels were checked on the host
    // when the batch was created.
    int label_check;
    // Ionic batches whose every system has fewer than three cells in every dimension (the
    // whole cell is one neighbourhood, every pair under the minimum image) and at most
    // kWholeCellMaxAtoms atoms: the largest system's atom count, and the mixed-precision ionic
    // pass runs the whole-cell kernel.  0: the cell-list pass.
    int whole_cell_n;
    int* wc_counter;                  // [nsys] CTAs of the whole-cell kernel done (self-resetting)
};

constexpr int kWholeCellMaxAtoms = 4096;

constexpr int kChunkAtoms = 128;      // atoms per queued chunk (the list kernels' CTA size)
constexpr int kCounters = 8;          // 0 items, 1 chunks, 2.. one ticket per pair launch
constexpr int kTicketDensity = 2, kTicketForce = 3, kTicketIonic = 4;

#ifdef __CUDACC__
__device__ __forceinline__ bool system_active(const BatchDev& b, int s)
{
    return b.active == nullptr || b.active[s] != 0;
}

// Neighbour-list row of sorted atom i of system s minus i: 0, or for an image of a group
// that shares its list (a skin) the offset to the same atom of the group's image 0.
__device__ __forceinline__ int list_shift(const BatchDev& b, int s)
{
    return b.n_images > 1 && b.skin > 0.0 ? b.geom[s % b.n_groups].atom_begin - b.geom[s].atom_begin : 0;
}
#endif

// ---------------------------------------------------------------------------------
// Programmatic dependent launch.  Every kernel of the force path is launched with
// programmatic stream serialisation: it may begin while the previous kernel on the stream
// is finishing.  Each kernel therefore waits for its predecessor (griddepcontrol.wait)
// before reading anything the predecessor wrote, and only then lets its own successor
// start (griddepcontrol.launch_dependents) -- so a successor can never run ahead of a
// kernel two places back.  The ionic force kernel is the one exception: it releases its
// successor at once and defers its wait to the reciprocal-space loop, which is the only
// part that reads the structure-factor kernel's output.
// ---------------------------------------------------------------------------------
#ifdef __CUDACC__
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <class... KArgs, class... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                       cudaStream_t s, Args&&... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}
#endif

// ---------------------------------------------------------------------------------
// kernel launchers (defined in the .cu files)
// ---------------------------------------------------------------------------------
cudaError_t launch_wrap_whole_cell(const BatchDev& b, double* pos, int* status, cudaStream_t s);
cudaError_t launch_cell_sort(const BatchDev& b, double* pos, int* status, int family,
                             int smem_cells, cudaStream_t s);
cudaError_t launch_eam_density(const BatchDev& b, const EamDev& p, double rc2, int* status,
                               int precision, cudaStream_t s);
cudaError_t launch_eam_force(const BatchDev& b, const EamDev& p, double rc2, double* force,
                             int* status, int precision, cudaStream_t s);
cudaError_t launch_structure_factor(const BatchDev& b, const IonicDev& p, int precision,
                                    cudaStream_t s);
// energy (whole-cell batches only; may be null): the kernel also writes each system's energy
// record, as energy_reduce_kernel does
cudaError_t launch_ionic_force(const BatchDev& b, const IonicDev& p, double rc2, double* force, double* energy,
                               int* status, int precision, cudaStream_t s);
cudaError_t launch_energy_reduce(const BatchDev& b, int family, const IonicDev* ip,
                                 double* energy, cudaStream_t s);
cudaError_t configure_cell_kernels();
cudaError_t configure_pair_kernels();

}  // namespace akmc
