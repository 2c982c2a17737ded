// Host-side internals shared by the C-ABI translation units (capi.cu, walkers.cu): the
// error helper, device buffers, kernel timing and the akmc_field / akmc_batch objects.
// Not part of the public ABI.
#pragma once

#include <string>
#include <vector>

#include "akmc_internal.h"
#include "potentials.h"

namespace akmc {

// Records the message for akmc_last_error and returns the code.
akmc_status fail(akmc_status code, const std::string& m);

#define AKMC_CUDA(call)                                                                      \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return fail(AKMC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));  \
    } while (0)

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t alloc(size_t count)
    {
        release();
        n = count;
        if (count == 0) return cudaSuccess;
        return cudaMalloc(&p, sizeof(T) * count);
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    ~DevBuf() { release(); }
};

enum KernelId { K_CELL = 0, K_EAM_DENSITY, K_EAM_FORCE, K_STRUCTURE, K_IONIC_FORCE, K_ENERGY, K_COUNT };
extern const char* const kKernelNames[K_COUNT];

// Event timing of the kernels of one batch (enabled by akmc_batch_profile).
struct KernelTimer {
    bool on = false;
    std::vector<cudaEvent_t> pool;
    struct Rec { int k; cudaEvent_t a, b; };
    std::vector<Rec> pending;
    double ms[K_COUNT] = {0};
    int count[K_COUNT] = {0};
    cudaEvent_t take()
    {
        if (pool.empty()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            return e;
        }
        cudaEvent_t e = pool.back();
        pool.pop_back();
        return e;
    }
    void drain()
    {
        for (auto& r : pending) {
            cudaEventSynchronize(r.b);
            float t = 0.f;
            cudaEventElapsedTime(&t, r.a, r.b);
            ms[r.k] += t;
            count[r.k] += 1;
            pool.push_back(r.a);
            pool.push_back(r.b);
        }
        pending.clear();
    }
    ~KernelTimer()
    {
        drain();
        for (auto e : pool) cudaEventDestroy(e);
    }
};

// One force call of a batch: cell sort, the family's passes, per-system energies (skipped
// when energy is null: a caller that needs forces only).
// active (device, [nsys], may be null): systems whose entry is 0 are skipped entirely --
// their positions, forces and energies are left as they are.  wrapped (may be null) is
// recorded once the positions are wrapped in place: nothing later in the call writes them.
akmc_status run_batch(akmc_batch* b, double* pos, double* force, double* energy, int* status,
                      cudaStream_t s, const int* active = nullptr, cudaEvent_t wrapped = nullptr);

// A batch of n_images copies of n_groups systems: system m * n_groups + k is image m of
// system k (natoms, box, label, charge given for the n_groups systems).  With an EAM list
// and a skin the images of a system share one sorted order and one neighbour list.
akmc_status batch_create_images(akmc_field* f, int n_groups, int n_images, const int* natoms,
                                const double* box, const int* label, const double* charge, double skin,
                                akmc_batch** out);

}  // namespace akmc

struct akmc_batch {
    akmc_field* field = nullptr;
    akmc::KernelTimer timer;
    akmc::DevBuf<double> h_pos_dev, h_force_dev, h_energy_dev;   // device side of the host path
    cudaStream_t side = nullptr;      // host path: the wrapped positions go back while the passes run
    cudaEvent_t ev_wrapped = nullptr, ev_side = nullptr;
    akmc::DevBuf<int> h_status_dev;
    int nsys = 0, n_total = 0, total_cells = 0, total_items = 0, max_cells = 0;
    std::vector<akmc::SysGeom> geo;        // host copy of the per-system plan (item windows per chunk)
    std::vector<int> ncell;          // cells per system
    std::vector<int> natoms;
    std::vector<double> box;
    akmc::DevBuf<akmc::SysGeom> geom;
    akmc::DevBuf<int> cell_start, perm, keys, slots, order, n_items, label, slabel, sk_counter;
    akmc::DevBuf<int> wc_counter;                     // whole-cell ionic kernel: CTAs done per system
    akmc::DevBuf<int> inv_perm;                       // caller atom -> sorted atom (descriptor rows)
    akmc::DevBuf<double> charge;
    akmc::DevBuf<double4> spos;
    akmc::DevBuf<double2> sextra, eatom, skpart, sk;
    akmc::DevBuf<double4> frec;
    akmc::DevBuf<float2> skf;
    akmc::DevBuf<unsigned short> nbr;
    akmc::DevBuf<int> nbr_count;
    akmc::DevBuf<double> ref_pos;                     // neighbour-list reuse (skin > 0)
    akmc::DevBuf<int> list_mode, list_ok;
    akmc::DevBuf<akmc::WorkItem> items;
    akmc::DevBuf<int> work, counters;                 // per-call work queues
    akmc::DevBuf<int2> chunks;
    akmc::BatchDev view{};
};

struct akmc_field {
    akmc::Potentials pot;
    bool ready = false;
    int precision = AKMC_PREC_MIXED;
    double r_split = 4.5;             // FP64 pair terms inside this distance (mixed ionic)
    double list_density = 0.0;        // floor of the number density sizing EAM neighbour lists
    double lat[9] = {0}, rcp[9] = {0};
    int max_atoms = 0;
    int device = 0;
    // device tables
    akmc::DevBuf<float4> eam_rows;
    akmc::DevBuf<double> eam_phi, eam_dphi, eam_rho, eam_drho, eam_F, eam_dF;
    akmc::EamDev eam{};
    akmc::EwaldSet ewald;
    akmc::DevBuf<int4> kint;
    akmc::DevBuf<double4> kd;
    akmc::DevBuf<float4> kf;
    akmc::DevBuf<int4> kt;
    akmc::DevBuf<int4> kgrp;
    akmc::DevBuf<double> g0;
    akmc::IonicDev ionic{};
    // host-buffer path
    cudaStream_t stream = nullptr;
    akmc_batch* single = nullptr;
    int single_n = -1;
    double* h_pos = nullptr;          // pinned [max_atoms*3]
    double* h_force = nullptr;        // pinned [max_atoms*3]
    double* h_energy = nullptr;       // pinned [5]
    int* h_status = nullptr;          // pinned [1]
    int* h_label = nullptr;           // pinned [max_atoms]
    double* h_charge = nullptr;       // pinned [max_atoms]
    akmc::DevBuf<double> d_pos, d_force, d_energy;
    akmc::DevBuf<int> d_status;
};
