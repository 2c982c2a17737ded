// KMC step on the GPU: FP64 event table, duplicate-saddle removal, rate selection and
// time advance (sm_100a).
//
// The reference builds its event list on the master rank in mixed precision (positions and
// energies sent as float, kmc/KineticMonteCarlo.cpp:1376-1460; Event::Event computes
// rate = prefactor * exp(-E_a / (k_B T)) from a float E_a, kmc/Event.cpp:66-105) and selects
// with KineticMonteCarlo.cpp:147-199 and 1151-1160:
//   R = sum of rates (in list order); the chosen event is the first i whose running sum of
//   rates exceeds u1 * R; the time advance is -(1/R) ln(u2), zero when |R| <= 1e-18.
// Here every event quantity is FP64 on the device: E_a = E_saddle - E_min, the rates, the
// running sums (summed sequentially in list order, as the reference does, so that the chosen
// index is the reference's for the same u1) and the time step.  u1, u2 come from a
// counter-based generator with an explicit seed (the reference seeds std::mt19937_64 from the
// clock, kmc/kmc.cpp:27-28, so its runs cannot be repeated): Philox4x64-10 (Salmon, Moraes,
// Dror and Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC 2011), doubles formed from
// the top 53 bits.
#include <cmath>
#include <cstdint>

#include "host_internal.h"
#include "philox.h"

namespace akmc {

namespace {

constexpr double kBoltzmann = 8.617333262145e-5;   // eV/K (potentials/metal/Energy.h:43)
constexpr int kDedupThreads = 256;

// n uniform doubles in [0, 1): block b of four comes from counter (counter + 1 + b) with the
// 128-bit counter's low word carrying into the next -- the sequence numpy's Philox bit
// generator gives for the same key and counter.
__global__ void uniforms_kernel(uint64_t k0, uint64_t k1, uint64_t c0, uint64_t c1, int n,
                                double* __restrict__ out)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (4 * b >= n) return;
    uint64_t c[4];
    philox_block(k0, k1, c0, c1, (uint64_t)b, c);
    for (int j = 0; j < 4 && 4 * b + j < n; j++) out[4 * b + j] = philox_to_unit(c[j]);
}

// Duplicate saddles: event i duplicates the first j < i of the same group (same basin and
// system) that is usable, within e_tol in saddle energy and within d_tol for every atom
// (minimum image).  One CTA per event.
__global__ void __launch_bounds__(kDedupThreads)
dedup_kernel(int n, const int* __restrict__ group, const int* __restrict__ usable,
             const double* __restrict__ energy, const double* __restrict__ pos,
             const long long* __restrict__ begin, const int* __restrict__ natoms,
             const double* __restrict__ box, double e_tol, double d_tol, int* __restrict__ dup)
{
    __shared__ int s_hit;
    const int i = blockIdx.x;
    if (threadIdx.x == 0) s_hit = -1;
    __syncthreads();
    if (!usable[i]) {
        if (threadIdx.x == 0) dup[i] = -1;
        return;
    }
    const double d2 = d_tol * d_tol;
    for (int j = 0; j < i; j++) {
        if (!usable[j] || group[j] != group[i] || natoms[j] != natoms[i]) continue;
        if (!(fabs(energy[j] - energy[i]) <= e_tol)) continue;
        const double* a = pos + 3 * begin[i];
        const double* b = pos + 3 * begin[j];
        const double L0 = box[3 * i], L1 = box[3 * i + 1], L2 = box[3 * i + 2];
        int far = 0;
        for (int t = threadIdx.x; t < natoms[i]; t += blockDim.x) {
            double dx = a[3 * t] - b[3 * t], dy = a[3 * t + 1] - b[3 * t + 1], dz = a[3 * t + 2] - b[3 * t + 2];
            dx -= L0 * rint(dx / L0);
            dy -= L1 * rint(dy / L1);
            dz -= L2 * rint(dz / L2);
            far |= (dx * dx + dy * dy + dz * dz > d2);
        }
        if (!__syncthreads_or(far)) {
            if (threadIdx.x == 0) s_hit = j;
            break;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) dup[i] = s_hit;
}

// Rates of every event (parallel), then one thread forms the running sums in list order and
// selects -- the reference's loops, in FP64.
__global__ void select_kernel(int n, const double* __restrict__ e_saddle, const double* __restrict__ e_min,
                              const int* __restrict__ usable, double prefactor, double beta,
                              const double* __restrict__ u, double* __restrict__ rate,
                              double* __restrict__ cum, akmc_kmc_step* __restrict__ out)
{
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double ea = e_saddle[i] - e_min[i];
        rate[i] = usable[i] ? prefactor * exp(-ea * beta) : 0.0;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    double total = 0.0;
    int nu = 0;
    for (int i = 0; i < n; i++) {
        total += rate[i];
        cum[i] = total;
        nu += usable[i] != 0;
    }
    const double threshold = u[0] * total;
    int chosen = -1;
    for (int i = 0; i < n; i++) {
        if (usable[i] && cum[i] > threshold) {
            chosen = i;
            break;
        }
    }
    akmc_kmc_step s;
    s.chosen = chosen;
    s.n_usable = nu;
    s.total_rate = total;
    // calculateTime: (1/R) ln(u2), negated by the caller; u2 = 0 is taken as 2^-53
    const double u2 = u[1] > 0.0 ? u[1] : 0x1.0p-53;
    s.dt = fabs(total) > 1.0e-18 ? -log(u2) / total : 0.0;
    s.barrier = chosen >= 0 ? e_saddle[chosen] - e_min[chosen] : 0.0;
    s.rate = chosen >= 0 ? rate[chosen] : 0.0;
    s.u1 = u[0];
    s.u2 = u[1];
    *out = s;
}

}  // namespace
}  // namespace akmc

using namespace akmc;

extern "C" {

akmc_status akmc_kmc_uniforms(uint64_t seed, uint64_t key_hi, uint64_t counter, int n,
                              double* out_dev, void* stream)
{
    if (n < 0 || (n > 0 && !out_dev)) return fail(AKMC_ERR_ARG, "bad uniforms arguments");
    if (n == 0) return AKMC_OK;
    const int blocks4 = (n + 3) / 4;
    uniforms_kernel<<<(blocks4 + 127) / 128, 128, 0, (cudaStream_t)stream>>>(seed, key_hi, counter, 0, n, out_dev);
    AKMC_CUDA(cudaGetLastError());
    return AKMC_OK;
}

akmc_status akmc_events_dedup(int n, const int* group_dev, const int* usable_dev,
                              const double* energy_dev, const double* pos_dev,
                              const long long* begin_dev, const int* natoms_dev, const double* box_dev,
                              double e_tol, double d_tol, int* dup_dev, void* stream)
{
    if (n < 0 || (n > 0 && (!group_dev || !usable_dev || !energy_dev || !pos_dev || !begin_dev ||
                            !natoms_dev || !box_dev || !dup_dev)))
        return fail(AKMC_ERR_ARG, "bad dedup arguments");
    if (n == 0) return AKMC_OK;
    dedup_kernel<<<n, kDedupThreads, 0, (cudaStream_t)stream>>>(n, group_dev, usable_dev, energy_dev, pos_dev,
                                                                  begin_dev, natoms_dev, box_dev, e_tol, d_tol, dup_dev);
    AKMC_CUDA(cudaGetLastError());
    return AKMC_OK;
}

akmc_status akmc_kmc_select(int n, const double* e_saddle_dev, const double* e_min_dev,
                            const int* usable_dev, double prefactor, double temperature,
                            const double* u_dev, double* rate_dev, double* cum_dev,
                            akmc_kmc_step* step_dev, void* stream)
{
    if (n < 0 || !u_dev || !step_dev || (n > 0 && (!e_saddle_dev || !e_min_dev || !usable_dev ||
                                                   !rate_dev || !cum_dev)))
        return fail(AKMC_ERR_ARG, "bad select arguments");
    if (!(temperature > 0.0) || !(prefactor > 0.0)) return fail(AKMC_ERR_ARG, "prefactor and temperature must be positive");
    const double beta = 1.0 / (kBoltzmann * temperature);
    select_kernel<<<1, 256, 0, (cudaStream_t)stream>>>(n, e_saddle_dev, e_min_dev, usable_dev, prefactor, beta,
                                                       u_dev, rate_dev, cum_dev, step_dev);
    AKMC_CUDA(cudaGetLastError());
    return AKMC_OK;
}

}  // extern "C"
