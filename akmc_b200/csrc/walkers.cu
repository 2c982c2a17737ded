// Batched walkers on the force path: FIRE relaxations and Dimer saddle searches of many
// independent systems at once (sm_100a).
//
// FIRE follows the reference's Relax::FIRERelax, Euler variant (optim/Relax.cpp:44-315,
// defaults Common/RelaxCntrl.h:15-38): mixing v <- (1-a) v + a |v|/|F| F when F.v > 0,
// time-step growth after N_min downhill steps, reset on uphill steps, x += dt v then
// v += dt*EVTODL*F, frozen forces zeroed after each force call (Basis::freezeForces),
// centre-of-mass velocity removed (Relax::centreOfMass), converged when |F| < normTol or
// max_i |F_i| < forceTol, checked after every step and never before the first.
//
// The Dimer.  The reference's optim/Dimer.cpp is an empty stub; its commented design
// (optim/Dimer.cpp:416-618) and controls (Common/DimerCntrl.h:18-88) fix the
// ingredients, and the published method fixes the rest:
//   forces F0 = F(x), F1 = F(x + Delta N); curvature C = (F0 - F1).N / Delta;
//   rotational force Frot = 2 (F1 - F0)_perp (the F1 - F2 of the design, F2 = 2 F0 - F1);
//   rotation (Kaestner and Sherwood, J. Chem. Phys. 128, 014106 (2008)): trial angle
//     theta1 = atan(|Frot| / (2 Delta |C|)) / 2, one force call at N' = N cos theta1 +
//     Theta sin theta1, C(theta) = a0/2 + a1 cos 2theta + b1 sin 2theta fitted to C(0),
//     dC/dtheta(0) and C(theta1), N turned to the fitted minimum, F1 carried to the new
//     N by the interpolation of Heyden, Bell and Keil, J. Chem. Phys. 123, 224101 (2005);
//     skipped when |Frot| / (2 Delta) is below the rotation tolerance;
//   translation: one FIRE step (the constants of DimerCntrl) on the modified force
//     F0 - 2 (F0.N) N when C < 0 and -(F0.N) N otherwise (Henkelman and Jonsson,
//     J. Chem. Phys. 111, 7010 (1999)), with a per-atom step cap;
//   a saddle when max_i |F0_i| < forceTol and C < maxEigenvalue.
//
// Layout: the FIRE kernels run one CTA per walker, the Dimer's rotation and end-of-iteration
// kernels one 4-CTA thread-block cluster per walker (reductions combined through distributed
// shared memory); all walker algebra (dot products, curvature, angles, energies) is FP64 and
// reduced in a fixed order, so runs repeat bit for bit.  The force calls are ordinary batch
// calls with a per-system active mask: walkers that have finished, or that need no rotation
// this step, cost nothing.  The Dimer's two ends and its rotation trial are three images of
// the walker in one batch, sharing a sorted order and a neighbour list.  One iteration
// (walker kernels + force calls) is captured once as a CUDA graph and replayed; the host
// reads a running-walker count every few iterations.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include <cooperative_groups.h>

#include "host_internal.h"

namespace akmc {

AKMC_CHECKS_FILE(walkers)

namespace {

constexpr int kWalkThreads = 512;
constexpr double kEvtodl = 9648.530821;   // Energy::timeStepUnit (potentials/metal/Energy.h:40)

constexpr int kLbfgsMem = 8;              // largest L-BFGS memory
constexpr int kLbfgsDots = 5 * kLbfgsMem; // dot products gathered by one L-BFGS pass
constexpr int kFinishThreads = 256;       // Dimer rotation and end-of-iteration kernels
constexpr int kWalkCluster = 4;           // CTAs per walker in those kernels (one cluster)

struct WalkerState {
    double dt, alpha;
    double energy, e_start, curvature, fmax, fnorm;
    double theta1, b1;                    // rotation in flight (prep -> finish)
    double best_fmax;                     // Dimer: smallest max|F| so far (patience)
    int nstep, iter, status, rotating, calls, best_iter;
    int lb_count, lb_head, lb_prev, lb_pad;   // L-BFGS ring: pairs held, next slot, xp/gp valid
    double lb_rho[kLbfgsMem];             // 1 / (s.y) of the stored pairs
};

struct FireDev {
    int max_iter, n_min;
    double norm_tol, force_tol, dt0, dt_max, alpha0, alpha_dec, step_inc, step_dec, max_move;
};

struct DimerDev {
    int max_iter, max_rotations, n_min, patience;
    double delta, rot_tol, force_tol, max_eigenvalue, min_trial, max_move, max_rise;
    double dt0, dt_max, alpha0, alpha_dec, step_inc, step_dec;
    int translation, lbfgs_memory;        // 0 FIRE, 1 L-BFGS
    double max_step, convex_step;         // L-BFGS step caps
};

// L-BFGS history of the walker set: ring slots of s = x_k+1 - x_k and y = g_k+1 - g_k
// (g = -modified force), the previous x and g, and a work vector.  [kLbfgsMem][3 n_total]
// for S and Y, [3 n_total] for the rest; per walker the Gram entries s_i.y_j and y_i.y_j of
// its slots, [W][2][kLbfgsMem][kLbfgsMem].
struct LbfgsDev {
    double* S;
    double* Y;
    double* xp;
    double* gp;
    double* r;
    double* gram;
};

struct WalkDev {
    int W, n_total;
    const int* begin;                     // [W] first atom of walker w
    const int* natoms;                    // [W]
    const double* box;                    // [W][3] box lengths
    const int* frozen;                    // [n_total] or null
    WalkerState* st;                      // [W]
    int* running;                         // walkers still running after this iteration
};

__device__ __forceinline__ double w_box_len(const WalkDev& w, int k, int d) { return w.box[3 * k + d]; }

__device__ double block_sum(double v, double* sh)
{
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double r = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) r += sh[w];   // fixed order, every thread
    return r;
}

__device__ double block_max(double v, double* sh)
{
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double r = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) r = fmax(r, sh[w]);
    return r;
}

// K reductions over the CTA at once, in a fixed order: the first K - M per-thread values
// are summed, the last M maxed (values >= 0).  out[0 .. K) (shared) holds the results for
// every thread on return; red is shared scratch of (blockDim.x / 32) * K.
template <int K, int M>
__device__ void block_reduce(double (&v)[K], double* red, double* out)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    #pragma unroll
    for (int j = 0; j < K; j++) {
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double u = __shfl_xor_sync(0xffffffffu, v[j], o);
            v[j] = j < K - M ? v[j] + u : fmax(v[j], u);
        }
    }
    __syncthreads();              // earlier readers of red and out are done
    if (lane == 0) {
        #pragma unroll
        for (int j = 0; j < K; j++) red[warp * K + j] = v[j];
    }
    __syncthreads();
    for (int j = threadIdx.x; j < K; j += blockDim.x) {
        double r = 0.0;
        for (int q = 0; q < nw; q++) r = j < K - M ? r + red[q * K + j] : fmax(r, red[q * K + j]);
        out[j] = r;
    }
    __syncthreads();
}

// The CTAs that share one walker: a thread-block cluster along x, the walker's atoms dealt
// round-robin over all its threads (atom a to CTA (a / blockDim.x) % size).  Every CTA runs
// the same code on its own atoms and obtains the same reductions, so the walker algebra is
// identical in all of them; rank 0 alone writes the walker's state.
struct Team {
    int rank, size, phase;
    __device__ int first() const { return rank * (int)blockDim.x + (int)threadIdx.x; }
    __device__ int stride() const { return size * (int)blockDim.x; }
    __device__ bool leader() const { return rank == 0 && threadIdx.x == 0; }
};

__device__ __forceinline__ Team make_team()
{
    cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
    return Team{(int)cl.block_rank(), (int)cl.num_blocks(), 0};
}

constexpr int kTeamMaxK = 20;             // values reduced at once by a team

// block_reduce over the walker's cluster: the CTA's partials go to part (shared, two
// buffers used in turn), the cluster barrier, then every CTA combines the partials of ranks
// 0 .. size-1 in that order through distributed shared memory into res (shared).  A CTA
// rewrites a partials buffer only after the next barrier, by which every CTA has read it;
// before a CTA exits after a team_reduce it must pass team_end.
template <int K, int M>
__device__ void team_reduce(Team& team, double (&v)[K], double* red, double* part, double* res)
{
    static_assert(K <= kTeamMaxK, "team reduction too wide");
    double* mine = part + team.phase * kTeamMaxK;
    team.phase ^= 1;
    block_reduce<K, M>(v, red, mine);
    if (team.size == 1) {
        for (int j = threadIdx.x; j < K; j += blockDim.x) res[j] = mine[j];
        __syncthreads();
        return;
    }
    cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
    cl.sync();
    for (int j = threadIdx.x; j < K; j += blockDim.x) {
        double r = 0.0;
        for (int q = 0; q < team.size; q++) {
            const double u = cl.map_shared_rank(mine, q)[j];
            r = j < K - M ? r + u : fmax(r, u);
        }
        res[j] = r;
    }
    __syncthreads();
}

// No CTA of the cluster leaves while another may still read its shared memory.
__device__ __forceinline__ void team_end(const Team& team)
{
    if (team.size > 1) cooperative_groups::this_cluster().sync();
}

// One FIRE step of one walker (every thread of its CTA), Relax.cpp:129-191.  force(i)
// gives component i (0 .. 3n) of the driving force; x and v are the walker's rows.
template <class Force>
__device__ void fire_update(WalkerState& st, int n_min, double dt_max, double alpha0,
                            double alpha_dec, double step_inc, double step_dec, double max_move,
                            const Force& force, double* x, double* v, int n, const int* frozen,
                            double* sh)
{
    double P = 0.0, f2 = 0.0, v2 = 0.0;
    for (int i = threadIdx.x; i < 3 * n; i += blockDim.x) {
        const double f = force(i), vv = v[i];
        P += f * vv;
        f2 += f * f;
        v2 += vv * vv;
    }
    P = block_sum(P, sh);
    f2 = block_sum(f2, sh);
    v2 = block_sum(v2, sh);
    const double fnorm = sqrt(f2), vnorm = sqrt(v2);
    const double one_less = 1.0 - st.alpha;
    const double alpha_force = fnorm > 0.0 ? st.alpha * vnorm / fnorm : 0.0;
    const bool downhill = P > 0.0;
    double dt = st.dt;
    if (downhill) {
        if (st.nstep > n_min) dt = fmin(dt * step_inc, dt_max);
    } else {
        dt *= step_dec;
    }
    auto mixed = [&](int i) {
        if (!downhill) return 0.0;
        if (frozen && frozen[i / 3]) return v[i];
        return one_less * v[i] + alpha_force * force(i);
    };
    double scale = 1.0;
    if (max_move > 0.0) {
        double m2 = 0.0;
        for (int a = threadIdx.x; a < n; a += blockDim.x) {
            const double u0 = mixed(3 * a), u1 = mixed(3 * a + 1), u2 = mixed(3 * a + 2);
            m2 = fmax(m2, u0 * u0 + u1 * u1 + u2 * u2);
        }
        const double vm = sqrt(block_max(m2, sh));
        if (dt * vm > max_move) scale = max_move / (dt * vm);
    }
    const double fact = dt * kEvtodl;
    __syncthreads();              // every thread has read v before any thread writes it
    for (int i = threadIdx.x; i < 3 * n; i += blockDim.x) {
        double vv = mixed(i) * scale;
        if (!(frozen && frozen[i / 3])) {
            x[i] += dt * vv;
            vv += fact * force(i);
        }
        v[i] = vv;
    }
    if (downhill) {
        if (st.nstep > n_min) st.alpha *= alpha_dec;
        st.nstep += 1;
    } else {
        st.nstep = 0;
        st.alpha = alpha0;
    }
    st.dt = dt;
    st.iter += 1;
}

__global__ void __launch_bounds__(kWalkThreads)
walkers_init_kernel(WalkDev w, double dt0, double alpha0, double* __restrict__ v,
                    double* __restrict__ mode, int* __restrict__ active, int n_active,
                    const int* __restrict__ run_mask)
{
    __shared__ double sh[32];
    const int k = blockIdx.x;
    if (run_mask && !run_mask[k]) {                 // not run: untouched, never active
        if (threadIdx.x == 0) {
            WalkerState st = {};
            st.status = AKMC_WALKER_SKIPPED;
            w.st[k] = st;
            for (int r = 0; r < n_active; r++) active[r * w.W + k] = 0;
        }
        return;
    }
    const int a0 = w.begin[k], n = w.natoms[k];
    if (AKMC_BAD(a0 < 0 || n < 0 || a0 + n > w.n_total, 1, k)) return;
    double* vk = v + 3 * (size_t)a0;
    for (int i = threadIdx.x; i < 3 * n; i += blockDim.x) vk[i] = 0.0;
    if (mode) {                                     // unit-normalise the initial mode
        double* Nk = mode + 3 * (size_t)a0;
        if (w.frozen)                               // frozen atoms take no part in the mode
            for (int i = threadIdx.x; i < 3 * n; i += blockDim.x)
                if (w.frozen[a0 + i / 3]) Nk[i] = 0.0;
        __syncthreads();
        double s = 0.0;
        for (int i = threadIdx.x; i < 3 * n; i += blockDim.x) s += Nk[i] * Nk[i];
        s = block_sum(s, sh);
        const double inv = s > 0.0 ? 1.0 / sqrt(s) : 0.0;
        for (int i = threadIdx.x; i < 3 * n; i += blockDim.x) Nk[i] *= inv;
    }
    if (threadIdx.x == 0) {
        WalkerState st = {};
        st.dt = dt0;
        st.alpha = alpha0;
        st.nstep = 1;                               // Relax.cpp:49
        w.st[k] = st;
        for (int r = 0; r < n_active; r++) active[r * w.W + k] = 1;
    }
}

// ---------------------------------------------------------------------------------
// FIRE
// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(kWalkThreads)
fire_step_kernel(WalkDev w, FireDev P, double* __restrict__ x, double* __restrict__ v,
                 const double* __restrict__ F, int* __restrict__ active)
{
    __shared__ double sh[32];
    const int k = blockIdx.x;
    WalkerState st = w.st[k];
    if (threadIdx.x == 0) active[k] = st.status == 0;
    if (st.status != 0) return;
    const int a0 = w.begin[k], n = w.natoms[k];
    if (AKMC_BAD(a0 < 0 || n < 0 || a0 + n > w.n_total, 1, k)) return;
    const double* Fk = F + 3 * (size_t)a0;
    fire_update(st, P.n_min, P.dt_max, P.alpha0, P.alpha_dec, P.step_inc, P.step_dec, P.max_move,
                [&](int i) { return Fk[i]; }, x + 3 * (size_t)a0, v + 3 * (size_t)a0, n,
                w.frozen ? w.frozen + a0 : nullptr, sh);
    if (threadIdx.x == 0) w.st[k] = st;
}

// After a force call: frozen forces zeroed, centre-of-mass velocity removed (check != 0),
// the convergence test (Relax.cpp:229-276).  Every thread ends with the same st.
__device__ void fire_check_body(const WalkDev& w, const FireDev& P, int k, double* v, double* F,
                                const double* energy, const int* fstatus, int check,
                                WalkerState& st, double* sh)
{
    const int a0 = w.begin[k], n = w.natoms[k];
    if (AKMC_BAD(a0 < 0 || n < 0 || a0 + n > w.n_total, 1, k)) return;
    double* Fk = F + 3 * (size_t)a0;
    double* vk = v + 3 * (size_t)a0;
    if (w.frozen)
        for (int i = threadIdx.x; i < 3 * n; i += blockDim.x)
            if (w.frozen[a0 + i / 3]) Fk[i] = 0.0;
    double c[3] = {0.0, 0.0, 0.0};
    if (check) {
        for (int d = 0; d < 3; d++) {
            double s = 0.0;
            for (int a = threadIdx.x; a < n; a += blockDim.x) s += vk[3 * a + d];
            c[d] = block_sum(s, sh) / n;
        }
    }
    __syncthreads();
    double f2 = 0.0, fm = 0.0;
    for (int a = threadIdx.x; a < n; a += blockDim.x) {
        double s = 0.0;
        for (int d = 0; d < 3; d++) {
            if (check) vk[3 * a + d] -= c[d];
            s += Fk[3 * a + d] * Fk[3 * a + d];
        }
        f2 += s;
        fm = fmax(fm, s);
    }
    f2 = block_sum(f2, sh);
    fm = block_max(fm, sh);
    st.energy = energy[5 * (size_t)k];
    st.fnorm = sqrt(f2);
    st.fmax = sqrt(fm);
    st.calls += 1;
    if (fstatus[k] != AKMC_OK) st.status = AKMC_WALKER_FORCE_ERROR;
    else if (check && (st.fnorm < P.norm_tol || st.fmax < P.force_tol)) st.status = AKMC_WALKER_CONVERGED;
    else if (check && st.iter >= P.max_iter) st.status = AKMC_WALKER_MAX_ITER;
}

// The force call before the loop: frozen forces zeroed, energy recorded, no test.
__global__ void __launch_bounds__(kWalkThreads)
fire_check_kernel(WalkDev w, FireDev P, double* __restrict__ v, double* __restrict__ F,
                  const double* __restrict__ energy, const int* __restrict__ fstatus)
{
    __shared__ double sh[32];
    const int k = blockIdx.x;
    WalkerState st = w.st[k];
    if (st.status != 0) return;
    fire_check_body(w, P, k, v, F, energy, fstatus, 0, st, sh);
    if (threadIdx.x == 0) w.st[k] = st;
}

// One loop iteration after its force call: the test of this step and, for a walker still
// running, its next FIRE step.
__global__ void __launch_bounds__(kWalkThreads)
fire_check_step_kernel(WalkDev w, FireDev P, double* __restrict__ x, double* __restrict__ v,
                       double* __restrict__ F, const double* __restrict__ energy,
                       const int* __restrict__ fstatus, int* __restrict__ active)
{
    __shared__ double sh[32];
    const int k = blockIdx.x;
    WalkerState st = w.st[k];
    if (st.status != 0) {
        if (threadIdx.x == 0) active[k] = 0;
        return;
    }
    fire_check_body(w, P, k, v, F, energy, fstatus, 1, st, sh);
    if (st.status != 0) {
        if (threadIdx.x == 0) {
            active[k] = 0;
            w.st[k] = st;
        }
        return;
    }
    const int a0 = w.begin[k], n = w.natoms[k];
    if (AKMC_BAD(a0 < 0 || n < 0 || a0 + n > w.n_total, 1, k)) return;
    const double* Fk = F + 3 * (size_t)a0;
    fire_update(st, P.n_min, P.dt_max, P.alpha0, P.alpha_dec, P.step_inc, P.step_dec, P.max_move,
                [&](int i) { return Fk[i]; }, x + 3 * (size_t)a0, v + 3 * (size_t)a0, n,
                w.frozen ? w.frozen + a0 : nullptr, sh);
    if (threadIdx.x == 0) {
        active[k] = 1;
        w.st[k] = st;
        atomicAdd(w.running, 1);
    }
}

// ---------------------------------------------------------------------------------
// Dimer
// ---------------------------------------------------------------------------------
// The second image x + Delta N of every running walker (image 1 of the walker in the
// three-image batch: system W + k).
__global__ void __launch_bounds__(kWalkThreads)
dimer_ends_kernel(WalkDev w, DimerDev P, double* __restrict__ pos2, const double* __restrict__ N,
                  int* __restrict__ active2)
{
    const int k = blockIdx.x;
    const bool run = w.st[k].status == 0;
    __syncthreads();              // every thread has read the state before thread 0 writes it
    if (threadIdx.x == 0) {
        active2[k] = run;
        active2[w.W + k] = run;
        if (run) w.st[k].calls += 2;
    }
    if (!run) return;
    const int a0 = w.begin[k], n = w.natoms[k];
    if (AKMC_BAD(a0 < 0 || n < 0 || a0 + n > w.n_total, 1, k)) return;
    const double* x = pos2 + 3 * (size_t)a0;
    double* x1 = pos2 + 3 * ((size_t)w.n_total + a0);
    const double* Nk = N + 3 * (size_t)a0;
    for (int i = threadIdx.x; i < 3 * n; i += blockDim.x) x1[i] = x[i] + P.delta * Nk[i];
}

// Frozen atoms of the Dimer (Basis::freezeForces, Common/Basis.cpp:966-981, applied to every
// image): their forces are zeroed after each force call, so the curvature, the rotational
// force, the saddle test and every translation step see only the free atoms, and the mode,
// zero on them from the start, stays so.
__global__ void __launch_bounds__(256)
dimer_freeze_kernel(const int* __restrict__ frozen, int n_total, int n_images, double* __restrict__ F2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_total || !frozen[i]) return;
    for (int m = 0; m < n_images; m++) {
        double* f = F2 + 3 * ((size_t)m * n_total + i);
        f[0] = 0.0;
        f[1] = 0.0;
        f[2] = 0.0;
    }
}

// Curvature, rotational force and the trial image x + Delta N' (rotation r of this
// iteration; a walker that declined rotation r-1 declines every later one).  One cluster
// of CTAs per walker.
__global__ void __launch_bounds__(kFinishThreads, 2)
dimer_rotate_prep_kernel(WalkDev w, DimerDev P, int r, const double* __restrict__ pos2,
                         const double* __restrict__ F2, const double* __restrict__ N,
                         double* __restrict__ theta, double* __restrict__ post,
                         int* __restrict__ active1)
{
    __shared__ double red[(kFinishThreads / 32) * kTeamMaxK];
    __shared__ double part[2 * kTeamMaxK];
    __shared__ double res[kTeamMaxK];
    Team team = make_team();
    const int k = blockIdx.x / team.size;
    WalkerState st = w.st[k];
    if (st.status != 0 || (r > 0 && !st.rotating)) {
        if (team.leader()) active1[k] = 0;
        return;
    }
    const int a0 = w.begin[k], n3 = 3 * w.natoms[k];
    if (AKMC_BAD(a0 < 0 || n3 < 0 || a0 + n3 / 3 > w.n_total, 1, k)) return;
    const double* F0 = F2 + 3 * (size_t)a0;
    const double* F1 = F2 + 3 * ((size_t)w.n_total + a0);
    const double* Nk = N + 3 * (size_t)a0;
    double* Th = theta + 3 * (size_t)a0;
    double v[1] = {0.0};
    for (int i = team.first(); i < n3; i += team.stride()) v[0] += (F1[i] - F0[i]) * Nk[i];
    team_reduce<1, 0>(team, v, red, part, res);
    const double dn = res[0];
    const double C = -dn / P.delta;
    v[0] = 0.0;
    for (int i = team.first(); i < n3; i += team.stride()) {
        const double fr = 2.0 * ((F1[i] - F0[i]) - dn * Nk[i]);
        Th[i] = fr;
        v[0] += fr * fr;
    }
    team_reduce<1, 0>(team, v, red, part, res);
    const double frn = sqrt(res[0]);
    const double torque = frn / (2.0 * P.delta);
    const bool rotate = torque > P.rot_tol && frn > 0.0;
    const double t1 = rotate ? fmax(0.5 * atan(torque / fmax(fabs(C), 1e-12)), P.min_trial) : 0.0;
    if (team.leader()) {
        st.curvature = C;
        st.rotating = rotate;
        active1[k] = rotate;
        if (rotate) {
            st.theta1 = t1;
            st.b1 = -torque;
            st.calls += 1;
        }
        w.st[k] = st;
    }
    if (rotate) {
        const double c1 = cos(t1), s1 = sin(t1), inv = 1.0 / frn;
        const double* x = pos2 + 3 * (size_t)a0;
        double* xt = post + 3 * (size_t)a0;
        for (int i = team.first(); i < n3; i += team.stride()) {
            const double th = Th[i] * inv;
            Th[i] = th;
            xt[i] = x[i] + P.delta * (Nk[i] * c1 + th * s1);
        }
    }
    team_end(team);
}

// One L-BFGS translation step of walker k on the modified force, g = -(F0 - 2 (F0.N) N)
// (Nocedal's two-loop recursion): while C >= 0 a fixed step up the energy along the unit
// mode; the history is dropped when C >= 0, when a new pair has s.y <= 1e-12, and when the
// step is not downhill on the modified force (then a steepest-descent step of 0.01 A per
// eV/A).  Every atom's step is capped at max_step; x1 receives the moved x + Delta N.
//
// The recursion runs on the coefficients of the step in the basis {s_j, y_j, g} (the
// vector-free form of Chen, Wang and Zhou, NIPS 2014): the dot products it needs are the
// Gram entries s_i.y_j and y_i.y_j, kept per walker and extended by one row and column per
// stored pair, and g.s_j, g.y_j, g.g of this step.  One pass over the walker forms the new
// pair and gathers those 5 m dot products, thread 0 runs the two loops on them (2 m^2
// multiply-adds), one pass forms the step and its largest atom move, one moves the walker.
// Every thread ends with the same st.
__device__ void lbfgs_translate(Team& team, const WalkDev& w, const DimerDev& P, const LbfgsDev& lb, int k,
                                double* x, double* x1, const double* F0, const double* Nk, double fn,
                                WalkerState& st, double* red, double* part, double* out, double* gram,
                                double* coef)
{
    const int a0 = w.begin[k], n = w.natoms[k];
    if (AKMC_BAD(a0 < 0 || n < 0 || a0 + n > w.n_total, 1, k)) return;
    const size_t slot = 3 * (size_t)w.n_total;
    const size_t base = 3 * (size_t)a0;
    double* r = lb.r + base;
    double* xp = lb.xp + base;
    double* gp = lb.gp + base;
    const int mem = min(P.lbfgs_memory, kLbfgsMem);
    const double L[3] = {w_box_len(w, k, 0), w_box_len(w, k, 1), w_box_len(w, k, 2)};
    int nuse = 0;                                 // stored pairs the step combines
    double cN = 0.0, cg = 0.0;                    // step = cN N + cg g + sum cS S + cY Y
    const double* Sb = lb.S + base;
    const double* Yb = lb.Y + base;
    size_t so[kLbfgsMem];                         // slot offset of each stored pair, newest first
    if (!(st.curvature < 0.0)) {
        st.lb_count = 0;
        st.lb_prev = 0;
        cN = (fn <= 0.0 ? 1.0 : -1.0) * P.convex_step;
    } else {
        const bool push = st.lb_prev;
        const int h = st.lb_head;
        const int nold = push ? min(st.lb_count, mem - 1) : 0;     // pairs that stay
        double* gw = lb.gram + (size_t)k * 2 * kLbfgsMem * kLbfgsMem;
        for (int t = threadIdx.x; t < 2 * kLbfgsMem * kLbfgsMem; t += blockDim.x) gram[t] = gw[t];
        __syncthreads();
        #pragma unroll
        for (int j = 0; j < kLbfgsMem; j++) so[j] = (size_t)((h - j + 2 * mem) % mem) * slot;  // j = 0: new pair
        double* Sn = lb.S + (size_t)h * slot + base;
        double* Yn = lb.Y + (size_t)h * slot + base;
        // acc[0..4]: s.y, y.y, g.s, g.y, g.g of the new pair and g; acc[5 j + 0..4] for the
        // stored pair j (1 = newest): s.Y_j, y.S_j, y.Y_j, g.S_j, g.Y_j
        // Two passes keep the accumulators of a thread at 20: the first forms the pair and
        // takes the stored pairs 1..3, the second (from the stored s and y) pairs 4..7.
        constexpr int kHalf = kLbfgsDots / 2;
        {
            double acc[kHalf];
            #pragma unroll
            for (int j = 0; j < kHalf; j++) acc[j] = 0.0;
            for (int a = team.first(); a < n; a += team.stride()) {
                #pragma unroll
                for (int d = 0; d < 3; d++) {
                    const int i = 3 * a + d;
                    const double gi = -(F0[i] - 2.0 * fn * Nk[i]);
                    const double xi = x[i];
                    if (push) {
                        double sv = xi - xp[i];
                        sv -= L[d] * rint(sv / L[d]);               // positions are wrapped in place
                        const double yv = gi - gp[i];
                        Sn[i] = sv;
                        Yn[i] = yv;
                        acc[0] += sv * yv;
                        acc[1] += yv * yv;
                        acc[2] += gi * sv;
                        acc[3] += gi * yv;
                        #pragma unroll
                        for (int j = 1; j < kHalf / 5; j++) {
                            if (j <= nold) {
                                const double sj = Sb[so[j] + i], yj = Yb[so[j] + i];
                                acc[5 * j + 0] += sv * yj;
                                acc[5 * j + 1] += yv * sj;
                                acc[5 * j + 2] += yv * yj;
                                acc[5 * j + 3] += gi * sj;
                                acc[5 * j + 4] += gi * yj;
                            }
                        }
                    }
                    acc[4] += gi * gi;
                    xp[i] = xi;
                    gp[i] = gi;
                }
            }
            team_reduce<kHalf, 0>(team, acc, red, part, out);
        }
        if (nold >= kHalf / 5) {
            double acc[kHalf];
            #pragma unroll
            for (int j = 0; j < kHalf; j++) acc[j] = 0.0;
            for (int a = team.first(); a < n; a += team.stride()) {
                #pragma unroll
                for (int d = 0; d < 3; d++) {
                    const int i = 3 * a + d;
                    const double sv = Sn[i], yv = Yn[i], gi = gp[i];
                    #pragma unroll
                    for (int j = kHalf / 5; j < kLbfgsMem; j++) {
                        if (j <= nold) {
                            const double sj = Sb[so[j] + i], yj = Yb[so[j] + i];
                            acc[5 * j - kHalf + 0] += sv * yj;
                            acc[5 * j - kHalf + 1] += yv * sj;
                            acc[5 * j - kHalf + 2] += yv * yj;
                            acc[5 * j - kHalf + 3] += gi * sj;
                            acc[5 * j - kHalf + 4] += gi * yj;
                        }
                    }
                }
            }
            team_reduce<kHalf, 0>(team, acc, red, part, out + kHalf);
        }
        // the new pair (the same decision in every thread)
        int count = st.lb_count;
        if (push) {
            if (out[0] > 1e-12) {
                st.lb_rho[h] = 1.0 / out[0];
                st.lb_head = (h + 1) % mem;
                count = nold + 1;
            } else {
                count = 0;
            }
        }
        if (threadIdx.x == 0) {
            double* SY = gram;                                      // [slot i][slot j] = s_i.y_j
            double* YY = gram + kLbfgsMem * kLbfgsMem;
            int sl[kLbfgsMem];
            #pragma unroll
            for (int j = 0; j < kLbfgsMem; j++) sl[j] = (h - j + 2 * mem) % mem;
            if (push && count > 0) {
                SY[h * kLbfgsMem + h] = out[0];
                YY[h * kLbfgsMem + h] = out[1];
                #pragma unroll
                for (int j = 1; j < kLbfgsMem; j++) {
                    if (j <= nold) {
                        SY[h * kLbfgsMem + sl[j]] = out[5 * j + 0];
                        SY[sl[j] * kLbfgsMem + h] = out[5 * j + 1];
                        YY[h * kLbfgsMem + sl[j]] = YY[sl[j] * kLbfgsMem + h] = out[5 * j + 2];
                    }
                }
                for (int t = 0; t < kLbfgsMem && team.rank == 0; t++) {
                    gw[h * kLbfgsMem + t] = SY[h * kLbfgsMem + t];
                    gw[t * kLbfgsMem + h] = SY[t * kLbfgsMem + h];
                    gw[kLbfgsMem * kLbfgsMem + h * kLbfgsMem + t] = YY[h * kLbfgsMem + t];
                    gw[kLbfgsMem * kLbfgsMem + t * kLbfgsMem + h] = YY[t * kLbfgsMem + h];
                }
            }
            // g.s and g.y of the stored pairs by age (0 = newest), then the two loops on the
            // coefficients: q = qg g + sum qa_l y_l, r = rg g + sum ra_l y_l + rb_l s_l
            auto gS = [&](int j) { return j == 0 ? out[2] : out[5 * j + 3]; };
            auto gY = [&](int j) { return j == 0 ? out[3] : out[5 * j + 4]; };
            auto rho = [&](int j) { return st.lb_rho[sl[j]]; };
            double qa[kLbfgsMem], al[kLbfgsMem], rb[kLbfgsMem];
            #pragma unroll
            for (int j = 0; j < kLbfgsMem; j++) {
                qa[j] = 0.0;
                al[j] = 0.0;
                rb[j] = 0.0;
            }
            const double gg = out[4];
            double qg = 1.0;
            #pragma unroll
            for (int j = 0; j < kLbfgsMem; j++) {                   // newest first
                if (j < count) {
                    double sq = qg * gS(j);
                    #pragma unroll
                    for (int l = 0; l < kLbfgsMem; l++)
                        if (l < count) sq += qa[l] * SY[sl[j] * kLbfgsMem + sl[l]];
                    al[j] = rho(j) * sq;
                    qa[j] -= al[j];
                }
            }
            const double gam = count > 0 ? (1.0 / rho(0)) / YY[sl[0] * kLbfgsMem + sl[0]] : 0.01;
            const double rg = gam * qg;
            #pragma unroll
            for (int j = 0; j < kLbfgsMem; j++) qa[j] *= gam;         // now ra
            #pragma unroll
            for (int j = kLbfgsMem - 1; j >= 0; j--) {              // oldest first
                if (j < count) {
                    double yr = rg * gY(j);
                    #pragma unroll
                    for (int l = 0; l < kLbfgsMem; l++) {
                        if (l < count)
                            yr += rb[l] * SY[sl[l] * kLbfgsMem + sl[j]] + qa[l] * YY[sl[l] * kLbfgsMem + sl[j]];
                    }
                    rb[j] += al[j] - rho(j) * yr;
                }
            }
            // the step is -r; keep it only if it goes down the modified force
            double rgd = rg * gg;
            #pragma unroll
            for (int l = 0; l < kLbfgsMem; l++)
                if (l < count) rgd += rb[l] * gS(l) + qa[l] * gY(l);
            const bool reset = !(-rgd < 0.0);
            #pragma unroll
            for (int j = 0; j < kLbfgsMem; j++) {
                coef[j] = reset || j >= count ? 0.0 : -rb[j];
                coef[kLbfgsMem + j] = reset || j >= count ? 0.0 : -qa[j];
            }
            coef[2 * kLbfgsMem] = reset ? -0.01 : -rg;
            coef[2 * kLbfgsMem + 1] = reset ? 0.0 : (double)count;
        }
        __syncthreads();
        nuse = (int)coef[2 * kLbfgsMem + 1];
        if (nuse == 0) st.lb_count = 0;
        else st.lb_count = count;
        cg = coef[2 * kLbfgsMem];
        st.lb_prev = 1;
        // slots by age after the push: age 0 is the new pair (slot h)
        #pragma unroll
        for (int j = 0; j < kLbfgsMem; j++) so[j] = (size_t)((st.lb_head - 1 - j + 2 * mem) % mem) * slot;
    }
    // the step and its largest atom move
    double m2[1] = {0.0};
    for (int a = team.first(); a < n; a += team.stride()) {
        double s2 = 0.0;
        #pragma unroll
        for (int d = 0; d < 3; d++) {
            const int i = 3 * a + d;
            double v = cN != 0.0 ? cN * Nk[i] : cg * gp[i];
            #pragma unroll
            for (int j = 0; j < kLbfgsMem; j++)
                if (j < nuse) v += coef[j] * Sb[so[j] + i] + coef[kLbfgsMem + j] * Yb[so[j] + i];
            r[i] = v;
            s2 += v * v;
        }
        m2[0] = fmax(m2[0], s2);
    }
    team_reduce<1, 1>(team, m2, red, part, out);
    const double mx = sqrt(out[0]);
    const double sc = mx > P.max_step ? P.max_step / mx : 1.0;
    // move (each thread reads the components it wrote) and the next iteration's second image
    for (int a = team.first(); a < n; a += team.stride()) {
        #pragma unroll
        for (int d = 0; d < 3; d++) {
            const int i = 3 * a + d;
            const double xi = x[i] + sc * r[i];
            x[i] = xi;
            x1[i] = xi + P.delta * Nk[i];
        }
    }
    st.iter += 1;
}

// Fit C(theta) through the trial, turn N to the fitted minimum, carry F1 along.  Returns
// false when the trial force call failed (st.status set).  Every thread ends with the
// same st.
__device__ bool rotate_finish_body(const WalkDev& w, const DimerDev& P, int k, double* F2,
                                   const double* Ft, const int* fstatus1, double* N,
                                   const double* theta, WalkerState& st, double* sh)
{
    if (fstatus1[k] != AKMC_OK) {
        st.status = AKMC_WALKER_FORCE_ERROR;
        return false;
    }
    const int a0 = w.begin[k], n = w.natoms[k];
    if (AKMC_BAD(a0 < 0 || n < 0 || a0 + n > w.n_total, 1, k)) {
        st.status = AKMC_WALKER_FORCE_ERROR;
        return false;
    }
    const double* F0 = F2 + 3 * (size_t)a0;
    double* F1 = F2 + 3 * ((size_t)w.n_total + a0);
    const double* F1t = Ft + 3 * (size_t)a0;
    double* Nk = N + 3 * (size_t)a0;
    const double* Th = theta + 3 * (size_t)a0;
    const double t1 = st.theta1, c1 = cos(t1), s1 = sin(t1);
    double dn = 0.0;
    for (int i = threadIdx.x; i < 3 * n; i += blockDim.x)
        dn += (F0[i] - F1t[i]) * (Nk[i] * c1 + Th[i] * s1);
    dn = block_sum(dn, sh);
    const double C0 = st.curvature, C1 = dn / P.delta, b1 = st.b1;
    const double a1 = (C0 - C1 + b1 * sin(2.0 * t1)) / (1.0 - cos(2.0 * t1));
    const double a0c = 2.0 * (C0 - a1);
    double tm = 0.5 * atan(b1 / a1);
    double Cm = 0.5 * a0c + a1 * cos(2.0 * tm) + b1 * sin(2.0 * tm);
    if (Cm > C0) {
        tm += 0.5 * kPi;
        Cm = 0.5 * a0c + a1 * cos(2.0 * tm) + b1 * sin(2.0 * tm);
    }
    const double cm = cos(tm), sm = sin(tm);
    double nn = 0.0;
    for (int i = threadIdx.x; i < 3 * n; i += blockDim.x) {
        const double y = Nk[i] * cm + Th[i] * sm;
        nn += y * y;
    }
    nn = block_sum(nn, sh);
    const double inv = 1.0 / sqrt(nn);
    const double w0 = sin(t1 - tm) / s1, w1 = sm / s1, wf = 1.0 - cm - sm * tan(0.5 * t1);
    for (int i = threadIdx.x; i < 3 * n; i += blockDim.x) {
        Nk[i] = (Nk[i] * cm + Th[i] * sm) * inv;
        F1[i] = w0 * F1[i] + w1 * F1t[i] + wf * F0[i];
    }
    st.curvature = Cm;
    __syncthreads();              // the new mode is complete before any thread reads it
    return true;
}

// A rotation that another rotation of the same iteration follows.
__global__ void __launch_bounds__(kWalkThreads)
dimer_rotate_finish_kernel(WalkDev w, DimerDev P, double* __restrict__ F2,
                           const double* __restrict__ Ft, const int* __restrict__ fstatus1,
                           double* __restrict__ N, const double* __restrict__ theta)
{
    __shared__ double sh[32];
    const int k = blockIdx.x;
    WalkerState st = w.st[k];
    if (st.status != 0 || !st.rotating) return;
    rotate_finish_body(w, P, k, F2, Ft, fstatus1, N, theta, st, sh);
    if (threadIdx.x == 0) w.st[k] = st;
}

// The end of an iteration: the last rotation (if the walker rotated), the saddle test at
// x, one translation step on the modified force, and the image x + Delta N of the next
// iteration's force call.  The rotation takes two passes over the walker: the first gathers
// the trial curvature, the norms of the two mode vectors (|N cos t + Theta sin t|^2 follows
// from N.N, N.Theta, Theta.Theta) and the largest atom force, the second turns N and gathers
// F0.N for the translation.  One cluster of CTAs per walker; the FIRE
// translation (fire_update) needs a cluster of one.
__global__ void __launch_bounds__(kFinishThreads, 2)
dimer_finish_translate_kernel(WalkDev w, DimerDev P, double* __restrict__ pos2,
                              double* __restrict__ F2, const double* __restrict__ Ft,
                              const int* __restrict__ fstatus1, const double* __restrict__ energy2,
                              const int* __restrict__ fstatus2, double* __restrict__ N,
                              const double* __restrict__ theta, double* __restrict__ v,
                              int* __restrict__ active2, LbfgsDev lb)
{
    __shared__ double sh[32];
    __shared__ double red[(kFinishThreads / 32) * kTeamMaxK];
    __shared__ double part[2 * kTeamMaxK];
    __shared__ double out[kLbfgsDots];
    __shared__ double gram[2 * kLbfgsMem * kLbfgsMem];
    __shared__ double coef[2 * kLbfgsMem + 2];
    Team team = make_team();
    const int k = blockIdx.x / team.size;
    WalkerState st = w.st[k];
    if (st.status != 0) {
        if (team.leader()) {
            active2[k] = 0;
            active2[w.W + k] = 0;
        }
        return;
    }
    const int a0 = w.begin[k], n = w.natoms[k];
    if (AKMC_BAD(a0 < 0 || n < 0 || a0 + n > w.n_total, 1, k)) return;
    const double* F0 = F2 + 3 * (size_t)a0;
    double* Nk = N + 3 * (size_t)a0;
    int done = 0;
    double fn = 0.0, fm = 0.0;
    if (st.rotating && fstatus1[k] != AKMC_OK) {
        done = AKMC_WALKER_FORCE_ERROR;
    } else if (st.rotating) {
        const double* F1t = Ft + 3 * (size_t)a0;
        const double* Th = theta + 3 * (size_t)a0;
        const double t1 = st.theta1, c1 = cos(t1), s1 = sin(t1);
        double g[5] = {0.0, 0.0, 0.0, 0.0, 0.0};    // (F0 - F1t).N', N.N, N.Theta, Theta.Theta; max |F0_a|^2
        for (int a = team.first(); a < n; a += team.stride()) {
            double f2 = 0.0;
            #pragma unroll
            for (int d = 0; d < 3; d++) {
                const int i = 3 * a + d;
                const double f0 = F0[i], nv = Nk[i], th = Th[i];
                g[0] += (f0 - F1t[i]) * (nv * c1 + th * s1);
                g[1] += nv * nv;
                g[2] += nv * th;
                g[3] += th * th;
                f2 += f0 * f0;
            }
            g[4] = fmax(g[4], f2);
        }
        team_reduce<5, 1>(team, g, red, part, out);
        fm = out[4];
        const double C0 = st.curvature, C1 = out[0] / P.delta, b1 = st.b1;
        const double a1 = (C0 - C1 + b1 * sin(2.0 * t1)) / (1.0 - cos(2.0 * t1));
        const double a0c = 2.0 * (C0 - a1);
        double tm = 0.5 * atan(b1 / a1);
        double Cm = 0.5 * a0c + a1 * cos(2.0 * tm) + b1 * sin(2.0 * tm);
        if (Cm > C0) {
            tm += 0.5 * kPi;
            Cm = 0.5 * a0c + a1 * cos(2.0 * tm) + b1 * sin(2.0 * tm);
        }
        const double cm = cos(tm), sm = sin(tm);
        const double nn = cm * cm * out[1] + 2.0 * cm * sm * out[2] + sm * sm * out[3];
        const double inv = 1.0 / sqrt(nn);
        // F1 is not carried to the turned mode here: the next iteration's first force call
        // evaluates it afresh (only a rotation that another one follows needs it carried)
        double f[1] = {0.0};
        for (int a = team.first(); a < n; a += team.stride()) {
            #pragma unroll
            for (int d = 0; d < 3; d++) {
                const int i = 3 * a + d;
                const double f0 = F0[i];
                const double nv = (Nk[i] * cm + Th[i] * sm) * inv;
                Nk[i] = nv;
                f[0] += f0 * nv;
            }
        }
        team_reduce<1, 0>(team, f, red, part, out);
        fn = out[0];
        st.curvature = Cm;
    } else {
        double g[2] = {0.0, 0.0};                   // F0.N; max |F0_a|^2
        for (int a = team.first(); a < n; a += team.stride()) {
            double f2 = 0.0;
            #pragma unroll
            for (int d = 0; d < 3; d++) {
                const int i = 3 * a + d;
                const double f0 = F0[i];
                g[0] += f0 * Nk[i];
                f2 += f0 * f0;
            }
            g[1] = fmax(g[1], f2);
        }
        team_reduce<2, 1>(team, g, red, part, out);
        fn = out[0];
        fm = out[1];
    }
    if (!done) {
        st.fmax = sqrt(fm);
        st.energy = energy2[5 * (size_t)k];
        if (st.iter == 0) st.e_start = st.energy;
        if (st.iter == 0 || st.fmax < 0.98 * st.best_fmax) {
            st.best_fmax = st.fmax;
            st.best_iter = st.iter;
        }
        if (fstatus2[k] != AKMC_OK || fstatus2[w.W + k] != AKMC_OK) done = AKMC_WALKER_FORCE_ERROR;
        else if (st.fmax < P.force_tol && st.curvature < P.max_eigenvalue) done = AKMC_WALKER_CONVERGED;
        else if (st.energy - st.e_start > P.max_rise) done = AKMC_WALKER_LOST;
        else if (st.iter >= P.max_iter) done = AKMC_WALKER_MAX_ITER;
        else if (P.patience > 0 && st.iter - st.best_iter > P.patience) done = AKMC_WALKER_MAX_ITER;
    }
    if (done) {
        if (team.leader()) {
            st.status = done;
            active2[k] = 0;
            active2[w.W + k] = 0;
            w.st[k] = st;
        }
        team_end(team);
        return;
    }
    const bool neg = st.curvature < 0.0;
    double* x = pos2 + 3 * (size_t)a0;
    double* x1 = pos2 + 3 * ((size_t)w.n_total + a0);
    if (P.translation == 1) {
        lbfgs_translate(team, w, P, lb, k, x, x1, F0, Nk, fn, st, red, part, out, gram, coef);
    } else {
        const double keep = neg ? 1.0 : 0.0, cf = neg ? 2.0 : 1.0;
        fire_update(st, P.n_min, P.dt_max, P.alpha0, P.alpha_dec, P.step_inc, P.step_dec, P.max_move,
                    [&](int i) { return keep * F0[i] - cf * fn * Nk[i]; }, x, v + 3 * (size_t)a0, n,
                    nullptr, sh);
        // the next iteration's second image (each thread reads the components it just wrote)
        for (int i = threadIdx.x; i < 3 * n; i += blockDim.x) x1[i] = x[i] + P.delta * Nk[i];
    }
    if (team.leader()) {
        st.calls += 2;
        active2[k] = 1;
        active2[w.W + k] = 1;
        w.st[k] = st;
        atomicAdd(w.running, 1);
    }
    team_end(team);
}

}  // namespace
}  // namespace akmc

using namespace akmc;

// ---------------------------------------------------------------------------------------
// host engine
// ---------------------------------------------------------------------------------------
// The per-size-class work-item table of a tuned batch (akmc_batch_autotune_classes).
struct TuneTable {
    int n = 0;
    int cells[16] = {0}, chunk[16] = {0};
    float ms[16] = {0.f};
};

struct akmc_walkers {
    akmc_field* field = nullptr;
    int W = 0, n_total = 0;
    std::vector<int> natoms, begin, label;
    std::vector<double> box, charge;
    bool has_frozen = false;
    double skin = 0.0;                 // EAM neighbour-list reuse between iterations, A
    akmc_batch* single = nullptr;      // W systems: FIRE forces, descriptors
    akmc_batch* tri = nullptr;         // 3 images of W systems: both Dimer ends, the rotation trial
    bool tuned_single = false, tuned_tri = false;
    TuneTable tune_single, tune_tri;
    DevBuf<int> d_begin, d_natoms, d_frozen, d_running, d_status1, d_status2, d_active1, d_active2;
    DevBuf<int> d_status3, d_active3;  // the Dimer's trial call on the image batch
    DevBuf<double> d_box;
    DevBuf<double> lbS, lbY, lbxp, lbgp, lbr, lbG;   // L-BFGS history of the Dimer translation
    DevBuf<double> pos1, F1, E1, pos2, F2, E2, v, N, theta;
    DevBuf<WalkerState> st;
    int* h_running = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;
    // captured iterations, valid for the parameters and work-item sizes they were made with
    cudaGraphExec_t fire_exec = nullptr, dimer_exec = nullptr;
    FireDev fire_key{};
    DimerDev dimer_key{};
    int fire_hc = -1, dimer_hc = -1;

    ~akmc_walkers()
    {
        if (fire_exec) cudaGraphExecDestroy(fire_exec);
        if (dimer_exec) cudaGraphExecDestroy(dimer_exec);
        if (single) akmc_batch_destroy(single);
        if (tri) akmc_batch_destroy(tri);
        if (h_running) cudaFreeHost(h_running);
        if (ev) cudaEventDestroy(ev);
        if (stream) cudaStreamDestroy(stream);
    }
    WalkDev dev() const
    {
        WalkDev d;
        d.W = W;
        d.n_total = n_total;
        d.begin = d_begin.p;
        d.natoms = d_natoms.p;
        d.box = d_box.p;
        d.frozen = has_frozen ? d_frozen.p : nullptr;
        d.st = st.p;
        d.running = d_running.p;
        return d;
    }
};

namespace {

// A walker kernel with `cluster` CTAs of kFinishThreads threads per walker, the CTAs of
// one walker forming one thread-block cluster.
template <class... KArgs, class... Args>
cudaError_t launch_team(void (*kernel)(KArgs...), int W, int cluster, cudaStream_t s, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(W * cluster), 1, 1);
    cfg.blockDim = dim3(kFinishThreads, 1, 1);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Replay a captured iteration until no walker is running (the count is read every
// `every` iterations) or the bound is reached.
akmc_status run_until_done(akmc_walkers* w, cudaGraphExec_t exec, int max_iter)
{
    const int every = 8;
    const int max_polls = max_iter / every + 3;
    for (int poll = 0; poll < max_polls; poll++) {
        for (int r = 0; r < every; r++) AKMC_CUDA(cudaGraphLaunch(exec, w->stream));
        AKMC_CUDA(cudaMemcpyAsync(w->h_running, w->d_running.p, sizeof(int), cudaMemcpyDeviceToHost, w->stream));
        AKMC_CUDA(cudaStreamSynchronize(w->stream));
        if (*w->h_running == 0) return AKMC_OK;
    }
    return fail(AKMC_ERR_STATE, "walkers still running past the iteration bound");
}

template <class Fn>
akmc_status capture(akmc_walkers* w, cudaGraphExec_t* exec, Fn&& body)
{
    if (*exec) {
        cudaGraphExecDestroy(*exec);
        *exec = nullptr;
    }
    cudaGraph_t g = nullptr;
    AKMC_CUDA(cudaStreamBeginCapture(w->stream, cudaStreamCaptureModeThreadLocal));
    akmc_status st = body();
    cudaError_t e = cudaStreamEndCapture(w->stream, &g);
    if (st) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) return fail(AKMC_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(AKMC_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    return AKMC_OK;
}

akmc_status read_results(akmc_walkers* w, akmc_walker_result* out)
{
    std::vector<WalkerState> h((size_t)w->W);
    AKMC_CUDA(cudaMemcpy(h.data(), w->st.p, sizeof(WalkerState) * w->W, cudaMemcpyDeviceToHost));
    for (int k = 0; k < w->W; k++) {
        const WalkerState& s = h[(size_t)k];
        out[k].status = s.status;
        out[k].iters = s.iter;
        out[k].force_calls = s.calls;
        out[k].reserved = 0;
        out[k].energy = s.energy;
        out[k].curvature = s.curvature;
        out[k].fmax = s.fmax;
        out[k].fnorm = s.fnorm;
    }
    return AKMC_OK;
}

// The work-item sizes of a batch, tuned per size class once on the first positions it sees;
// the table (cells per system of the class, chosen size, ms per call) is kept for reporting.
akmc_status tune(akmc_batch* b, double* pos, double* F, double* E, int* status, cudaStream_t s, bool* done,
                 TuneTable* table)
{
    if (*done) return AKMC_OK;
    akmc_status st = akmc_batch_autotune_classes(b, pos, F, E, status, s, &table->n, table->cells, table->chunk,
                                                 table->ms, 16);
    if (st) return st;
    *done = true;
    return AKMC_OK;
}

// Forget the neighbour lists of a batch (the next call rebuilds them), so that a walker
// call's results depend on its inputs only, not on lists left by an earlier call.
akmc_status reset_lists(akmc_batch* b, cudaStream_t s)
{
    if (b && b->view.skin > 0.0)
        AKMC_CUDA(cudaMemsetAsync(b->list_ok.p, 0, sizeof(int) * b->nsys, s));
    return AKMC_OK;
}

// run_batch with profiling events off (events cannot sit inside a captured graph)
akmc_status quiet_batch(akmc_batch* b, double* pos, double* F, double* E, int* status,
                        cudaStream_t s, const int* active)
{
    const bool on = b->timer.on;
    b->timer.on = false;
    akmc_status st = run_batch(b, pos, F, E, status, s, active);
    b->timer.on = on;
    return st;
}

}  // namespace

extern "C" {

void akmc_fire_defaults(akmc_fire_params* p)
{
    if (!p) return;
    p->max_iter = 3000;            // RelaxCntrl (Common/RelaxCntrl.h:15-38)
    p->n_min = 5;
    p->norm_tol = 1.0e-5;
    p->force_tol = 1.0e-4;
    p->dt0 = 0.0005;
    p->dt_max = 0.00075;
    p->alpha0 = 0.1;
    p->alpha_dec = 0.99;
    p->step_inc = 1.1;
    p->step_dec = 0.5;
    p->max_move = 0.0;
}

void akmc_dimer_defaults(akmc_dimer_params* p)
{
    if (!p) return;
    p->max_iter = 300;             // L-BFGS searches that converge do so within ~200 steps
    p->max_rotations = 1;
    p->n_min = 5;                  // DimerCntrl FIRE constants (Common/DimerCntrl.h:80-88)
    p->patience = 0;               // no stall rule
    p->delta = 0.01;               // dimerDisplacement
    p->rot_tol = 0.1;              // normTol
    p->force_tol = 1.0e-2;         // forceTol
    p->max_eigenvalue = 0.0;       // maxEigenvalue
    p->min_trial = 1.0e-3;
    p->max_move = 0.02;
    p->max_rise = 8.0;
    p->dt0 = 0.001;
    p->dt_max = 0.004;
    p->alpha0 = 0.1;
    p->alpha_dec = 0.99;
    p->step_inc = 1.1;
    p->step_dec = 0.5;
    p->translation = 1;            // L-BFGS on the modified force
    p->lbfgs_memory = 8;
    p->max_step = 0.2;
    p->convex_step = 0.05;
}

akmc_status akmc_walkers_create(akmc_field* f, int nwalk, const int* natoms, const double* box,
                                const int* label, const double* charge, const int* frozen,
                                akmc_walkers** out)
{
    if (!f || !out || nwalk < 1 || !natoms || !box || !label) return fail(AKMC_ERR_ARG, "bad walker arguments");
    *out = nullptr;
    auto w = std::make_unique<akmc_walkers>();
    w->field = f;
    w->W = nwalk;
    w->natoms.assign(natoms, natoms + nwalk);
    w->box.assign(box, box + 3 * (size_t)nwalk);
    int n = 0;
    for (int k = 0; k < nwalk; k++) {
        if (natoms[k] < 1) return fail(AKMC_ERR_ARG, "every walker needs at least one atom");
        w->begin.push_back(n);
        n += natoms[k];
    }
    w->n_total = n;
    w->label.assign(label, label + n);
    if (charge) w->charge.assign(charge, charge + n);
    // EAM walkers reuse neighbour lists between iterations (a FIRE or Dimer step moves an
    // atom by at most a few hundredths of an angstrom); 0.4 A unless every box is too small
    double minL = 1e300;
    for (int k = 0; k < 3 * nwalk; k++) minL = std::min(minL, box[k]);
    if (akmc_field_family(f) == AKMC_FAMILY_EAM && akmc_field_cutoff(f) + 0.4 <= 0.5 * minL) w->skin = 0.4;
    akmc_status st = akmc_batch_create_skin(f, nwalk, natoms, box, label, charge, w->skin, &w->single);
    if (st) return st;
    const size_t n3 = 3 * (size_t)n;
    AKMC_CUDA(cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking));
    AKMC_CUDA(cudaEventCreateWithFlags(&w->ev, cudaEventDisableTiming));
    AKMC_CUDA(cudaMallocHost(&w->h_running, sizeof(int)));
    AKMC_CUDA(w->d_begin.alloc(nwalk));
    AKMC_CUDA(w->d_natoms.alloc(nwalk));
    AKMC_CUDA(cudaMemcpy(w->d_begin.p, w->begin.data(), sizeof(int) * nwalk, cudaMemcpyHostToDevice));
    AKMC_CUDA(cudaMemcpy(w->d_natoms.p, natoms, sizeof(int) * nwalk, cudaMemcpyHostToDevice));
    AKMC_CUDA(w->d_box.alloc(3 * (size_t)nwalk));
    AKMC_CUDA(cudaMemcpy(w->d_box.p, box, sizeof(double) * 3 * nwalk, cudaMemcpyHostToDevice));
    if (frozen) {
        w->has_frozen = true;
        AKMC_CUDA(w->d_frozen.alloc((size_t)n));
        AKMC_CUDA(cudaMemcpy(w->d_frozen.p, frozen, sizeof(int) * n, cudaMemcpyHostToDevice));
    }
    AKMC_CUDA(w->d_running.alloc(1));
    AKMC_CUDA(w->d_status1.alloc(nwalk));
    AKMC_CUDA(w->d_active1.alloc(nwalk));
    AKMC_CUDA(w->pos1.alloc(n3));
    AKMC_CUDA(w->F1.alloc(n3));
    AKMC_CUDA(w->E1.alloc(5 * (size_t)nwalk));
    AKMC_CUDA(w->v.alloc(n3));
    AKMC_CUDA(w->st.alloc(nwalk));
    *out = w.release();
    return AKMC_OK;
}

akmc_status akmc_walkers_destroy(akmc_walkers* w)
{
    if (w && w->stream) cudaStreamSynchronize(w->stream);
    delete w;
    return AKMC_OK;
}

int akmc_walkers_count(const akmc_walkers* w) { return w ? w->W : 0; }

akmc_status akmc_walkers_set_skin(akmc_walkers* w, double skin)
{
    if (!w || !(skin >= 0.0)) return fail(AKMC_ERR_ARG, "bad skin");
    AKMC_CUDA(cudaStreamSynchronize(w->stream));
    if (w->fire_exec) cudaGraphExecDestroy(w->fire_exec);
    if (w->dimer_exec) cudaGraphExecDestroy(w->dimer_exec);
    w->fire_exec = w->dimer_exec = nullptr;
    akmc_batch* nb = nullptr;
    akmc_status st = akmc_batch_create_skin(w->field, w->W, w->natoms.data(), w->box.data(), w->label.data(),
                                           w->charge.empty() ? nullptr : w->charge.data(), skin, &nb);
    if (st) return st;
    akmc_batch_destroy(w->single);
    w->single = nb;
    if (w->tri) {
        akmc_batch_destroy(w->tri);
        w->tri = nullptr;
        w->pos2.release();                  // dimer_buffers makes them again with the new batch
    }
    w->skin = skin;
    w->tuned_single = w->tuned_tri = false;
    return AKMC_OK;
}

double akmc_walkers_skin(const akmc_walkers* w) { return w ? w->skin : 0.0; }

akmc_status akmc_walkers_skip_tuning(akmc_walkers* w)
{
    if (!w) return fail(AKMC_ERR_ARG, "null walker set");
    w->tuned_single = w->tuned_tri = true;
    return AKMC_OK;
}

int akmc_walkers_tuning(const akmc_walkers* w, int which, int* cells, int* chunk, float* ms, int max)
{
    if (!w) return 0;
    const TuneTable& t = which == 0 ? w->tune_single : w->tune_tri;
    for (int c = 0; c < t.n && c < max; c++) {
        if (cells) cells[c] = t.cells[c];
        if (chunk) chunk[c] = t.chunk[c];
        if (ms) ms[c] = t.ms[c];
    }
    return t.n;
}

akmc_status akmc_walkers_relax(akmc_walkers* w, double* pos, const akmc_fire_params* p,
                               akmc_walker_result* out, void* stream)
{
    return akmc_walkers_relax_subset(w, pos, p, nullptr, out, stream);
}

akmc_status akmc_walkers_relax_subset(akmc_walkers* w, double* pos, const akmc_fire_params* p,
                                      const int* run_mask, akmc_walker_result* out, void* stream)
{
    if (!w || !pos || !p || !out) return fail(AKMC_ERR_ARG, "null argument");
    if (p->max_iter < 1) return fail(AKMC_ERR_ARG, "max_iter must be positive");
    cudaStream_t us = (cudaStream_t)stream;
    cudaStream_t s = w->stream;
    const size_t n3 = 3 * (size_t)w->n_total;
    FireDev P{};
    P.max_iter = p->max_iter;
    P.n_min = p->n_min;
    P.norm_tol = p->norm_tol;
    P.force_tol = p->force_tol;
    P.dt0 = p->dt0;
    P.dt_max = p->dt_max;
    P.alpha0 = p->alpha0;
    P.alpha_dec = p->alpha_dec;
    P.step_inc = p->step_inc;
    P.step_dec = p->step_dec;
    P.max_move = p->max_move;
    AKMC_CUDA(cudaEventRecord(w->ev, us));              // after the caller's writes to pos
    AKMC_CUDA(cudaStreamWaitEvent(s, w->ev, 0));
    AKMC_CUDA(cudaMemcpyAsync(w->pos1.p, pos, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
    akmc_status st = AKMC_OK;
    if (!w->tuned_single) {
        if ((st = tune(w->single, w->pos1.p, w->F1.p, w->E1.p, w->d_status1.p, s, &w->tuned_single,
                       &w->tune_single)))
            return st;
        // tuning wrapped its positions in place: start from the caller's copy
        AKMC_CUDA(cudaMemcpyAsync(w->pos1.p, pos, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
    }
    if ((st = reset_lists(w->single, s))) return st;
    const WalkDev d = w->dev();
    walkers_init_kernel<<<w->W, kWalkThreads, 0, s>>>(d, P.dt0, P.alpha0, w->v.p, nullptr, w->d_active1.p, 1,
                                                      run_mask);
    AKMC_CUDA(cudaGetLastError());
    if ((st = quiet_batch(w->single, w->pos1.p, w->F1.p, w->E1.p, w->d_status1.p, s,
                          run_mask ? w->d_active1.p : nullptr)))
        return st;
    fire_check_kernel<<<w->W, kWalkThreads, 0, s>>>(d, P, w->v.p, w->F1.p, w->E1.p, w->d_status1.p);
    AKMC_CUDA(cudaGetLastError());
    fire_step_kernel<<<w->W, kWalkThreads, 0, s>>>(d, P, w->pos1.p, w->v.p, w->F1.p, w->d_active1.p);
    AKMC_CUDA(cudaGetLastError());
    const int hc = akmc_batch_total_items(w->single);     // the plan the captured grids are sized for
    if (!w->fire_exec || std::memcmp(&P, &w->fire_key, sizeof(P)) != 0 || hc != w->fire_hc) {
        st = capture(w, &w->fire_exec, [&]() -> akmc_status {
            AKMC_CUDA(cudaMemsetAsync(w->d_running.p, 0, sizeof(int), s));
            akmc_status s2 = quiet_batch(w->single, w->pos1.p, w->F1.p, w->E1.p, w->d_status1.p, s, w->d_active1.p);
            if (s2) return s2;
            fire_check_step_kernel<<<w->W, kWalkThreads, 0, s>>>(d, P, w->pos1.p, w->v.p, w->F1.p, w->E1.p,
                                                                  w->d_status1.p, w->d_active1.p);
            AKMC_CUDA(cudaGetLastError());
            return AKMC_OK;
        });
        if (st) return st;
        w->fire_key = P;
        w->fire_hc = hc;
    }
    if ((st = run_until_done(w, w->fire_exec, P.max_iter))) return st;
    AKMC_CUDA(cudaMemcpyAsync(pos, w->pos1.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
    AKMC_CUDA(cudaStreamSynchronize(s));
    return read_results(w, out);
}

akmc_status akmc_walkers_dimer(akmc_walkers* w, double* pos, double* mode,
                               const akmc_dimer_params* p, akmc_walker_result* out, void* stream)
{
    return akmc_walkers_dimer_subset(w, pos, mode, p, nullptr, out, stream);
}

akmc_status akmc_walkers_dimer_subset(akmc_walkers* w, double* pos, double* mode,
                                      const akmc_dimer_params* p, const int* run_mask,
                                      akmc_walker_result* out, void* stream)
{
    if (!w || !pos || !mode || !p || !out) return fail(AKMC_ERR_ARG, "null argument");
    if (p->max_iter < 1 || p->max_rotations < 1 || !(p->delta > 0.0) ||
        (p->translation != 0 && p->translation != 1) ||
        (p->translation == 1 && !(p->max_step > 0.0 && p->convex_step > 0.0)))
        return fail(AKMC_ERR_ARG, "bad dimer parameters");
    cudaStream_t us = (cudaStream_t)stream;
    cudaStream_t s = w->stream;
    const size_t n3 = 3 * (size_t)w->n_total;
    akmc_status st;
    if (!w->tri) {
        // images 0 and 1 (x, x + Delta N) run in the first force call of an iteration, image 2
        // (the rotation trial) in the second: two masks and two status arrays over the 3W
        // systems, each zero outside its images
        if ((st = batch_create_images(w->field, w->W, 3, w->natoms.data(), w->box.data(), w->label.data(),
                                      w->charge.empty() ? nullptr : w->charge.data(), w->skin, &w->tri)))
            return st;
        AKMC_CUDA(w->pos2.alloc(3 * n3));
        AKMC_CUDA(w->F2.alloc(3 * n3));
        AKMC_CUDA(w->E2.alloc(15 * (size_t)w->W));
        AKMC_CUDA(w->d_status2.alloc(3 * (size_t)w->W));
        AKMC_CUDA(w->d_active2.alloc(3 * (size_t)w->W));
        AKMC_CUDA(w->d_status3.alloc(3 * (size_t)w->W));
        AKMC_CUDA(w->d_active3.alloc(3 * (size_t)w->W));
        AKMC_CUDA(cudaMemset(w->d_active2.p, 0, sizeof(int) * 3 * (size_t)w->W));
        AKMC_CUDA(cudaMemset(w->d_active3.p, 0, sizeof(int) * 3 * (size_t)w->W));
        AKMC_CUDA(w->N.alloc(n3));
        AKMC_CUDA(w->theta.alloc(n3));
        AKMC_CUDA(w->lbS.alloc((size_t)kLbfgsMem * n3));
        AKMC_CUDA(w->lbY.alloc((size_t)kLbfgsMem * n3));
        AKMC_CUDA(w->lbxp.alloc(n3));
        AKMC_CUDA(w->lbgp.alloc(n3));
        AKMC_CUDA(w->lbr.alloc(n3));
        AKMC_CUDA(w->lbG.alloc((size_t)2 * kLbfgsMem * kLbfgsMem * w->W));
    }
    DimerDev P{};
    P.max_iter = p->max_iter;
    P.max_rotations = p->max_rotations;
    P.n_min = p->n_min;
    P.patience = std::max(0, p->patience);
    P.delta = p->delta;
    P.rot_tol = p->rot_tol;
    P.force_tol = p->force_tol;
    P.max_eigenvalue = p->max_eigenvalue;
    P.min_trial = p->min_trial;
    P.max_move = p->max_move;
    P.max_rise = p->max_rise;
    P.dt0 = p->dt0;
    P.dt_max = p->dt_max;
    P.alpha0 = p->alpha0;
    P.alpha_dec = p->alpha_dec;
    P.step_inc = p->step_inc;
    P.step_dec = p->step_dec;
    P.translation = p->translation;
    P.lbfgs_memory = std::max(1, std::min(p->lbfgs_memory, kLbfgsMem));
    P.max_step = p->max_step;
    P.convex_step = p->convex_step;
    AKMC_CUDA(cudaEventRecord(w->ev, us));              // after the caller's writes
    AKMC_CUDA(cudaStreamWaitEvent(s, w->ev, 0));
    for (int m = 0; m < 3; m++)
        AKMC_CUDA(cudaMemcpyAsync(w->pos2.p + m * n3, pos, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
    AKMC_CUDA(cudaMemcpyAsync(w->N.p, mode, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
    if ((st = tune(w->tri, w->pos2.p, w->F2.p, w->E2.p, w->d_status2.p, s, &w->tuned_tri, &w->tune_tri)))
        return st;
    // tuning wrapped its positions in place: start from the caller's copy
    AKMC_CUDA(cudaMemcpyAsync(w->pos2.p, pos, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
    if ((st = reset_lists(w->tri, s))) return st;
    const WalkDev d = w->dev();
    walkers_init_kernel<<<w->W, kWalkThreads, 0, s>>>(d, P.dt0, P.alpha0, w->v.p, w->N.p, w->d_active2.p, 2,
                                                      run_mask);
    AKMC_CUDA(cudaGetLastError());
    dimer_ends_kernel<<<w->W, kWalkThreads, 0, s>>>(d, P, w->pos2.p, w->N.p, w->d_active2.p);
    AKMC_CUDA(cudaGetLastError());
    const int hc = akmc_batch_total_items(w->tri);        // the plan the captured grids are sized for
    if (!w->dimer_exec || std::memcmp(&P, &w->dimer_key, sizeof(P)) != 0 || hc != w->dimer_hc) {
        st = capture(w, &w->dimer_exec, [&]() -> akmc_status {
            // images x, x + Delta N of every running walker are in place (the previous
            // iteration's last kernel, or dimer_ends before the loop)
            AKMC_CUDA(cudaMemsetAsync(w->d_running.p, 0, sizeof(int), s));
            akmc_status s2 = quiet_batch(w->tri, w->pos2.p, w->F2.p, w->E2.p, w->d_status2.p, s, w->d_active2.p);
            if (s2) return s2;
            auto freeze = [&](int images) -> akmc_status {
                if (!w->has_frozen) return AKMC_OK;
                dimer_freeze_kernel<<<(w->n_total + 255) / 256, 256, 0, s>>>(w->d_frozen.p, w->n_total, images,
                                                                               w->F2.p);
                AKMC_CUDA(cudaGetLastError());
                return AKMC_OK;
            };
            if ((s2 = freeze(2))) return s2;
            // the rotation trial is image 2: its positions, forces, status and mask
            double* xt = w->pos2.p + 2 * n3;
            double* Ft = w->F2.p + 2 * n3;
            int* st_t = w->d_status3.p + 2 * w->W;
            int* act_t = w->d_active3.p + 2 * w->W;
            for (int r = 0; r < P.max_rotations; r++) {
                AKMC_CUDA(launch_team(dimer_rotate_prep_kernel, w->W, kWalkCluster, s, d, P, r, w->pos2.p,
                                      (const double*)w->F2.p, (const double*)w->N.p, w->theta.p, xt, act_t));
                // the rotation needs the trial forces only
                if ((s2 = quiet_batch(w->tri, w->pos2.p, w->F2.p, nullptr, w->d_status3.p, s, w->d_active3.p)))
                    return s2;
                if ((s2 = freeze(3))) return s2;
                if (r + 1 < P.max_rotations) {
                    dimer_rotate_finish_kernel<<<w->W, kWalkThreads, 0, s>>>(d, P, w->F2.p, Ft, st_t, w->N.p,
                                                                              w->theta.p);
                    AKMC_CUDA(cudaGetLastError());
                }
            }
            LbfgsDev lb{w->lbS.p, w->lbY.p, w->lbxp.p, w->lbgp.p, w->lbr.p, w->lbG.p};
            // the FIRE translation runs one CTA per walker
            AKMC_CUDA(launch_team(dimer_finish_translate_kernel, w->W, P.translation == 1 ? kWalkCluster : 1, s,
                                  d, P, w->pos2.p, w->F2.p, (const double*)Ft, (const int*)st_t,
                                  (const double*)w->E2.p, (const int*)w->d_status2.p, w->N.p,
                                  (const double*)w->theta.p, w->v.p, w->d_active2.p, lb));
            return AKMC_OK;
        });
        if (st) return st;
        w->dimer_key = P;
        w->dimer_hc = hc;
    }
    if ((st = run_until_done(w, w->dimer_exec, P.max_iter))) return st;
    AKMC_CUDA(cudaMemcpyAsync(pos, w->pos2.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
    AKMC_CUDA(cudaMemcpyAsync(mode, w->N.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
    AKMC_CUDA(cudaStreamSynchronize(s));
    return read_results(w, out);
}

akmc_status akmc_walkers_descriptors(akmc_walkers* w, const double* pos, float* desc, float* basis,
                                     void* stream)
{
    if (!w || !pos || !desc) return fail(AKMC_ERR_ARG, "null argument");
    cudaStream_t us = (cudaStream_t)stream;
    cudaStream_t s = w->stream;
    const size_t n3 = 3 * (size_t)w->n_total;
    AKMC_CUDA(cudaEventRecord(w->ev, us));              // after the caller's writes to pos
    AKMC_CUDA(cudaStreamWaitEvent(s, w->ev, 0));
    AKMC_CUDA(cudaMemcpyAsync(w->pos1.p, pos, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
    akmc_status st = AKMC_OK;
    if ((st = reset_lists(w->single, s))) return st;
    if ((st = quiet_batch(w->single, w->pos1.p, w->F1.p, w->E1.p, w->d_status1.p, s, nullptr))) return st;
    if ((st = akmc_batch_descriptors(w->single, desc, basis, s))) return st;
    AKMC_CUDA(cudaEventRecord(w->ev, s));               // the caller's stream sees the results
    AKMC_CUDA(cudaStreamWaitEvent(us, w->ev, 0));
    return AKMC_OK;
}

akmc_status akmc_walkers_descriptors_rows(akmc_walkers* w, const double* pos, const int* rows, int n_rows,
                                          float* desc, float* basis, void* stream)
{
    if (!w || !pos || n_rows < 0 || (n_rows > 0 && (!rows || !desc))) return fail(AKMC_ERR_ARG, "bad arguments");
    cudaStream_t us = (cudaStream_t)stream;
    cudaStream_t s = w->stream;
    const size_t n3 = 3 * (size_t)w->n_total;
    AKMC_CUDA(cudaEventRecord(w->ev, us));              // after the caller's writes to pos and rows
    AKMC_CUDA(cudaStreamWaitEvent(s, w->ev, 0));
    AKMC_CUDA(cudaMemcpyAsync(w->pos1.p, pos, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
    akmc_status st = AKMC_OK;
    if ((st = reset_lists(w->single, s))) return st;
    if ((st = quiet_batch(w->single, w->pos1.p, w->F1.p, w->E1.p, w->d_status1.p, s, nullptr))) return st;
    if ((st = akmc_batch_descriptors_rows(w->single, rows, n_rows, desc, basis, s))) return st;
    AKMC_CUDA(cudaEventRecord(w->ev, s));
    AKMC_CUDA(cudaStreamWaitEvent(us, w->ev, 0));
    return AKMC_OK;
}

}  // extern "C"
