/* akmc.h -- C ABI of the B200-native AKMC force/energy path.
 *
 * The reference has no FFI: its force path is the C++ class Field, chosen at compile
 * time (potentials/metal/Field.h:126-219 for EAM metals, potentials/pair/Field.h:
 * 658-748 for Buckingham + Ewald ionics).  Every optimiser reaches it through one call,
 * Field::calculateForces (metal/Field.h:192-193).  The entry points below are the
 * C-ABI equivalents of those methods; akmc_b200/cpp/Field.h wraps them in a
 * C++ class with the reference's method signatures, and akmc_b200/field.py in a
 * Python class for tests and benchmarks.
 *
 * Conventions
 * - Every call returns an akmc_status (0 = success).  Nothing here calls exit() or
 *   traps; kernels report range errors through per-system status words.
 * - Units: Angstrom, eV, eV/Angstrom, charges in e (Coulomb prefactor 14.3996454784).
 * - Lattice vectors are the rows of lat[9] (a = lat[0..2], b = lat[3..5],
 *   c = lat[6..8]); only orthorhombic cells are supported, as in the reference's Ewald
 *   half-space weighting (potentials/pair/Ewald.cpp:304-311).
 * - One akmc_field per thread or stream: a field owns device scratch; calls on one
 *   field must not overlap.  There is no hidden global state.
 * - Device pointers are plain CUDA device addresses; streams are cudaStream_t passed
 *   as void* so that this header needs no CUDA include.
 */
#ifndef AKMC_H
#define AKMC_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int akmc_status;

enum {
    AKMC_OK = 0,
    AKMC_ERR_ARG = 1,            /* null pointer, bad size, bad index */
    AKMC_ERR_EMBED_RANGE = 2,    /* rho outside the embedding table (ManyBody.cpp:603-608) */
    AKMC_ERR_TABLE_RANGE = 3,    /* pair distance below the first table bin */
    AKMC_ERR_CUTOFF = 4,         /* cutoff + shell > half the smallest cell width (Field.cpp:99-106) */
    AKMC_ERR_IO = 5,             /* potentials / table file missing */
    AKMC_ERR_PARSE = 6,          /* unknown keyword or malformed entry */
    AKMC_ERR_UNSUPPORTED = 7,    /* non-orthorhombic cell, potential form not on this path */
    AKMC_ERR_CUDA = 8,           /* CUDA runtime error (message in akmc_last_error) */
    AKMC_ERR_NONFINITE = 9,      /* NaN / Inf position or force */
    AKMC_ERR_STATE = 10,         /* call order: setup before forces, batch before use */
    AKMC_ERR_CAPACITY = 11       /* more atoms, cells or systems than the field was set up for */
};

/* Potential families (the reference's two compile-time Field variants). */
enum { AKMC_FAMILY_EAM = 1, AKMC_FAMILY_IONIC = 2 };

/* Arithmetic of the pair terms.  Geometry (separations, minimum image, r) and all
 * accumulations are FP64 in every mode. */
enum {
    AKMC_PREC_MIXED = 0,         /* pair terms FP32, accumulation FP64 (default) */
    AKMC_PREC_FP64 = 1           /* pair terms FP64 */
};

/* Energy record: the fields of the reference's Energy class (metal/Energy.h:13-108)
 * that Field::calculateForces writes.  total = rcp + real + vdw + many. */
typedef struct {
    double total;
    double rcp;    /* Ewald reciprocal space */
    double real;   /* Ewald real space, self term included */
    double vdw;    /* short-range pair (Buckingham) or EAM pair */
    double many;   /* EAM embedding */
} akmc_energy;

typedef struct akmc_field akmc_field;
typedef struct akmc_batch akmc_batch;

/* ---- lifetime --------------------------------------------------------------------- */

/* Read a reference-format `potentials` file: Field::readPotential
 * (potentials/metal/Field.cpp:122-205, potentials/pair/Field.cpp:215-317), including
 * the species block (potentials/Species.cpp:31-70), EAM setfl tables
 * (MetalPotential.cpp:276-361) and Buckingham entries (TwoBody.cpp:56-266). */
akmc_status akmc_field_create(const char* potentials_path, akmc_field** out);

/* The same reader on the text of a potentials file, for callers that hold the file as
 * a stream (Field::readPotential takes a std::ifstream).  Table files named inside are
 * opened relative to the working directory, as the reference opens them. */
akmc_status akmc_field_create_from_text(const char* text, akmc_field** out);

/* Field::setup (potentials/metal/Field.cpp:24-97, potentials/pair/Field.cpp:80-169):
 * cutoff check against the cell, Ewald eta and k-vector set for lat, device tables.
 * rcp may be NULL (computed from lat).  max_atoms bounds the single-system path. */
akmc_status akmc_field_setup(akmc_field* f, const double lat[9], const double rcp[9],
                             int max_atoms);

/* ~Field (metal/Field.cpp:12-16): frees device and host resources. */
akmc_status akmc_field_destroy(akmc_field* f);

/* ---- the reference call ----------------------------------------------------------- */

/* Field::calculateForces (potentials/metal/Field.h:192-193; pair/Field.cpp:323-381).
 * Host SoA buffers, reference semantics: forces and stress are overwritten, positions
 * are wrapped into the minimum-image cell IN PLACE, charge is per atom (ignored by
 * EAM), atmLabel indexes the species block.  lat must equal the setup lattice.
 * stress is written as zeros (no optimiser on this path reads it). */
akmc_status akmc_forces(akmc_field* f, int n, double* posX, double* posY, double* posZ,
                        const int* atmLabel, const double* charge, double* forceX,
                        double* forceY, double* forceZ, double stress[6], akmc_energy* out);

/* ---- batched, device-resident path (new: walkers of uneven size) -------------------- */

/* Plan a batch of nsys independent systems: natoms[s] atoms in an orthorhombic box
 * box[3*s .. 3*s+2] (host arrays).  Atoms of system s occupy rows
 * [offset_s, offset_s + natoms[s]) of every per-atom device array, offsets being the
 * prefix sums of natoms.  label[] and charge[] (host, per atom, batch order) are
 * uploaded once.  For the ionic family every box must equal the setup cell. */
akmc_status akmc_batch_create(akmc_field* f, int nsys, const int* natoms, const double* box,
                              const int* label, const double* charge, akmc_batch** out);

/* The same batch with EAM neighbour lists reused across calls: each system's list holds
 * the pairs within cutoff + skin (A) at the positions of its last rebuild and serves every
 * later call until some atom of that system has moved more than skin/2; the pair terms
 * still take exactly the pairs with rsq <= cutoff^2 (the reference criterion).  For callers
 * whose consecutive calls move atoms a little (relaxation and saddle-search steps).
 * cutoff + skin must not exceed half the smallest box length.  Ignored (skin 0) for the
 * ionic family.  Summation order follows the list, so results can differ in the last bits
 * from a batch without skin. */
akmc_status akmc_batch_create_skin(akmc_field* f, int nsys, const int* natoms, const double* box,
                                   const int* label, const double* charge, double skin,
                                   akmc_batch** out);

akmc_status akmc_batch_destroy(akmc_batch* b);

/* What the last force call did with each system's neighbour list (host int[nsys]):
 * 0 no skin (cells scanned), 1 list rebuilt, 2 list reused.  Synchronises the device. */
akmc_status akmc_batch_list_modes(akmc_batch* b, int* modes);

/* Forces and energies for every system of the batch, asynchronously on `stream`.
 *   pos_dev     double[n_total*3]  xyz rows; wrapped into the minimum-image cell in place
 *   force_dev   double[n_total*3]  written
 *   energy_dev  double[nsys*5]     written: total, rcp, real, vdw, many per system
 *   status_dev  int[nsys]          written: AKMC_OK or the first error of that system
 * No host synchronisation, no allocation: the call can be replayed or captured. */
akmc_status akmc_batch_forces(akmc_batch* b, double* pos_dev, double* force_dev,
                              double* energy_dev, int* status_dev, void* stream);

/* The same call on HOST buffers (pageable or pinned): copies the positions in, runs the
 * batch on `stream`, copies wrapped positions, forces, energies and statuses back and
 * synchronises `stream` before returning.  Device buffers are allocated on first use.
 * This is the batched form of akmc_forces for callers whose walkers live in host memory. */
akmc_status akmc_batch_forces_host(akmc_batch* b, double* pos, double* force, double* energy,
                                   int* status, void* stream);

/* Neighbour sets the last EAM force call of this batch used: for every atom, the atoms
 * j != i within the cutoff under the minimum image (rsq <= rc^2), the criterion of the
 * reference's neighbour list (potentials/metal/NbrListPBC.cpp:41-125).  Host arrays in
 * the caller's atom numbering: counts[n_total]; nbrs[n_total * max_per_atom], each row
 * sorted ascending and padded with -1.  Synchronises the device.  For testing and
 * inspection; EAM batches only.  With a skin the rows hold the pairs within cutoff + skin
 * at the last rebuild. */
akmc_status akmc_batch_neighbours(akmc_batch* b, int* counts, int* nbrs, int max_per_atom);

/* Work decomposition of the pair kernels: home atoms per CTA work item (8, 16 or 32).
 * akmc_batch_create picks one from the batch size; akmc_batch_autotune times all three
 * on the caller's buffers (3 calls each after a warm-up) and keeps the fastest, writing
 * it to *chosen.  Both synchronise the device; call them between force calls, not during
 * a stream capture. */
akmc_status akmc_batch_set_home_chunk(akmc_batch* b, int home_chunk);
int akmc_batch_home_chunk(const akmc_batch* b);
akmc_status akmc_batch_autotune(akmc_batch* b, double* pos_dev, double* force_dev,
                                double* energy_dev, int* status_dev, void* stream, int* chosen);

/* Per size class: systems with the same cell grid (uneven walker sets hold several) may
 * take different work-item sizes.  akmc_batch_set_system_chunks sets one per system
 * (chunks[nsys], each 8, 16 or 32).  akmc_batch_autotune_classes starts from
 * akmc_batch_autotune's uniform choice, then for each class in turn (ascending cell count)
 * times the three sizes for that class with the others fixed (3 calls each after a warm-up)
 * and keeps the fastest; it writes the number of classes and, for up to max_classes of them,
 * the cell count, the chosen size and the batch's time per call (ms) with it.  Both
 * synchronise the device. */
akmc_status akmc_batch_set_system_chunks(akmc_batch* b, const int* chunks);
akmc_status akmc_batch_autotune_classes(akmc_batch* b, double* pos_dev, double* force_dev, double* energy_dev,
                                        int* status_dev, void* stream, int* n_classes, int* class_cells,
                                        int* class_chunk, float* class_ms, int max_classes);
/* Work items the current plan has (the grid of a pair kernel launched without queues). */
int akmc_batch_total_items(const akmc_batch* b);

/* Number of kernel launches one akmc_batch_forces call makes. */
int akmc_batch_launches(const akmc_batch* b);

/* Device time per kernel: when enabled, every kernel this batch launches is bracketed by
 * CUDA events on its stream.  akmc_batch_kernel_times synchronises those events and
 * returns, per kernel, the accumulated milliseconds and launch count since the previous
 * call (then resets); names[k] points at a static kernel name.  Returns the number of
 * kernel kinds written (<= max). */
akmc_status akmc_batch_profile(akmc_batch* b, int enable);
int akmc_batch_kernel_times(akmc_batch* b, double* ms, int* launches, const char** names, int max);

/* ---- allocation-free call (no counterpart in the reference) ------------------------ */

/* Largest system the allocation-free call accepts. */
#define AKMC_NOALLOC_MAX_ATOMS 4096
#define AKMC_NOALLOC_MAX_CELLS 4096

/* EAM forces and energy of ONE system without allocating anything.
 *
 * This entry point has no counterpart in the reference; it exists for callers that
 * cannot call cudaMalloc at the moment they need forces.  Typical cases: code that is
 * enqueuing work while its stream is being captured into a CUDA graph (cudaMalloc and
 * cudaFree are not stream-ordered, and the runtime rejects them during a global-mode
 * capture); a serving or training process whose device memory is owned by a caching
 * allocator or a fixed budget, where an extra cudaMalloc can fail or fragment the pool;
 * and latency-critical loops that cannot afford cudaFree, which synchronises the whole
 * device.  akmc_batch_forces needs a batch whose scratch was allocated by
 * akmc_batch_create; this call instead keeps its scratch (cell list, sorted positions,
 * densities, per-atom energies, work items) in one fixed array of about 0.42 MB that is
 * part of the library image, so it calls no cudaMalloc, cudaFree or allocating library
 * routine.  The field itself must already be set up (akmc_field_setup allocates its
 * tables once, earlier).
 *
 * Inputs and outputs are the caller's device buffers, exactly as in akmc_batch_forces
 * for a batch of one: pos_dev double[n*3] (wrapped in place), label_dev int[n],
 * force_dev double[n*3], energy_dev double[5] (total, rcp, real, vdw, many),
 * status_dev int[1].  Every label must lie in [0, number of species of the field): the
 * labels are read on the device only, so an out-of-range label is reported there, as
 * AKMC_ERR_ARG in status_dev[0], and is read as species 0 (the energies and forces of
 * such a call are not meaningful).  box[3] (host) is the orthorhombic cell; n <= AKMC_NOALLOC_MAX_ATOMS
 * and at most AKMC_NOALLOC_MAX_CELLS cells (cells are one cutoff wide), otherwise the
 * call returns AKMC_ERR_CAPACITY without launching anything.
 *
 * Limits of the shared array:
 * - Every GPU that loads the library holds the array until the process exits.
 * - The first call on a device looks up the array's device address on that device
 *   (the calling thread's current device, which must be the field's); make that first
 *   call before any stream capture begins.  The address is kept for the life of the
 *   process: a cudaDeviceReset after the first call on a device is not supported.
 * - All calls on a device share the one array and it keeps the previous call's
 *   contents; the call re-initialises what must start fresh.  Two calls that overlap on
 *   the GPU (different streams, or different host threads) race on the array: issue
 *   them on one stream. */
akmc_status akmc_eam_forces_noalloc(akmc_field* f, int n, const double box[3], double* pos_dev,
                                    const int* label_dev, double* force_dev, double* energy_dev,
                                    int* status_dev, void* stream);

/* ---- batched walkers: FIRE relaxation and Dimer saddle search ---------------------
 *
 * A walker set holds W independent systems of one field (sizes may differ) and runs
 * every walker's optimiser on the GPU: the per-walker algebra in FP64 kernels, the
 * forces through batch calls that skip finished walkers, one iteration captured as a
 * CUDA graph.  Both calls are synchronous: they return when every walker has stopped.
 *
 * akmc_walkers_relax replaces Relax::RelaxStructure with method "fire"
 * (optim/Relax.cpp:19-39, 44-315): the same Euler FIRE update, controls and
 * convergence test, for all walkers at once.  The reference has no working Dimer
 * (optim/Dimer.cpp is a stub; its commented design is optim/Dimer.cpp:416-618, its
 * controls Common/DimerCntrl.h:18-88); akmc_walkers_dimer is the minimum-mode search
 * that design describes. */
typedef struct akmc_walkers akmc_walkers;

/* Walker outcome codes. */
enum {
    AKMC_WALKER_RUNNING = 0,
    AKMC_WALKER_CONVERGED = 1,   /* FIRE: minimum; Dimer: first-order saddle */
    AKMC_WALKER_MAX_ITER = 2,    /* the reference's setStatusFailed (Relax.cpp:297) */
    AKMC_WALKER_LOST = 3,        /* Dimer: energy rose more than max_rise above the start */
    AKMC_WALKER_FORCE_ERROR = 4, /* a force call of this walker returned a non-zero status */
    AKMC_WALKER_SKIPPED = 5      /* not run (mask 0 of akmc_walkers_relax_subset / _dimer_subset) */
};

/* RelaxCntrl (Common/RelaxCntrl.h:15-38); akmc_fire_defaults fills its defaults. */
typedef struct akmc_fire_params {
    int max_iter;                /* maxIter 3000 */
    int n_min;                   /* N_min 5 */
    double norm_tol;             /* normTol 1e-5: converged when |F| < norm_tol ... */
    double force_tol;            /* forceTol 1e-4: ... or max_i |F_i| < force_tol */
    double dt0;                  /* initTimeStep 0.0005 */
    double dt_max;               /* maxTimeStep 0.00075 */
    double alpha0;               /* alphaStart 0.1 */
    double alpha_dec;            /* alphaDecrease 0.99 */
    double step_inc;             /* stepIncrease 1.1 */
    double step_dec;             /* stepDecrease 0.5 */
    double max_move;             /* per-atom step cap in Angstrom; 0 = none (the reference) */
} akmc_fire_params;

/* DimerCntrl (Common/DimerCntrl.h:18-88) names where one exists; akmc_dimer_defaults
 * fills the defaults. */
typedef struct akmc_dimer_params {
    int max_iter;                /* translation steps, 300 */
    int max_rotations;           /* rotations per translation step (>= 1), 1 */
    int n_min;                   /* FIRE N_min 5 */
    int patience;                /* > 0: a walker whose max|F| has not fallen 2 % below its best for this many
                                    steps stops as AKMC_WALKER_MAX_ITER (stalled); 0: off (the default) */
    double delta;                /* dimerDisplacement 0.01 A */
    double rot_tol;              /* normTol 0.1 eV/A^2: no rotation below this |dC/dtheta|/2 */
    double force_tol;            /* forceTol 1e-2 eV/A: saddle when max_i |F_i| < force_tol ... */
    double max_eigenvalue;       /* ... and curvature < maxEigenvalue (0) */
    double min_trial;            /* smallest trial rotation angle, 1e-3 rad */
    double max_move;             /* FIRE per-atom translation cap per step, 0.02 A */
    double max_rise;             /* lost when E rises this far above the start, 8 eV */
    double dt0, dt_max;          /* FIRE time steps of the translation, 0.001 / 0.004 */
    double alpha0, alpha_dec, step_inc, step_dec;   /* DimerCntrl FIRE constants */
    int translation;             /* 1 L-BFGS on the modified force (default), 0 FIRE */
    int lbfgs_memory;            /* stored (s, y) pairs, 1..8 (8) */
    double max_step;             /* L-BFGS per-atom cap of a translation step, 0.2 A */
    double convex_step;          /* L-BFGS step along the unit mode while C >= 0, 0.05 A */
} akmc_dimer_params;

typedef struct akmc_walker_result {
    int status;                  /* AKMC_WALKER_* */
    int iters;                   /* optimiser steps taken */
    int force_calls;             /* system force evaluations spent on this walker */
    int reserved;
    double energy;               /* total energy at the final positions, eV */
    double curvature;            /* Dimer: curvature along the final mode, eV/A^2 */
    double fmax;                 /* max_i |F_i| at the final positions, eV/A */
    double fnorm;                /* FIRE: |F| at the final positions, eV/A */
} akmc_walker_result;

void akmc_fire_defaults(akmc_fire_params* p);
void akmc_dimer_defaults(akmc_dimer_params* p);

/* Walker w holds natoms[w] atoms in box[3w..3w+2]; label/charge (charge may be null:
 * species charges) and frozen (may be null; 1 = frozen, as Basis::frozen) are indexed
 * by atom, walkers back to back. */
akmc_status akmc_walkers_create(akmc_field* f, int nwalk, const int* natoms, const double* box,
                                const int* label, const double* charge, const int* frozen,
                                akmc_walkers** out);
akmc_status akmc_walkers_destroy(akmc_walkers* w);
int akmc_walkers_count(const akmc_walkers* w);
/* Neighbour-list skin of the walkers' force calls (akmc_batch_create_skin), in A: 0.4 by
 * default for EAM fields whose boxes allow it, 0 otherwise.  Setting it rebuilds the
 * walkers' batches. */
akmc_status akmc_walkers_set_skin(akmc_walkers* w, double skin);
double akmc_walkers_skin(const akmc_walkers* w);

/* FIRE-relax every walker.  pos: device [3 * total atoms] FP64, relaxed in place
 * (wrapped into the minimum-image cell, as every force call does).  out: host [W]. */
akmc_status akmc_walkers_relax(akmc_walkers* w, double* pos, const akmc_fire_params* p,
                               akmc_walker_result* out, void* stream);

/* akmc_walkers_relax for the walkers whose run_mask entry (device int [W]) is non-zero; the
 * others are not run: their pos keeps its values, out[k].status = AKMC_WALKER_SKIPPED.
 * run_mask = NULL relaxes every walker. */
akmc_status akmc_walkers_relax_subset(akmc_walkers* w, double* pos, const akmc_fire_params* p,
                                      const int* run_mask, akmc_walker_result* out, void* stream);

/* Dimer search of every walker from pos along mode (device, [3 * total atoms] each,
 * mode need not be normalised).  On return pos holds the final points (saddles for
 * converged walkers) and mode the final unit modes.  out: host [W]. */
akmc_status akmc_walkers_dimer(akmc_walkers* w, double* pos, double* mode,
                               const akmc_dimer_params* p, akmc_walker_result* out,
                               void* stream);

/* akmc_walkers_dimer for the walkers whose run_mask entry (device int [W]) is non-zero; the
 * others are not run: pos and mode keep their values, out[k].status =
 * AKMC_WALKER_SKIPPED.  run_mask = NULL runs every walker. */
akmc_status akmc_walkers_dimer_subset(akmc_walkers* w, double* pos, double* mode,
                                      const akmc_dimer_params* p, const int* run_mask,
                                      akmc_walker_result* out, void* stream);

/* ---- KMC step: FP64 event table, duplicate saddles, rate selection --------------------
 *
 * The reference's master rank keeps its event list in float (kmc/KineticMonteCarlo.cpp:
 * 1376-1460, kmc/Event.cpp:66-105) and selects with KineticMonteCarlo.cpp:147-199 and
 * 1151-1160.  These calls do the same step on device buffers in FP64: E_a = E_saddle -
 * E_min, rate = prefactor * exp(-E_a / (k_B T)), running sums in list order, the first
 * event whose running sum exceeds u1 * R, and dt = -ln(u2) / R (0 when R <= 1e-18).  All
 * pointers ending in _dev are device buffers; the calls are asynchronous on `stream`. */
typedef struct akmc_kmc_step {
    int chosen;                  /* index of the selected event, -1 when no rate is positive */
    int n_usable;                /* events that entered the sum */
    double total_rate;           /* R, 1/s */
    double dt;                   /* time advance, s */
    double barrier;              /* E_a of the chosen event, eV */
    double rate;                 /* its rate, 1/s */
    double u1, u2;               /* the uniforms used */
} akmc_kmc_step;

/* n uniform doubles in [0, 1) from Philox4x64-10 with key (seed, key_hi) and 128-bit
 * counter (counter, 0): the sequence numpy.random.Philox(key=[seed, key_hi],
 * counter=[counter, 0, 0, 0]) gives, 53 bits per double. */
akmc_status akmc_kmc_uniforms(uint64_t seed, uint64_t key_hi, uint64_t counter, int n,
                              double* out_dev, void* stream);

/* dup_dev[i] = the first j < i with usable_dev[j], the same group, saddle energies within
 * e_tol and every atom within d_tol (minimum image in box_dev[3i..3i+2]); -1 if none or if
 * event i is not usable.  Event i's saddle has natoms_dev[i] atoms at rows
 * [begin_dev[i], begin_dev[i] + natoms_dev[i]) of pos_dev. */
akmc_status akmc_events_dedup(int n, const int* group_dev, const int* usable_dev,
                              const double* energy_dev, const double* pos_dev,
                              const long long* begin_dev, const int* natoms_dev,
                              const double* box_dev, double e_tol, double d_tol, int* dup_dev,
                              void* stream);

/* Rates of the usable events (rate_dev), their running sums (cum_dev), and the selection
 * with u_dev[0], u_dev[1] written to *step_dev. */
akmc_status akmc_kmc_select(int n, const double* e_saddle_dev, const double* e_min_dev,
                            const int* usable_dev, double prefactor, double temperature,
                            const double* u_dev, double* rate_dev, double* cum_dev,
                            akmc_kmc_step* step_dev, void* stream);

/* ---- learned proposal directions: descriptors and a small MLP ---------------------
 *
 * No counterpart in the reference (its searches start from random displacements,
 * SaddleSearch.cpp:356-421).  Descriptors: 64 per atom (32 Gaussian radial functions on
 * 0.5-5 A and 32 Behler G4 angular functions), FP32, from the neighbours within 5 A.  MLP:
 * 64 -> 128 -> 128 -> 128 -> 3 with SiLU, standardised inputs, BF16 inputs / weights /
 * hidden activations, FP32 accumulation and biases; parameters are one FP32 vector
 * (W1 b1 W2 b2 W3 b3 W4 b4, W stored [in][out]) of akmc_mlp_num_params() floats; norm is
 * {mean[64], 1/std[64]}. */
int akmc_mlp_num_params(void);

/* Descriptors of every atom of an EAM batch at the positions of its last force call (its
 * neighbour list must reach 5 A), written to desc_dev[n_total][64] in the caller's atom
 * order.  When basis_dev is not null it receives the three per-atom vectors of the
 * equivariant readout, basis_dev[n_total][3][3] (vector m, component c):
 * B_m = sum_j phi_m(r_ij) (r_j - r_i) / r_ij, phi_m(r) = exp(-8 (r - nu_m)^2) fc(r),
 * nu = 2.5, 3.6, 4.4 A. */
akmc_status akmc_batch_descriptors(akmc_batch* b, float* desc_dev, float* basis_dev, void* stream);

/* The same for the n_rows atoms rows_dev[] (caller atom numbers, device int32) only:
 * desc_dev[n_rows][64] and basis_dev[n_rows][3][3] in the order of rows_dev.  A row outside
 * [0, n_total) gets zeros. */
akmc_status akmc_batch_descriptors_rows(akmc_batch* b, const int* rows_dev, int n_rows, float* desc_dev,
                                        float* basis_dev, void* stream);

/* y = MLP(desc_dev[n][64]) (3 numbers per row); out_dev[n][3] = y, or, when basis_dev
 * ([n][3][3]) is not null, the displacement sum_m y_m B_m.  Layers 1-3 on the tensor cores
 * (tcgen05, 128-row tiles, FP32 accumulation in tensor memory). */
akmc_status akmc_mlp_forward(int n, const float* desc_dev, const float* norm_dev,
                             const float* params_dev, const float* basis_dev, float* out_dev,
                             void* stream);

/* The same network on the FP32 pipe (BF16 operands, FP32 fma in a fixed order): the
 * cross-check of akmc_mlp_forward. */
akmc_status akmc_mlp_forward_fp32pipe(int n, const float* desc_dev, const float* norm_dev,
                                      const float* params_dev, const float* basis_dev, float* out_dev,
                                      void* stream);

/* AKMC_OK unless a tensor-core wait of an earlier akmc_mlp_forward gave up (its bounded
 * wait on the accumulator ran out; the outputs of that call are not valid).  Synchronous. */
akmc_status akmc_mlp_check(void);

/* One full-batch training step on n rows: mean over rows of the squared error summed over
 * the three components of the prediction (y, or sum_m y_m B_m with basis_dev), its gradient
 * reduced over 128-row tiles in fixed order (written to grad_dev when not null), then one Adam
 * step (beta 0.9 / 0.999, eps 1e-8, bias-corrected for `step` >= 1) on params_dev with learning
 * rate lr (lr = 0: gradient only).  On the tensor cores (tcgen05): the forward as in
 * akmc_mlp_forward; in the backward the hidden-layer errors dZ are rounded to BF16 (the tensor
 * core's operand; the bias gradients sum these values) and dW = H^T dZ, dH = dZ W^T run as
 * MMAs with FP32 accumulation.  loss_dev[ceil(n/128)] receives per-tile sums of squared
 * errors (their sum / n is the loss); scratch_dev holds ceil(n/128) *
 * akmc_mlp_num_params() floats. */
akmc_status akmc_mlp_train_step(int n, const float* desc_dev, const float* target_dev,
                                const float* norm_dev, const float* basis_dev,
                                float* params_dev, float* adam_m_dev, float* adam_v_dev,
                                float* scratch_dev, int step, float lr, float* loss_dev,
                                float* grad_dev, void* stream);

/* The same step on the FP32 pipe (32-row tiles, dZ in FP32): the cross-check of
 * akmc_mlp_train_step.  loss_dev[ceil(n/32)], scratch_dev ceil(n/32) * akmc_mlp_num_params()
 * floats. */
akmc_status akmc_mlp_train_step_fp32pipe(int n, const float* desc_dev, const float* target_dev,
                                         const float* norm_dev, const float* basis_dev,
                                         float* params_dev, float* adam_m_dev, float* adam_v_dev,
                                         float* scratch_dev, int step, float lr, float* loss_dev,
                                         float* grad_dev, void* stream);

/* akmc_batch_descriptors of a walker set's systems at pos (device, n_total x 3): one force
 * call on the set's own batch builds the neighbour lists, then the descriptors (and, when
 * basis is not null, the readout vectors) of every atom, on the caller's stream order. */
akmc_status akmc_walkers_descriptors(akmc_walkers* w, const double* pos, float* desc, float* basis,
                                     void* stream);

/* akmc_walkers_descriptors for the n_rows atoms rows[] of the set only (as
 * akmc_batch_descriptors_rows): the starting-atom candidates of a proposal. */
akmc_status akmc_walkers_descriptors_rows(akmc_walkers* w, const double* pos, const int* rows, int n_rows,
                                          float* desc, float* basis, void* stream);

/* Starting displacements of n_walkers Dimer walkers from the model's predictions.  Walker w
 * owns atoms begin_dev[w] .. begin_dev[w+1]-1 of pos_dev (n_atoms x 3), box_dev[w][3] is its
 * orthorhombic box, center_dev (optional, [W][3]) a centre per walker that, with
 * params->region > 0, restricts its candidates to atoms within region of it (minimum image;
 * the walker's local search region), pred_dev[atom][3] the predicted displacement, score_dev[atom *
 * score_stride] the predicted score.  The candidates of a walker are its atoms whose
 * predicted displacement is at least min_disp long and whose score is >= threshold * (the
 * largest such score); from the uniforms u_q of the Philox4x64-10 stream of key
 * (seed, w) and counter (counter, 0) -- numpy.random.Philox(key=[seed, w], counter=[counter,
 * 0, 0, 0]).random() -- the chosen atom c is candidate floor(u_0 * count) in atom order.
 * disp_dev = scale * pred[c] on c plus noise * z on every atom within radius of c (minimum
 * image), z_k = sqrt(-2 ln(1 - u_a)) cos(2 pi u_b), (a, b) = (1 + 6j + 2k, 2 + 6j + 2k) for
 * atom j (index within the walker) and component k; mode_dev (optional) = pred[c] on c and
 * zero elsewhere; chosen_dev[w] = c (index within the walker), or -1 with zero displacement
 * and mode when the walker has no candidate or its largest score is below min_score (the caller then seeds it at
 * random, SaddleSearch.cpp:356-421). */
typedef struct akmc_proposal_params {
    double threshold;   /* candidate score relative to the walker's largest, in [0, 1] */
    double min_score;   /* below this largest score the walker gets no proposal */
    double scale;       /* displacement of the chosen atom, in units of its prediction */
    double noise;       /* standard deviation (A) of the noise on the chosen atom's neighbourhood */
    double radius;      /* neighbourhood radius (A) */
    double min_disp;    /* an atom is a candidate only if its predicted displacement is this long (A) */
    double region;      /* with center_dev: candidates only within this distance of the walker's centre (A) */
    int group;          /* walkers per group of consecutive walkers searching one system: the g-th walker of a
                           group takes the candidate at fraction (g + u) / group of the candidate list (u one
                           uniform per walker), so a group's walkers start from different candidates whenever
                           there are at least as many; 0 or 1: an independent draw per walker */
} akmc_proposal_params;

akmc_status akmc_proposal_seeds(int n_walkers, const long long* begin_dev, const double* pos_dev,
                                const double* box_dev, const double* center_dev, const float* pred_dev,
                                const float* score_dev, int score_stride, const akmc_proposal_params* params,
                                uint64_t seed, uint64_t counter, double* disp_dev, double* mode_dev,
                                int* chosen_dev, void* stream);

/* The per-size-class work-item sizes the walker set's batches were tuned to on their first
 * call (akmc_batch_autotune_classes): which = 0 the FIRE batch (W systems), 1 the Dimer's
 * image batch (3W systems).  Writes up to max rows (cells per system of the class, chosen
 * size, the batch's ms per force call with it) and returns the number of classes (0 before
 * tuning). */
int akmc_walkers_tuning(const akmc_walkers* w, int which, int* cells, int* chunk, float* ms, int max);

/* Keep the batches' default work-item sizes: no tuning on the first call (for walker sets
 * made for one search, where a dozen timed trial force calls would cost more than they save). */
akmc_status akmc_walkers_skip_tuning(akmc_walkers* w);

/* ---- self-checking build -----------------------------------------------------------
 *
 * The library built with `python -m akmc_b200.build --checks` (libakmc_b200_checks.so)
 * bounds-checks the indices of its kernels (cell-sort scatter and permutations, staged
 * candidates, neighbour-list rows, counts and entries, output permutations, walker atom
 * ranges, listed near pairs): a failed check counts a hit under its code, keeps the first
 * offending value and skips the access, and the kernel carries on; nothing traps.  The
 * checks stand in for a memory checker.  The default library compiles them away. */

/* 1 in the self-checking build, 0 otherwise. */
int akmc_checks_enabled(void);

/* Hit counts and first offending values of every check, AKMC_CHECK_FILES x 32 entries each
 * (file 0 cell kernels, 1 pair kernels, 2 walker kernels; entry = check code); clear != 0
 * resets them.  Synchronous.  AKMC_ERR_UNSUPPORTED in the default build. */
#define AKMC_CHECK_FILES 3
akmc_status akmc_checks_read(int* hits, int* first, int clear);

/* ---- configuration and introspection ---------------------------------------------- */

/* EAM neighbour lists are sized, per batch, for 1.5 x the mean neighbour count at the batch's
 * densest mean density (atoms / cell volume) plus 16.  Atoms clustered in part of their cell
 * (a local region cut out of a crystal and placed in an isolated cell) are denser than that
 * mean: rho (atoms per cubic Angstrom) sets a floor for the density of batches created
 * afterwards, including the one akmc_forces uses.  0 (the default) removes it.  A list that
 * would overflow reports AKMC_ERR_CAPACITY. */
akmc_status akmc_field_set_list_density(akmc_field* f, double rho);

akmc_status akmc_field_set_precision(akmc_field* f, int mode);
int akmc_field_family(const akmc_field* f);
int akmc_field_num_species(const akmc_field* f);
/* name must hold 16 bytes. */
akmc_status akmc_field_species(const akmc_field* f, int i, char* name, double* mass,
                               double* charge);
double akmc_field_cutoff(const akmc_field* f);
/* Ewald parameters after setup: eta, number of k-vectors, gcell[3]. */
akmc_status akmc_field_ewald(const akmc_field* f, double* eta, int* nk, int gcell[3]);
/* Thread-local message of the last failing call on this thread. */
const char* akmc_last_error(void);
const char* akmc_version(void);

#ifdef __cplusplus
}
#endif
#endif
