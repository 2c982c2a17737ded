/* FP64 CPU restatement of the AKMC force/energy path -- the ORACLE.
 *
 * Test infrastructure only: tests/, __graft_entry__.smoke() and the cpu_baseline leg
 * of bench.py call it as the checker. The product library never links it.
 *
 * The arithmetic follows the reference line by line (file:line cited at each function
 * in akmc_oracle.c); the data layout is this project's own (flat arrays, one struct per
 * table). Parity of this restatement with the reference's own Field, compiled from the
 * reference sources (oracle/Makefile -> oracle/_ref), is pinned in tests/.
 */
#ifndef AKMC_ORACLE_H
#define AKMC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* One tabulated EAM potential as MetalPotential::readLEAM builds it
 * (potentials/metal/MetalPotential.cpp:276-361): value tables p[i] on the grid
 * i*step and forward-difference derivative tables (:388-392) with deriv[n-1] = 0. */
typedef struct {
    int n_embed, n_r;
    double step_embed, step_r, pot_cutoff;
    const double *F, *dF;        /* parEmbed, derivEmbed   [n_embed] */
    const double *rho, *drho;    /* parDens,  derivDens    [n_r]     */
    const double *phi, *dphi;    /* parRep,   derivRep     [n_r]     */
} orc_eam_pot;

/* energies[] layout shared by both families: 0 total, 1 rcp, 2 real, 3 vdw, 4 many */
enum { ORC_E_TOTAL = 0, ORC_E_RCP, ORC_E_REAL, ORC_E_VDW, ORC_E_MANY, ORC_E_COUNT };

/* Status codes (mirror the product's akmc_status values for the same conditions). */
enum { ORC_OK = 0, ORC_ERR_ARG = 1, ORC_ERR_EMBED_RANGE = 2, ORC_ERR_CUTOFF = 4 };

/* EAM forces and energy, brute-force minimum image over all pairs.
 * Positions are wrapped in place (as the reference does). rho_out may be NULL. */
int orc_eam_forces(int n_pot, const orc_eam_pot* pots, int n_species, const int* mesh_table,
                   double short_range_cut, int n, double* x, double* y, double* z,
                   const int* label, const double lat[9], const double rcp[9],
                   double* fx, double* fy, double* fz, double* rho_out, double energies[5]);

/* Ewald k-vector set (potentials/pair/Ewald.cpp:88-319). Returns the number of
 * vectors written (<= max_k), or -1 if max_k is too small. kx,ky,kz are the 2*pi-scaled
 * vectors, g0 the energy prefactor including the half-space weight. */
int orc_ewald_kvectors(double eta, double cutoff, double precis, const double lat[9],
                       const double rcp[9], int max_k, double* kx, double* ky, double* kz,
                       double* g0, int gcell_out[3]);

/* eta from `ewald precis` (potentials/pair/Field.cpp:129-133). */
double orc_ewald_eta(double precis, double cutoff);

/* Ionic forces: Ewald reciprocal + self + real-space erfc + Buckingham.
 * buck[3*(a*ns+b) + {0,1,2}] = A, rho, C; buck_present[a*ns+b] = 1 when listed. */
int orc_ionic_forces(int n_species, const double* buck, double cutoff, double eta,
                     double coulomb_factor, int nk, const double* kx, const double* ky,
                     const double* kz, const double* g0, int n, double* x, double* y,
                     double* z, const double* q, const int* label, const double lat[9],
                     const double rcp[9], double* fx, double* fy, double* fz,
                     double energies[5]);

/* Full minimum-image neighbour count per atom, rsq <= rc^2, j != i
 * (potentials/metal/NbrListPBC.cpp:41-125 criterion). Returns total pairs. */
long long orc_neighbour_counts(int n, const double* x, const double* y, const double* z,
                               const double lat[9], const double rcp[9], double rc,
                               int* counts);

/* Neighbour list in CSR form: offsets[n+1], neighbours sorted ascending per atom. */
long long orc_neighbour_list(int n, const double* x, const double* y, const double* z,
                             const double lat[9], const double rcp[9], double rc,
                             long long max_pairs, long long* offsets, int* nbr);

#ifdef __cplusplus
}
#endif
#endif
