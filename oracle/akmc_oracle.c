/* FP64 CPU restatement of the AKMC force/energy path -- the ORACLE (test infrastructure).
 *
 * Only tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py use this
 * file, always as the checker. The product (akmc_b200/csrc) never links it.
 *
 * Each routine restates the reference's arithmetic in the same order, with the
 * reference location cited. Brute-force O(N^2) minimum image, exactly as the
 * reference's image-convention path (no neighbour list: potentials/metal/Field.cpp:
 * 296-490, potentials/pair/Field.cpp:660-842).
 */
#include "akmc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static const double ORC_PI = 3.14159265358979323846;
static const double ORC_TWOPI = 6.28318530717958647692;
static const double ORC_CTOEV = 14.3996454784;          /* shared constants header */
static const double ORC_TWO_OVER_ROOTPI = 1.128379167095512; /* pair/Field.cpp:2223 */

/* ------------------------------------------------------------------------------------
 * geometry
 * ------------------------------------------------------------------------------------ */

/* Field::resetSimulationCellMinImage (metal/Field.cpp:1894-1920; pair copy 2164-2190). */
static void wrap_min_image(int n, double* x, double* y, double* z, const double* lat,
                           const double* rcp)
{
    for (int i = 0; i < n; i++) {
        double rx = x[i], ry = y[i], rz = z[i];
        double xx = rx * rcp[0] + ry * rcp[3] + rz * rcp[6];
        double yy = rx * rcp[1] + ry * rcp[4] + rz * rcp[7];
        double zz = rx * rcp[2] + ry * rcp[5] + rz * rcp[8];
        xx -= rint(xx);
        yy -= rint(yy);
        zz -= rint(zz);
        x[i] = xx * lat[0] + yy * lat[3] + zz * lat[6];
        y[i] = xx * lat[1] + yy * lat[4] + zz * lat[7];
        z[i] = xx * lat[2] + yy * lat[5] + zz * lat[8];
    }
}

/* The pair separation of the force loops (metal/Field.cpp:397-414). */
static double min_image_sep(double ax, double ay, double az, double bx, double by, double bz,
                            const double* lat, const double* rcp, double* rx, double* ry,
                            double* rz)
{
    double dx = ax - bx, dy = ay - by, dz = az - bz;
    double xx = dx * rcp[0] + dy * rcp[3] + dz * rcp[6];
    double yy = dx * rcp[1] + dy * rcp[4] + dz * rcp[7];
    double zz = dx * rcp[2] + dy * rcp[5] + dz * rcp[8];
    xx -= rint(xx);
    yy -= rint(yy);
    zz -= rint(zz);
    *rx = xx * lat[0] + yy * lat[3] + zz * lat[6];
    *ry = xx * lat[1] + yy * lat[4] + zz * lat[7];
    *rz = xx * lat[2] + yy * lat[5] + zz * lat[8];
    return (*rx) * (*rx) + (*ry) * (*ry) + (*rz) * (*rz);
}

/* dcell (Common/Utility.cpp:23-84): lengths [0..2], cosines [3..5], perpendicular
 * widths [6..8], volume [9] of the cell whose vectors are the rows of a[9]. */
static void dcell(const double* a, double* b)
{
    b[0] = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    b[1] = sqrt(a[3] * a[3] + a[4] * a[4] + a[5] * a[5]);
    b[2] = sqrt(a[6] * a[6] + a[7] * a[7] + a[8] * a[8]);
    b[3] = (a[0] * a[3] + a[1] * a[4] + a[2] * a[5]) / (b[0] * b[1]);
    b[4] = (a[0] * a[6] + a[1] * a[7] + a[2] * a[8]) / (b[0] * b[2]);
    b[5] = (a[3] * a[6] + a[4] * a[7] + a[5] * a[8]) / (b[1] * b[2]);
    double axb1 = a[1] * a[5] - a[2] * a[4], axb2 = a[2] * a[3] - a[0] * a[5],
           axb3 = a[0] * a[4] - a[1] * a[3];
    double bxc1 = a[4] * a[8] - a[5] * a[7], bxc2 = a[5] * a[6] - a[3] * a[8],
           bxc3 = a[3] * a[7] - a[4] * a[6];
    double cxa1 = a[7] * a[2] - a[1] * a[8], cxa2 = a[0] * a[8] - a[2] * a[6],
           cxa3 = a[1] * a[6] - a[0] * a[7];
    b[9] = fabs(a[0] * bxc1 + a[1] * bxc2 + a[2] * bxc3);
    b[6] = b[9] / sqrt(bxc1 * bxc1 + bxc2 * bxc2 + bxc3 * bxc3);
    b[7] = b[9] / sqrt(cxa1 * cxa1 + cxa2 * cxa2 + cxa3 * cxa3);
    b[8] = b[9] / sqrt(axb1 * axb1 + axb2 * axb2 + axb3 * axb3);
}

/* ------------------------------------------------------------------------------------
 * EAM
 * ------------------------------------------------------------------------------------ */

/* ManyBody::eamMeshEnergy (metal/ManyBody.cpp:455-460); dist[i] = i*step
 * (MetalPotential.cpp:331,343,354). */
static double mesh_interp(const double* p, double r, double dr, int idx)
{
    double d = idx * dr;
    return p[idx] + ((p[idx + 1] - p[idx]) * (r - d) / dr);
}

/* ManyBody::calculateManyBodyDensEnergy, EAM branch (ManyBody.cpp:462-553):
 * density pot of type b (b*ns+b). */
static double dens_energy(const orc_eam_pot* p, double r)
{
    if (r < 1.0e-8) return 0.0;
    if (!(r < p->pot_cutoff)) return 0.0;
    double dr = p->step_r;
    int idx = (int)(r / dr);
    return mesh_interp(p->rho, r, dr, idx);
}

/* ManyBody::embed, EAM branch (ManyBody.cpp:554-619). Range error instead of exit. */
static int embed(const orc_eam_pot* p, double rho, double* out)
{
    double dr = p->step_embed;
    int idx = (int)(rho / dr);
    if (idx < 0 || idx >= p->n_embed) return ORC_ERR_EMBED_RANGE;
    *out = mesh_interp(p->F, rho, dr, idx);
    return ORC_OK;
}

int orc_eam_forces(int n_pot, const orc_eam_pot* pots, int ns, const int* mesh_table,
                   double short_range_cut, int n, double* x, double* y, double* z,
                   const int* label, const double lat[9], const double rcp[9],
                   double* fx, double* fy, double* fz, double* rho_out, double energies[5])
{
    if (n < 0 || (n > 0 && (!x || !y || !z || !label || !fx || !fy || !fz))) return ORC_ERR_ARG;
    (void)n_pot;
    int status = ORC_OK;
    double radius = short_range_cut * short_range_cut;   /* metal/Field.cpp:325 */
    double* rho = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));

    /* Field::calculateForces zeroes forces then wraps (metal/Field.cpp:219-232). */
    for (int i = 0; i < n; i++) fx[i] = fy[i] = fz[i] = 0.0;
    wrap_min_image(n, x, y, z, lat, rcp);

    /* pass 1: calculateAtomRho (metal/Field.cpp:1782-1853) */
    for (int a = 0; a < n; a++) {
        double s = 0.0;
        for (int b = 0; b < n; b++) {
            if (a == b) continue;
            double rx, ry, rz;
            double rsq = min_image_sep(x[a], y[a], z[a], x[b], y[b], z[b], lat, rcp, &rx, &ry, &rz);
            if (rsq <= radius) {
                int pot = mesh_table[label[b] * ns + label[b]];
                if (pot >= 0) s += dens_energy(&pots[pot], sqrt(rsq));
            }
        }
        rho[a] = s;
    }

    /* embedding energy (metal/Field.cpp:358-367) */
    double many = 0.0;
    for (int a = 0; a < n; a++) {
        int pot = mesh_table[label[a] * ns + label[a]];
        if (pot < 0) continue;
        double e;
        int st = embed(&pots[pot], rho[a], &e);
        if (st) { status |= st; continue; }
        many += e;
    }

    /* pass 2: ordered-pair force loop (metal/Field.cpp:371-449) with
     * calculateManyBodyPairForce (ManyBody.cpp:621-710) and
     * calculateManyBodyForce (ManyBody.cpp:711-831), EAM branches. */
    double two = 0.0;
    for (int a = 0; a < n; a++) {
        for (int b = 0; b < n; b++) {
            if (a == b) continue;
            double rx, ry, rz;
            double rsq = min_image_sep(x[a], y[a], z[a], x[b], y[b], z[b], lat, rcp, &rx, &ry, &rz);
            if (!(rsq <= radius)) continue;
            double r = sqrt(rsq);
            int pot = mesh_table[label[a] * ns + label[b]];
            double eng_s = 0.0, forc_s = 0.0, forc_m = 0.0;
            if (pot >= 0 && r >= 1.0e-8) {
                const orc_eam_pot* p = &pots[pot];
                if (r < p->pot_cutoff) {
                    double dr = p->step_r;
                    int idx = (int)(r / dr);
                    eng_s = mesh_interp(p->phi, r, dr, idx);
                    forc_s = -r * mesh_interp(p->dphi, r, dr, idx);
                }
                const double tiny = 1.0e-8;
                if (!(rho[a] < tiny || rho[b] < tiny) && r < p->pot_cutoff) {
                    double de = p->step_embed;
                    int ia = (int)(rho[a] / de), ib = (int)(rho[b] / de);
                    if (ia < 0 || ia >= p->n_embed || ib < 0 || ib >= p->n_embed) {
                        status |= ORC_ERR_EMBED_RANGE;
                    } else {
                        double d1 = mesh_interp(p->dF, rho[a], de, ia);
                        double d2 = mesh_interp(p->dF, rho[b], de, ib);
                        double dd = p->step_r;
                        int ir = (int)(r / dd);
                        double t1 = mesh_interp(p->drho, r, dd, ir);
                        forc_m = ((d1 + d2) * t1) * r;
                    }
                }
            }
            double ftot = (forc_s - forc_m) / (rsq * 2.0);
            two += 0.5 * eng_s;
            fx[a] += rx * ftot; fy[a] += ry * ftot; fz[a] += rz * ftot;
            fx[b] -= rx * ftot; fy[b] -= ry * ftot; fz[b] -= rz * ftot;
        }
    }

    if (rho_out) memcpy(rho_out, rho, (size_t)n * sizeof(double));
    free(rho);
    /* metal/Field.cpp:260-264 */
    energies[ORC_E_RCP] = 0.0;
    energies[ORC_E_REAL] = 0.0;
    energies[ORC_E_MANY] = many;
    energies[ORC_E_VDW] = two;
    energies[ORC_E_TOTAL] = many + two;
    return status;
}

/* ------------------------------------------------------------------------------------
 * Ewald
 * ------------------------------------------------------------------------------------ */

double orc_ewald_eta(double precis, double cutoff)
{
    double eps = fmin(fabs(precis), 0.5);
    double tol = sqrt(fabs(log(eps * cutoff)));
    return sqrt(fabs(log(eps * cutoff * tol))) / cutoff;
}

/* Ewald::setEwaldImage (Ewald.cpp:88-120) + findGvector (Ewald.cpp:188-319). */
int orc_ewald_kvectors(double eta, double cutoff, double precis, const double lat[9],
                       const double rcp[9], int max_k, double* kx, double* ky, double* kz,
                       double* g0, int gcell_out[3])
{
    double eps = fmin(fabs(precis), 0.5);
    double tol = sqrt(fabs(log(eps * cutoff)));
    double cel[10];
    dcell(lat, cel);
    double volume = cel[9];
    double tol1 = sqrt(-log(eps * cutoff * pow(2.0 * tol * eta, 2)));
    int gx = (int)rint(0.25 + cel[0] * eta * tol1 / ORC_PI);
    int gy = (int)rint(0.25 + cel[1] * eta * tol1 / ORC_PI);
    int gz = (int)rint(0.25 + cel[2] * eta * tol1 / ORC_PI);
    dcell(rcp, cel);
    double cx = (double)gx * cel[6], cy = (double)gy * cel[7], cz = (double)gz * cel[8];
    double rcut = fmin(fmin(cx, cy), cz);
    double rcutsq = rcut * rcut;
    if (gcell_out) { gcell_out[0] = gx; gcell_out[1] = gy; gcell_out[2] = gz; }

    double etasq = eta * eta, gsqfct = 1.0 / (4.0 * etasq);
    double gfct0 = ORC_CTOEV * ORC_PI / (etasq * volume);
    int nk = 0;
    for (int nx = 0; nx <= gx; nx++)
        for (int ny = -gy; ny <= gy; ny++)
            for (int nz = -gz; nz <= gz; nz++) {
                double X = nx * rcp[0] + ny * rcp[1] + nz * rcp[2];
                double Y = nx * rcp[3] + ny * rcp[4] + nz * rcp[5];
                double Z = nx * rcp[6] + ny * rcp[7] + nz * rcp[8];
                double gsq = X * X + Y * Y + Z * Z;
                if (gsq < rcutsq && gsq > 1.0e-8) {
                    if (nk >= max_k) return -1;
                    kx[nk] = X; ky[nk] = Y; kz[nk] = Z;
                    nk++;
                }
            }
    for (int i = 0; i < nk; i++) {
        kx[i] *= ORC_TWOPI; ky[i] *= ORC_TWOPI; kz[i] *= ORC_TWOPI;
        double gsq = kx[i] * kx[i] + ky[i] * ky[i] + kz[i] * kz[i];
        double xg = gsq * gsqfct;
        double gzz = exp(-xg) / xg;
        g0[i] = (kx[i] < 1.0e-8) ? gzz * gfct0 : gzz * gfct0 * 2.0;
    }
    return nk;
}

/* Ewald::recipSpaceForce, compiled variant (Ewald.cpp:560-662), forces and energy. */
static double recip_force(int nk, const double* kx, const double* ky, const double* kz,
                          const double* g0, int n, const double* x, const double* y,
                          const double* z, const double* q, double* fx, double* fy, double* fz)
{
    double* cp = (double*)malloc((size_t)(n > 0 ? n : 1) * sizeof(double));
    double* sp = (double*)malloc((size_t)(n > 0 ? n : 1) * sizeof(double));
    double e = 0.0;
    for (int k = 0; k < nk; k++) {
        double C = 0.0, S = 0.0, vx = kx[k], vy = ky[k], vz = kz[k], v0 = g0[k];
        for (int i = 0; i < n; i++) {
            double ph = vx * x[i] + vy * y[i] + vz * z[i];
            cp[i] = q[i] * cos(ph);
            sp[i] = q[i] * sin(ph);
            C += cp[i];
            S += sp[i];
        }
        for (int i = 0; i < n; i++) {
            e += v0 * (cp[i] * C + sp[i] * S);
            double pf = -v0 * (-sp[i] * C + cp[i] * S);
            fx[i] += pf * vx; fy[i] += pf * vy; fz[i] += pf * vz;
        }
    }
    free(cp); free(sp);
    return 0.5 * e;
}

int orc_ionic_forces(int ns, const double* buck, double cutoff, double eta,
                     double cfact, int nk, const double* kx, const double* ky,
                     const double* kz, const double* g0, int n, double* x, double* y,
                     double* z, const double* q, const int* label, const double lat[9],
                     const double rcp[9], double* fx, double* fy, double* fz,
                     double energies[5])
{
    if (n < 0 || (n > 0 && (!x || !y || !z || !q || !label || !fx || !fy || !fz))) return ORC_ERR_ARG;
    for (int i = 0; i < n; i++) fx[i] = fy[i] = fz[i] = 0.0;

    /* pair/Field.cpp:342-348: reciprocal space on the positions as given, then wrap */
    double erc = recip_force(nk, kx, ky, kz, g0, n, x, y, z, q, fx, fy, fz);
    wrap_min_image(n, x, y, z, lat, rcp);

    /* pair/Field.cpp:704-720: self term, hfunc2(0) = 2/sqrt(pi) */
    double ereal = 0.0, evdw = 0.0;
    for (int a = 0; a < n; a++) {
        double h0 = ORC_TWO_OVER_ROOTPI;
        ereal += -h0 * (0.5 * cfact * q[a] * q[a]) * eta;
    }

    double radius = cutoff * cutoff, eta3 = eta * eta * eta;
    /* half-pair loop (pair/Field.cpp:722-828) */
    for (int a = 0; a < n; a++) {
        double qa = cfact * q[a];
        double fxi = 0.0, fyi = 0.0, fzi = 0.0;
        for (int b = a + 1; b < n; b++) {
            double rx, ry, rz;
            double rsq = min_image_sep(x[a], y[a], z[a], x[b], y[b], z[b], lat, rcp, &rx, &ry, &rz);
            double eng = 0.0, eng_s = 0.0, forc = 0.0, forc_s = 0.0;
            if (rsq <= radius) {
                double r = sqrt(rsq);
                double qq = qa * q[b];
                /* hfunc1 (pair/Field.cpp:2218-2236) */
                double xr = eta * r;
                if (xr != 0.0) {
                    double h0 = erfc(xr) / xr;
                    double xsq = xr * xr;
                    double h1 = (-h0 - ORC_TWO_OVER_ROOTPI * exp(-xsq)) / xsq;
                    eng = h0 * qq * eta;
                    forc = h1 * qq * eta3;
                }
                /* TwoBody::shortrangeone, Buckingham (TwoBody.h:173-215) */
                if (r >= 1.0e-8) {
                    const double* p = &buck[3 * (label[a] * ns + label[b])];
                    double e1 = p[0] * exp(-r / p[1]);
                    double f1 = e1 / (r * p[1]);
                    double e2 = -p[2] / (rsq * rsq * rsq);
                    double f2 = 6 * e2 / rsq;
                    eng_s = e1 + e2;
                    forc_s = f1 + f2;
                }
            }
            ereal += eng;
            evdw += eng_s;
            forc -= forc_s;
            fxi -= rx * forc; fyi -= ry * forc; fzi -= rz * forc;
            fx[b] += rx * forc; fy[b] += ry * forc; fz[b] += rz * forc;
        }
        fx[a] += fxi; fy[a] += fyi; fz[a] += fzi;
    }
    energies[ORC_E_RCP] = erc;
    energies[ORC_E_REAL] = ereal;
    energies[ORC_E_VDW] = evdw;
    energies[ORC_E_MANY] = 0.0;
    energies[ORC_E_TOTAL] = erc + ereal + evdw;
    return ORC_OK;
}

/* ------------------------------------------------------------------------------------
 * neighbour sets (NbrListPBC::calculateNbrList criterion, NbrListPBC.cpp:41-125)
 * ------------------------------------------------------------------------------------ */
long long orc_neighbour_counts(int n, const double* x, const double* y, const double* z,
                               const double lat[9], const double rcp[9], double rc,
                               int* counts)
{
    long long tot = 0;
    double rc2 = rc * rc;
    for (int a = 0; a < n; a++) {
        int c = 0;
        for (int b = 0; b < n; b++) {
            if (a == b) continue;
            double rx, ry, rz;
            if (min_image_sep(x[a], y[a], z[a], x[b], y[b], z[b], lat, rcp, &rx, &ry, &rz) <= rc2) c++;
        }
        counts[a] = c;
        tot += c;
    }
    return tot;
}

long long orc_neighbour_list(int n, const double* x, const double* y, const double* z,
                             const double lat[9], const double rcp[9], double rc,
                             long long max_pairs, long long* offsets, int* nbr)
{
    long long m = 0;
    double rc2 = rc * rc;
    offsets[0] = 0;
    for (int a = 0; a < n; a++) {
        for (int b = 0; b < n; b++) {
            if (a == b) continue;
            double rx, ry, rz;
            if (min_image_sep(x[a], y[a], z[a], x[b], y[b], z[b], lat, rcp, &rx, &ry, &rz) <= rc2) {
                if (m >= max_pairs) return -1;
                nbr[m++] = b;
            }
        }
        offsets[a + 1] = m;
    }
    return m;
}
