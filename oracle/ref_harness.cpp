// C entry points around the reference's own Field class, compiled from the reference
// sources in place (see oracle/Makefile). One build per potential family, because the
// reference defines a class named Field in both potentials/metal and potentials/pair.
//
// Test infrastructure only: used by tests/, the golden-vector generator and the
// CPU-baseline leg of bench.py. The product never links or calls it.
//
// The call sequence mirrors the reference driver (kmc/kmc.cpp:188-221):
//   Field::readPotential(potentials stream, log, Species&)   metal/Field.cpp:122-205,
//                                                            pair/Field.cpp:215-317
//   Field::setup(mpi, lat, rcp, minDim, volume, maxAtoms, Species, log)
//   Field::calculateForces(mpi, posX, posY, posZ, fX, fY, fZ, stress, lat, rcp,
//                          charge, atmLabel, frozen, N, Energy&)   metal/Field.h:192-193
#include <cmath>
#include <fstream>
#include <string>
#include <vector>
#include "Field.h"
#include "Relax.h"
#include "ref_handle.h"

#define REF_API extern "C" __attribute__((visibility("default")))

namespace {

// Reciprocal vectors with the same index layout as Basis::setRcpVec (Common/Basis.cpp:987-1010).
void reciprocal(const double* L, double* R)
{
    R[0] = L[4] * L[8] - L[7] * L[5];
    R[1] = L[6] * L[5] - L[3] * L[8];
    R[2] = L[3] * L[7] - L[6] * L[4];
    R[3] = L[7] * L[2] - L[1] * L[8];
    R[4] = L[0] * L[8] - L[6] * L[2];
    R[7] = L[6] * L[1] - L[0] * L[7];
    R[6] = L[1] * L[5] - L[4] * L[2];
    R[5] = L[2] * L[3] - L[5] * L[0];
    R[8] = L[0] * L[4] - L[3] * L[1];
    double det = L[0] * R[0] + L[1] * R[3] + L[2] * R[6];
    double f = std::fabs(det) > 0.0 ? 1.0 / det : 1.0;
    for (int i = 0; i < 9; i++) R[i] *= f;
}

double minimum_dimension(const double* L)
{
    // Basis::minDimension (Common/Basis.cpp:1064-1088)
    double cx = L[0] * L[0] + L[3] * L[3] + L[6] * L[6];
    double cy = L[1] * L[1] + L[4] * L[4] + L[7] * L[7];
    double cz = L[2] * L[2] + L[5] * L[5] + L[8] * L[8];
    double m = cx;
    if (cy < cx) m = cy;
    if (cz < cy) m = cz;
    return std::sqrt(m);
}

double volume(const double* L)
{
    double b1 = L[4] * L[8] - L[5] * L[7];
    double b2 = L[5] * L[6] - L[3] * L[8];
    double b3 = L[3] * L[7] - L[4] * L[6];
    return std::fabs(L[0] * b1 + L[1] * b2 + L[2] * b3);
}

}  // namespace

// min_dim_override > 0 replaces the minimum cell dimension handed to Field::setup.  The
// pair Field uses that value only for its guard cutoff + verletShell <= minDim/2
// (pair/Field.cpp:98-107); the shell belongs to a neighbour-list path the image-convention
// force loops do not use, so the override lets the unmodified force loops run a 10 A
// cutoff in a 21.05 A cell (cutoff < L/2, minimum image still exact).
REF_API void* ref_create(const char* potentials_path, const char* log_path,
                         const double* lat, int max_atoms, double min_dim_override)
{
    RefHandle* h = new RefHandle();
    h->log.open(log_path);
    std::ifstream in(potentials_path);
    if (!in.good()) { delete h; return nullptr; }
    h->field.readPotential(in, h->log, h->spec);
    for (int i = 0; i < 9; i++) h->lat[i] = lat[i];
    reciprocal(h->lat, h->rcp);
    const double md = min_dim_override > 0.0 ? min_dim_override : minimum_dimension(h->lat);
    h->field.setup(h->mpi, h->lat, h->rcp, md, volume(h->lat), max_atoms, h->spec, h->log);
    h->log.flush();
    return h;
}

REF_API int ref_num_species(void* hp)
{
    return static_cast<RefHandle*>(hp)->spec.getNumSpecies();
}

REF_API double ref_species_charge(void* hp, int i)
{
    return static_cast<RefHandle*>(hp)->spec.getSpecies(i).charge;
}

// energies[0..5] = total, rcp, real, vdw, many, getTotalEnergy()
REF_API void ref_forces(void* hp, int n, double* px, double* py, double* pz,
                        const double* charge, const int* label,
                        double* fx, double* fy, double* fz, double* stress, double* energies)
{
    RefHandle* h = static_cast<RefHandle*>(hp);
    std::vector<double> q(charge, charge + n);
    std::vector<int> lab(label, label + n);
    std::vector<int> frozen(n, 0);
    Energy eng;
    h->field.calculateForces(h->mpi, px, py, pz, fx, fy, fz, stress, h->lat, h->rcp,
                             q.data(), lab.data(), frozen.data(), n, eng);
    energies[0] = eng.totalEnergy;
    energies[1] = eng.rcpEnergy;
    energies[2] = eng.realEnergy;
    energies[3] = eng.vdwEnergy;
    energies[4] = eng.manyEnergy;
    energies[5] = eng.getTotalEnergy();
}

REF_API void ref_destroy(void* hp)
{
    delete static_cast<RefHandle*>(hp);
}

// The reference's own relaxation, Relax::RelaxStructure (optim/Relax.cpp:19-39) with
// method "fire" (Relax::FIRERelax, Euler update, optim/Relax.cpp:44-315) or "fire2".
// Positions are relaxed in place.  Returns the reference's status (0 success, 1 failed)
// and writes the final energies as ref_forces does.
REF_API int ref_relax(void* hp, const char* method, int n, double* px, double* py, double* pz,
                      const double* charge, const int* label, const int* frozen,
                      int max_iter, double norm_tol, double force_tol, double init_dt,
                      double max_dt, double* energies)
{
    RefHandle* h = static_cast<RefHandle*>(hp);
    std::vector<double> q(charge, charge + n);
    std::vector<int> lab(label, label + n);
    std::vector<int> frz(n, 0);
    Basis bas;
    bas.numberOfAtoms = n;
    for (int i = 0; i < n; i++) {
        frz[i] = frozen ? frozen[i] : 0;
        bas.numFrozenAtoms += frz[i] == 1;
    }
    bas.posX = px;
    bas.posY = py;
    bas.posZ = pz;
    bas.charge = q.data();
    bas.atmLabel = lab.data();
    bas.frozen = frz.data();
    for (int i = 0; i < 9; i++) {
        bas.latVector[i] = h->lat[i];
        bas.rcpVector[i] = h->rcp[i];
    }
    RelaxCntrl rc;
    rc.method = method;
    rc.maxIter = max_iter;
    rc.normTol = norm_tol;
    rc.forceTol = force_tol;
    rc.initTimeStep = init_dt;
    rc.maxTimeStep = max_dt;
    Energy eng;
    Status status;
    Relax relax;
    relax.RelaxStructure(h->mpi, bas, &h->field, n, rc, eng, status, h->log);
    energies[0] = eng.totalEnergy;
    energies[1] = eng.rcpEnergy;
    energies[2] = eng.realEnergy;
    energies[3] = eng.vdwEnergy;
    energies[4] = eng.manyEnergy;
    energies[5] = eng.getTotalEnergy();
    return status.getStatus();
}
