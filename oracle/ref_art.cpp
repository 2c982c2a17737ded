// The reference's own ART saddle search (optim/ART.cpp, compiled unchanged from the reference
// tree) driven on the reference's own EAM Field, as an oracle for saddle energies.
// Test infrastructure only: the product never links or calls it.  The SaddleSearch members
// and the dstev_ stand-in ART needs are in shim/art_support.cpp.
#include <vector>

#include "ART.h"
#include "art_support.h"
#include "ref_handle.h"

#define REF_API extern "C" __attribute__((visibility("default")))

// One ART search from the minimum pos (relaxed) plus seed, on the reference's own Field:
// ART::findSaddlePoint with the ARTCntrl defaults (Common/ArtCntrl.h) except those given
// (the FIRE time steps: the defaults, 0.005 -> 0.01 in the Energy time unit, move the atoms of
// the metal workloads by about 1 A per step and drive the reference's embedding out of its
// table, where the reference Field exits).  The search climbs only from a start whose lowest
// curvature is already negative: from a positive-curvature start this ART relaxes the
// perpendicular forces and returns to the minimum.  pos receives the final positions;
// energies[0] the saddle's total energy.  Returns the reference's status (0 success).
REF_API int ref_art(void* hp, int n, double* px, double* py, double* pz, const double* charge,
                    const int* label, const double* seed, int max_par_iter, double force_tol,
                    int go_perpendicular, double init_dt, double max_dt, double* energies)
{
    RefHandle* h = static_cast<RefHandle*>(hp);
    std::vector<double> q(charge, charge + n);
    std::vector<int> lab(label, label + n);
    std::vector<int> frz(n, 0);
    Basis basin1;
    basin1.numberOfAtoms = n;
    basin1.posX = px;
    basin1.posY = py;
    basin1.posZ = pz;
    basin1.charge = q.data();
    basin1.atmLabel = lab.data();
    basin1.frozen = frz.data();
    for (int i = 0; i < 9; i++) {
        basin1.latVector[i] = h->lat[i];
        basin1.rcpVector[i] = h->rcp[i];
    }
    Basis saddle;
    JobControl job;
    job.artParameters.maxParIter = max_par_iter;
    job.artParameters.forceTol = force_tol;
    job.artParameters.goPeprepedicular = go_perpendicular != 0;
    job.artParameters.initTimeStep = job.artParameters.initTimeStepPerp = init_dt;
    job.artParameters.maxTimeStep = job.artParameters.maxTimeStepPerp = max_dt;
    job.artParameters.debug = false;
    Energy e1, es;
    Status status;
    double centre[3] = {0.0, 0.0, 0.0};
    art_support_set_seed(seed);
    ART art;
    art.findSaddlePoint(h->mpi, h->spec, job, &h->field, basin1, saddle, status, e1, es, centre, false, h->log);
    art_support_set_seed(nullptr);
    energies[0] = es.getTotalEnergy();
    return status.getStatus();
}
