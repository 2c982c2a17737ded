// The reference's own ART saddle search (optim/ART.cpp, compiled unchanged from the reference
// tree) driven on the reference's own EAM Field, as an oracle for saddle energies.
// Test infrastructure only: the product never links or calls it.
//
// ART::findSaddlePoint (optim/ART.cpp:17-131) calls three SaddleSearch members whose source
// file (optim/SaddleSearch.cpp) needs MPI; they are defined here.  Every atom is active (the
// reference's global region, regionStyle 1), and instead of a random displacement the search
// starts from a given one: the atoms are moved by it and the initial Lanczos vector is its
// unit vector -- what SaddleSearch::makeGaussDisplacement (optim/SaddleSearch.cpp:423-490)
// does with the displacement it draws.  LAPACK's dstev_, which ART calls for the lowest
// eigenpair of the Lanczos tridiagonal matrix (optim/ART.cpp:764-793), is absent here; a
// cyclic Jacobi eigensolver written for this harness stands in for it.
#include <algorithm>
#include <cmath>
#include <fstream>
#include <string>
#include <vector>

#include "ART.h"
#include "ref_handle.h"

#define REF_API extern "C" __attribute__((visibility("default")))

namespace {
const double* g_seed = nullptr;      // the starting displacement of the next search, [n][3]

void place_seed(Basis& bas, int vectorSize, double*& rVector)
{
    rVector = alloc_dvector(vectorSize, "ART::rVector", 0.0);
    double norm = 0.0;
    for (int i = 0; i < vectorSize; i++) norm += g_seed[i] * g_seed[i];
    norm = std::sqrt(norm);
    for (int i = 0; i < vectorSize; i++) rVector[i] = g_seed[i] / norm;
    bas.displaceAtoms(g_seed);
}
}  // namespace

SaddleSearch::SaddleSearch() {}
SaddleSearch::~SaddleSearch() {}

void SaddleSearch::constructActiveRegion(const MPIComms&, Basis& bas, const Species&, const JobControl&,
                                         double* centre, std::ofstream&)
{
    bas.numFrozenAtoms = 0;
    for (int i = 0; i < bas.numberOfAtoms; i++) bas.frozen[i] = 0;
    vectorSize = 3 * bas.numberOfAtoms;
    centre[0] = centre[1] = centre[2] = 0.0;
}

void SaddleSearch::makeGaussDisplacement(const MPIComms&, Basis& bas, double*, double, double, std::ofstream&)
{
    place_seed(bas, vectorSize, rVector);
}

void SaddleSearch::makeRandomDisplacement(const MPIComms&, Basis& bas, double, std::ofstream&)
{
    place_seed(bas, vectorSize, rVector);
}

// Eigenvalues (ascending, in d) and eigenvectors (columns of z, n x n, column-major as
// LAPACK returns them) of the symmetric tridiagonal matrix with diagonal d and sub-diagonal
// e: cyclic Jacobi rotations on the dense matrix until the off-diagonal mass is below
// 1e-30 of the total.  Only jobz = 'V' is supported; info = 0.
extern "C" int dstev_(char* jobz, int* n_in, double* d, double* e, double* z, int* ldz, double*, int* info)
{
    const int n = *n_in, ld = *ldz;
    *info = 0;
    if (*jobz != 'V' || n < 1 || ld < n) {
        *info = -1;
        return 0;
    }
    std::vector<double> A((size_t)n * n, 0.0), V((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++) {
        A[(size_t)i * n + i] = d[i];
        if (i + 1 < n) A[(size_t)i * n + i + 1] = A[(size_t)(i + 1) * n + i] = e[i];
        V[(size_t)i * n + i] = 1.0;
    }
    auto a = [&](int r, int c) -> double& { return A[(size_t)r * n + c]; };
    double total = 0.0;
    for (double x : A) total += x * x;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0;
        for (int p = 0; p < n; p++)
            for (int q = p + 1; q < n; q++) off += a(p, q) * a(p, q);
        if (off <= 1e-30 * total) break;
        for (int p = 0; p < n; p++) {
            for (int q = p + 1; q < n; q++) {
                if (a(p, q) == 0.0) continue;
                // rotation that zeroes a(p, q): tan(2 theta) = 2 a_pq / (a_qq - a_pp)
                const double theta = 0.5 * std::atan2(2.0 * a(p, q), a(q, q) - a(p, p));
                const double c = std::cos(theta), s = std::sin(theta);
                for (int k = 0; k < n; k++) {             // columns p, q: A <- A J
                    const double akp = a(k, p), akq = a(k, q);
                    a(k, p) = c * akp - s * akq;
                    a(k, q) = s * akp + c * akq;
                }
                for (int k = 0; k < n; k++) {             // rows p, q: A <- J^T A
                    const double apk = a(p, k), aqk = a(q, k);
                    a(p, k) = c * apk - s * aqk;
                    a(q, k) = s * apk + c * aqk;
                }
                for (int k = 0; k < n; k++) {             // eigenvectors: V <- V J
                    const double vkp = V[(size_t)k * n + p], vkq = V[(size_t)k * n + q];
                    V[(size_t)k * n + p] = c * vkp - s * vkq;
                    V[(size_t)k * n + q] = s * vkp + c * vkq;
                }
            }
        }
    }
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int x, int y) { return a(x, x) < a(y, y); });
    std::vector<double> ev(n);
    for (int i = 0; i < n; i++) ev[i] = a(order[i], order[i]);
    for (int i = 0; i < n; i++) {
        d[i] = ev[i];
        for (int k = 0; k < n; k++) z[(size_t)i * ld + k] = V[(size_t)k * n + order[i]];
    }
    return 0;
}

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
    g_seed = seed;
    ART art;
    art.findSaddlePoint(h->mpi, h->spec, job, &h->field, basin1, saddle, status, e1, es, centre, false, h->log);
    g_seed = nullptr;
    energies[0] = es.getTotalEnergy();
    return status.getStatus();
}
