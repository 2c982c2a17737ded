// The reference's own ART saddle search, unchanged, on the drop-in Field of this project.
//
// Compiled by oracle/Makefile (target `dropin`) from the reference's optim/ART.cpp and
// optim/Relax.cpp -- read in place -- with akmc_b200/cpp ahead of the reference's
// directories on the include path, so that the reference's `#include "Field.h"` resolves
// to akmc_b200/cpp/Field.h, and linked against libakmc_b200.so.  The SaddleSearch members
// and the dstev_ stand-in ART needs come from oracle/shim/art_support.cpp (the reference's
// optim/SaddleSearch.cpp needs MPI; LAPACK is absent).  Test infrastructure:
// tests/test_dropin.py runs it and compares with the same ART on the reference's own Field.
//
//   art_dropin <potentials> <configuration> <seed> <output> [maxParIter initDt maxDt forceTol]
//
// configuration file: "n" / nine lattice numbers (rows a, b, c) / n lines "label x y z"
// (the minimum).  seed file: n lines "dx dy dz", the starting displacement (its unit
// vector is the initial Lanczos vector).  output file: "status saddle_energy" / n lines
// "x y z" (the final positions).
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "ART.h"          // the reference's optim/ART.h (its Field is akmc_b200/cpp/Field.h)
#include "Species.h"      // the reference's potentials/Species.h
#include "art_support.h"

int main(int argc, char** argv)
{
    if (argc < 5) {
        std::fprintf(stderr, "usage: art_dropin potentials config seed out [maxParIter initDt maxDt forceTol]\n");
        return 2;
    }
    std::ifstream cfg(argv[2]);
    int n = 0;
    cfg >> n;
    double lat[9], rcp[9];
    for (double& v : lat) cfg >> v;
    std::vector<double> x(n), y(n), z(n), q(n, 0.0), seed(3 * (size_t)n);
    std::vector<int> lab(n), frozen(n, 0);
    for (int i = 0; i < n; i++) cfg >> lab[i] >> x[i] >> y[i] >> z[i];
    std::ifstream sd(argv[3]);
    for (double& v : seed) sd >> v;

    // reciprocal vectors in the reference's index layout (Basis::setRcpVec,
    // Common/Basis.cpp:987-1010)
    rcp[0] = lat[4] * lat[8] - lat[7] * lat[5];
    rcp[1] = lat[6] * lat[5] - lat[3] * lat[8];
    rcp[2] = lat[3] * lat[7] - lat[6] * lat[4];
    rcp[3] = lat[7] * lat[2] - lat[1] * lat[8];
    rcp[4] = lat[0] * lat[8] - lat[6] * lat[2];
    rcp[5] = lat[2] * lat[3] - lat[5] * lat[0];
    rcp[6] = lat[1] * lat[5] - lat[4] * lat[2];
    rcp[7] = lat[6] * lat[1] - lat[0] * lat[7];
    rcp[8] = lat[0] * lat[4] - lat[3] * lat[1];
    const double det = lat[0] * rcp[0] + lat[1] * rcp[3] + lat[2] * rcp[6];
    for (double& v : rcp) v /= det;

    MPIComms mpi;
    Species spec;
    std::ofstream log(std::string(argv[4]) + ".log");
    std::ifstream pot(argv[1]);
    Field fld;
    try {
        fld.readPotential(pot, log, spec);
        fld.setup(mpi, lat, rcp, 0.0, 0.0, n, spec, log);
        for (int i = 0; i < n; i++) q[i] = spec.getSpecies(lab[i]).charge;   // Basis::charge

        Basis basin1;
        basin1.numberOfAtoms = n;
        basin1.posX = x.data();
        basin1.posY = y.data();
        basin1.posZ = z.data();
        basin1.charge = q.data();
        basin1.atmLabel = lab.data();
        basin1.frozen = frozen.data();
        for (int i = 0; i < 9; i++) {
            basin1.latVector[i] = lat[i];
            basin1.rcpVector[i] = rcp[i];
        }
        Basis saddle;
        JobControl job;                  // ARTCntrl defaults (Common/ArtCntrl.h) except:
        job.artParameters.maxParIter = argc > 5 ? std::stoi(argv[5]) : 3000;
        const double init_dt = argc > 6 ? std::stod(argv[6]) : 0.0005;
        const double max_dt = argc > 7 ? std::stod(argv[7]) : 0.001;
        job.artParameters.initTimeStep = job.artParameters.initTimeStepPerp = init_dt;
        job.artParameters.maxTimeStep = job.artParameters.maxTimeStepPerp = max_dt;
        job.artParameters.forceTol = argc > 8 ? std::stod(argv[8]) : 1.0e-3;
        job.artParameters.goPeprepedicular = false;
        job.artParameters.debug = false;
        Energy e1, es;
        Status status;
        double centre[3] = {0.0, 0.0, 0.0};
        art_support_set_seed(seed.data());
        ART art;
        art.findSaddlePoint(mpi, spec, job, &fld, basin1, saddle, status, e1, es, centre, false, log);
        art_support_set_seed(nullptr);

        std::ofstream out(argv[4]);
        out.precision(17);
        out << status.getStatus() << " " << es.getTotalEnergy() << "\n";
        for (int i = 0; i < n; i++) out << x[i] << " " << y[i] << " " << z[i] << "\n";
    } catch (const std::exception& e) {
        std::fprintf(stderr, "art_dropin: %s\n", e.what());
        return 1;
    }
    return 0;
}
