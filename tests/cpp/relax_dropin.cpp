// The reference's own relaxation driver, unchanged, on the drop-in Field of this project.
//
// Compiled by oracle/Makefile (target `dropin`) from the reference's optim/Relax.cpp,
// potentials/Species.cpp and Common/Utility.cpp -- read in place -- with akmc_b200/cpp
// ahead of the reference's directories on the include path, so that Relax.cpp's
// `#include "Field.h"` resolves to akmc_b200/cpp/Field.h, and linked against
// libakmc_b200.so.  Test infrastructure: tests/test_gpu_dropin.py runs it and compares
// with the reference's own FIRE on its own Field.
//
//   relax_dropin <potentials file> <configuration file> <output file> [fire|fire2] [maxIter]
//
// configuration file: "n" / nine lattice numbers (rows a, b, c) / n lines "label x y z".
// output file: "status energy" / n lines "x y z" (relaxed, wrapped positions).
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "Field.h"        // akmc_b200/cpp/Field.h
#include "Relax.h"        // the reference's optim/Relax.h
#include "Species.h"      // the reference's potentials/Species.h

int main(int argc, char** argv)
{
    if (argc < 4) {
        std::fprintf(stderr, "usage: relax_dropin potentials config out [fire|fire2]\n");
        return 2;
    }
    std::ifstream cfg(argv[2]);
    int n = 0;
    cfg >> n;
    double lat[9], rcp[9];
    for (double& v : lat) cfg >> v;
    std::vector<double> x(n), y(n), z(n), q(n, 0.0);
    std::vector<int> lab(n), frozen(n, 0);
    for (int i = 0; i < n; i++) cfg >> lab[i] >> x[i] >> y[i] >> z[i];

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
    std::ofstream log(std::string(argv[3]) + ".log");
    std::ifstream pot(argv[1]);
    Field fld;
    try {
        fld.readPotential(pot, log, spec);
        fld.setup(mpi, lat, rcp, 0.0, 0.0, n, spec, log);
        for (int i = 0; i < n; i++) q[i] = spec.getSpecies(lab[i]).charge;   // Basis::charge

        Basis bas;
        bas.numberOfAtoms = n;
        bas.posX = x.data();
        bas.posY = y.data();
        bas.posZ = z.data();
        bas.charge = q.data();
        bas.atmLabel = lab.data();
        bas.frozen = frozen.data();
        for (int i = 0; i < 9; i++) {
            bas.latVector[i] = lat[i];
            bas.rcpVector[i] = rcp[i];
        }
        RelaxCntrl rc;
        if (argc > 4) rc.method = argv[4];
        if (argc > 5) rc.maxIter = std::stoi(argv[5]);
        Energy eng;
        Status status;
        Relax relax;
        relax.RelaxStructure(mpi, bas, &fld, n, rc, eng, status, log);

        std::ofstream out(argv[3]);
        out.precision(17);
        out << status.getStatus() << " " << eng.getTotalEnergy() << "\n";
        for (int i = 0; i < n; i++) out << x[i] << " " << y[i] << " " << z[i] << "\n";
    } catch (const std::exception& e) {
        std::fprintf(stderr, "relax_dropin: %s\n", e.what());
        return 1;
    }
    return 0;
}
