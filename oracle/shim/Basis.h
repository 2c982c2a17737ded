// Minimal stand-in for the reference's Basis class, whose header is absent from the
// reference tree.  It holds the fields that the Ewald sources (fragment insert/remove
// routines the force path never calls), the FIRE relaxation (optim/Relax.cpp) and the ART
// saddle search (optim/ART.cpp) name: freezeForces as Common/Basis.cpp:966-981 defines it,
// displaceAtoms as Common/Basis.cpp:880-897 defines it, and inert versions of the restart
// reader and the basin report that the ART driver reaches only on paths the harness does
// not take.  Test infrastructure only.
#pragma once
#include <cstdio>
#include <cstdlib>
#include <fstream>

class MPIComms;
class Species;
struct JobControl;

class Basis
{
public:
    int numberOfAtoms = 0;
    int numFrozenAtoms = 0;
    double *posX = nullptr, *posY = nullptr, *posZ = nullptr, *charge = nullptr;
    int *atmLabel = nullptr, *frozen = nullptr;
    double latVector[9] = {0.0};
    double rcpVector[9] = {0.0};

    // moves the unfrozen atoms by delta, three entries per unfrozen atom in atom order
    void displaceAtoms(const double* delta)
    {
        int j = 0;
        for (int i = 0; i < numberOfAtoms; i++) {
            if (frozen[i] == 0) {
                posX[i] += delta[j];
                posY[i] += delta[j + 1];
                posZ[i] += delta[j + 2];
                j += 3;
            }
        }
    }

    void inputBasis(int&, double&, const Species&, const JobControl&, std::ifstream&, std::ofstream&)
    {
        std::fprintf(stderr, "reference oracle: Basis::inputBasis is not available\n");
        std::abort();
    }

    void reportBasisDifference(const MPIComms&, Basis&, const Species&, double, std::ofstream&) {}

    void freezeForces(double* forceX, double* forceY, double* forceZ)
    {
        if (numFrozenAtoms == 0) return;
        for (int i = 0; i < numberOfAtoms; i++) {
            if (frozen[i] == 1) {
                forceX[i] = 0.0;
                forceY[i] = 0.0;
                forceZ[i] = 0.0;
            }
        }
    }
};
