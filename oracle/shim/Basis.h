// Minimal stand-in for the reference's Basis class, whose header is absent from the
// reference tree.  It holds the fields that the Ewald sources (fragment insert/remove
// routines the force path never calls) and the FIRE relaxation (optim/Relax.cpp) name,
// and freezeForces as Common/Basis.cpp:966-981 defines it.  Test infrastructure only.
#pragma once
class Basis
{
public:
    int numberOfAtoms = 0;
    int numFrozenAtoms = 0;
    double *posX = nullptr, *posY = nullptr, *posZ = nullptr, *charge = nullptr;
    int *atmLabel = nullptr, *frozen = nullptr;
    double latVector[9] = {0.0};
    double rcpVector[9] = {0.0};

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
