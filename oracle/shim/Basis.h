// Minimal stand-in for the reference's Basis class: the Ewald sources only name the
// fields below (fragment insert/remove routines that the force path never calls).
// Test infrastructure only.
#pragma once
class Basis
{
public:
    int numberOfAtoms = 0;
    double *posX = nullptr, *posY = nullptr, *posZ = nullptr, *charge = nullptr;
};
