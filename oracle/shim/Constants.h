// Constants header for building the reference's potential sources as a test oracle.
// The reference includes "Constants.h" but does not ship it; these values are fixed
// once here and shared by the oracle restatement and the CUDA path (akmc_constants.h).
// Test infrastructure only: nothing in the product links this file.
#pragma once
#include <cmath>

const double PI = 3.14159265358979323846;
const double TWOPI = 2.0 * PI;
const double ROOTPI = 1.77245385090551602730;
// e^2 / (4 pi eps0) in eV * Angstrom
const double CTOEV = 14.3996454784;
// converts the FIRE time step (ps, eV, Angstrom, amu) into internal units
const double EVTODL = 9648.530821;
const double BOLTZMANN = 8.617333262145e-5;
const int MAXMESH = 5000;
const int DOFFSET = 64;

enum statusvalues { SUCCESS = 0, FAILED = 1, INTERRUPTED = 3, TERMINATED = 4 };
