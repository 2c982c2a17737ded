// Definitions the reference's potential sources need at link time but whose
// implementation files are absent from the reference tree (MPICommunicator.cpp) or
// live in the driver (getRandomNumber in kmc/kmc.cpp). Single-process, no MPI.
// Test infrastructure only.
#include <cstdio>
#include <cstdlib>
#include "MPICommunicator.h"

MPIComms::MPIComms() {}
MPIComms::~MPIComms() {}
void MPIComms::commsAbortWorld(void) const
{
    std::fprintf(stderr, "reference oracle: commsAbortWorld called\n");
    std::abort();
}
double getRandomNumber(void) { return 0.5; }
