// The state of one reference Field instance behind the oracle's C entry points
// (ref_harness.cpp, ref_art.cpp).  Test infrastructure only.
#pragma once
#include <fstream>

#include "Field.h"

struct RefHandle
{
    MPIComms mpi;
    Species spec;
    Field field;
    std::ofstream log;
    double lat[9];
    double rcp[9];
};
