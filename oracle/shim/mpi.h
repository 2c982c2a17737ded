// Stand-in for <mpi.h>, which is absent here: kmc/Event.h includes it directly.  The one
// MPI call kmc/Event.cpp makes outside MPIComms (Event::setPositions, on an out-of-range
// atom) aborts the single process.  MPI_Comm itself comes from Common/MPICommunicator.h
// under -DNOMPI.  Test infrastructure only.
#pragma once
#include <cstdio>
#include <cstdlib>

static const int MPI_COMM_WORLD = 0;

inline int MPI_Abort(int, int code)
{
    std::fprintf(stderr, "reference oracle: MPI_Abort(%d)\n", code);
    std::abort();
}
