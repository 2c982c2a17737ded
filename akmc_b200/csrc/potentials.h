// Host-side potential description and the reference-format readers.
#pragma once

#include <string>
#include <vector>

#include "akmc_internal.h"

namespace akmc {

struct Potentials {
    int family = 0;                      // AKMC_FAMILY_EAM or AKMC_FAMILY_IONIC
    double cutoff = 15.0;                // shortRangeCut default (metal/Field.h:53)
    bool use_nbrlist = false;
    double verlet_shell = 0.0;           // metal -0.5 (metal/Field.h:57), pair 1.0 (pair/Field.h:66)
    bool minimum_image = true;
    std::vector<SpeciesRec> species;
    // EAM
    std::vector<EamTable> eam;
    std::vector<int> eam_mesh;           // [ns*ns], -1 = no potential
    // ionic
    std::vector<BuckRec> buck;
    std::vector<int> buck_mesh;          // [ns*ns], default 0 (TwoBody.cpp:509)
    int do_ewald = 1;                    // pair/Field.h default; 1 = Ewald sum, 0 = none
    double precis = 1.0e-6;              // madelungAcc default
    double cfact = 1.0;                  // set to CTOEV by `twobody`
};

// Parse a `potentials` file.  Returns AKMC_OK or an error code; msg explains failures.
akmc_status read_potentials(const std::string& path, Potentials& out, std::string& msg);
// The same reader on the text of a potentials file (the reference reads from a stream).
akmc_status read_potentials_text(const std::string& text, Potentials& out, std::string& msg);
akmc_status read_potential_lines(const std::vector<std::string>& lines, const std::string& source,
                                 Potentials& out, std::string& msg);

// Ewald parameters of Field::setup / Ewald::setEwaldImage / findGvector for an
// orthorhombic cell with edge lengths L[3].
struct EwaldSet {
    double eta = 0.0;
    int gcell[3] = {0, 0, 0};
    std::vector<int> nx, ny, nz;
    std::vector<double> g0;
};
akmc_status ewald_setup(double precis, double cutoff, const double lat[9], const double rcp[9],
                        EwaldSet& out, std::string& msg);

void reciprocal_vectors(const double lat[9], double rcp[9]);

}  // namespace akmc
