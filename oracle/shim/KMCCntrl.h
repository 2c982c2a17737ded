// Stand-in for the reference's KMC controls, whose header is absent from the reference
// tree: the members the relaxation and ART sources name (the ART driver reads the seeding
// choice and the basin radius of its report).  Test infrastructure only.
#pragma once
struct KMCCntrl
{
    bool useGauss = false;
    double gaussWidth = 1.0;
    double kmcBasinRadius = 0.1;
};
