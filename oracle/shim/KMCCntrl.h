// Empty stand-in for the reference's KMC controls, whose header is absent from the
// reference tree.  Only its name is needed (a member of JobControl, which the relaxation
// sources include but do not use).  Test infrastructure only.
#pragma once
struct KMCCntrl
{
};
