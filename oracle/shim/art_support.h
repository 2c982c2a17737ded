// The starting displacement ([n][3], atom order) of the next ART search (art_support.cpp);
// the pointer must stay valid until that search returns.  Test infrastructure only.
#pragma once
void art_support_set_seed(const double* seed);
