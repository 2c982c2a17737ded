// The reference's event record (kmc/Event.cpp, compiled unchanged from the reference tree)
// behind a C entry point: Event::Event(int*, float*, int, double, double) computes the
// harmonic-TST rate prefactor * exp(-E_a / (k_B T)) from the float record the KMC task farm
// sends (kmc/Event.cpp:66-105; E_a at vecf[6 natoms + 3]).  Test infrastructure only.
#include "Event.h"

extern "C" __attribute__((visibility("default")))
double ref_event_rate(double e_act, double prefactor, double temperature, double* e_act_stored)
{
    int veci[1] = {0};
    float vecf[6 + 7] = {0.0f};
    vecf[6 + 3] = (float)e_act;         // the record carries E_a as float
    Event e(veci, vecf, 1, prefactor, temperature);
    if (e_act_stored) *e_act_stored = e.getActivationEnergy();
    return e.getRate();
}
