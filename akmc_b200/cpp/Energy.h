// Energy record of the drop-in Field (akmc_b200/cpp/Field.h).
//
// The reference's optimisers read energies through the class Energy of its potential
// directory (potentials/metal/Energy.h:13-108, potentials/pair/Energy.h): public members
// named totalEnergy, rcpEnergy, realEnergy, vdwEnergy, manyEnergy, extEnergy,
// timeStepUnit and the accessors getTotalEnergy, getTimeStepUnit, getEnergyUnit,
// printEnergy.  Callers written against that class compile against this one: the
// member and method names are the interface and are kept; the bodies are this
// project's.  getTotalEnergy sums the components (rcp + real + vdw + many + ext), as
// the reference does.
#pragma once

#include <fstream>
#include <iomanip>
#include <string>

class Energy
{
public:
    double totalEnergy = 0.0, rcpEnergy = 0.0, selfEnergy = 0.0, realEnergy = 0.0,
           manyEnergy = 0.0, vdwEnergy = 0.0, extEnergy = 0.0;
    double timeStepUnit = 9648.530821;              // eV/(A amu) -> A/ps^2
    double boltzmann = 8.617333262145e-5;           // eV/K
    std::string energyUnit = " eV";

    std::string getEnergyUnit(void) { return energyUnit; }
    void setEnergyUnit(std::string unit) { energyUnit = unit; }
    void setTotalEnergy(double e) { totalEnergy = e; }
    double getTotalEnergy(void) { return rcpEnergy + realEnergy + vdwEnergy + manyEnergy + extEnergy; }
    double getTimeStepUnit(void) { return timeStepUnit; }
    void setTimeStepUnit(double u) { timeStepUnit = u; }
    double getBoltzmannConstant(void) { return boltzmann; }

    void zero(void)
    {
        totalEnergy = rcpEnergy = selfEnergy = realEnergy = manyEnergy = vdwEnergy = extEnergy = 0.0;
    }

    void printEnergy(int box, std::ofstream& out)
    {
        out << std::scientific << std::setprecision(10)
            << " energies (system " << box << ")" << energyUnit << "\n"
            << "   reciprocal space " << rcpEnergy << "\n"
            << "   real space       " << realEnergy << "\n"
            << "   short range      " << vdwEnergy << "\n"
            << "   many body        " << manyEnergy << "\n"
            << "   external         " << extEnergy << "\n"
            << "   total            " << getTotalEnergy() << std::endl;
    }
};
