// Drop-in replacement for the reference's force field class, over the C ABI (akmc.h).
//
// The reference selects its Field at compile time: potentials/metal/Field.h:126-219 (EAM)
// or potentials/pair/Field.h:658-748 (Buckingham + Ewald); its optimisers (optim/Relax.cpp,
// optim/ART.cpp, optim/Dimer.cpp) and the KMC driver (kmc/kmc.cpp:188-221) call it through
// the methods below.  A caller compiled with this directory ahead of the reference's
// potential directory on the include path gets the GPU path with no source change: same
// class name, method names, argument lists and meanings.  Both families are served by the
// one class (the family comes from the potentials file).
//
// Behaviour kept from the reference: positions are wrapped into the minimum-image cell in
// place by calculateForces; forces are overwritten; units A, eV, eV/A.  Changed: the
// reference exits the process on bad input (metal/Field.cpp:35-60, ManyBody.cpp:603-608);
// here every failure throws std::runtime_error carrying the C-ABI status and message --
// the exception ART already catches around its force calls (optim/ART.cpp:489-510).
// calculateConfig / calculateEnergy return the energies of the force path: the reference's
// EAM energy-only path counts each pair twice (ManyBody.cpp:449), which is not reproduced.
#pragma once

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iterator>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <unistd.h>
#include <utility>
#include <vector>

#include "Energy.h"
#include "akmc.h"

class MPIComms;   // the reference's communicator: accepted, not used (one process per GPU)

namespace akmc_dropin {

inline void check(akmc_status st, const char* where)
{
    if (st != AKMC_OK)
        throw std::runtime_error(std::string(where) + ": status " + std::to_string(st) + ": " +
                                 akmc_last_error());
}

// Does the caller's species class read "name mass charge" lines from a file stream, as
// Species::loadSpecies (potentials/Species.cpp:31-70) does?
template <class S, class = void>
struct has_load_species : std::false_type {};
template <class S>
struct has_load_species<S, std::void_t<decltype(std::declval<S&>().loadSpecies(
                               std::declval<std::ifstream&>(), 0))>> : std::true_type {};

}  // namespace akmc_dropin

class Field
{
public:
    Field() = default;
    virtual ~Field()
    {
        if (f_) akmc_field_destroy(f_);
    }
    Field(const Field&) = delete;
    Field& operator=(const Field&) = delete;

    // The GPU path follows the minimum-image convention (metal/Field.h:137-138).
    bool getImageConvention() { return true; }

    // Field::readPotential: the rest of the potentials stream; fills the caller's species
    // table through its own loadSpecies when it has one.
    template <class SpeciesT>
    void readPotential(std::ifstream& inStream, std::ofstream& outStream, SpeciesT& spec)
    {
        std::string text((std::istreambuf_iterator<char>(inStream)), std::istreambuf_iterator<char>());
        if (f_) {
            akmc_field_destroy(f_);
            f_ = nullptr;
        }
        akmc_dropin::check(akmc_field_create_from_text(text.c_str(), &f_), "Field::readPotential");
        const int n = akmc_field_num_species(f_);
        if constexpr (akmc_dropin::has_load_species<SpeciesT>::value) {
            std::string tmpl = (std::filesystem::temp_directory_path() / "akmc_species_XXXXXX").string();
            std::vector<char> pbuf(tmpl.begin(), tmpl.end());
            pbuf.push_back('\0');
            char* path = pbuf.data();
            const int fd = mkstemp(path);
            if (fd < 0) throw std::runtime_error("Field::readPotential: no temporary file");
            close(fd);
            {
                std::ofstream sp(path);
                for (int i = 0; i < n; i++) {
                    char name[16];
                    double mass = 0.0, charge = 0.0;
                    akmc_field_species(f_, i, name, &mass, &charge);
                    sp << name << " " << std::setprecision(17) << mass << " " << charge << "\n";
                }
            }
            std::ifstream sp(path);
            spec.loadSpecies(sp, n);
            unlink(path);
        }
        print(outStream);
    }

    // Field::setup: cutoff check against the cell, Ewald parameters, device tables.
    // minDimension and volume are recomputed from the lattice.
    template <class SpeciesT>
    void setup(const MPIComms&, double* latVector, double* rcpVector, double /*minDimension*/,
               double /*volume*/, int numAtoms, const SpeciesT&, std::ofstream& outStream)
    {
        require();
        akmc_dropin::check(akmc_field_setup(f_, latVector, rcpVector, numAtoms), "Field::setup");
        for (int i = 0; i < 9; i++) lat_[i] = latVector[i];
        double eta = 0.0;
        int nk = 0, g[3] = {0, 0, 0};
        if (akmc_field_family(f_) == AKMC_FAMILY_IONIC && akmc_field_ewald(f_, &eta, &nk, g) == AKMC_OK)
            outStream << " Ewald: eta " << eta << " 1/A, " << nk << " k-vectors, cells " << g[0]
                      << " " << g[1] << " " << g[2] << std::endl;
    }

    // Field::calculateForces (metal/Field.h:192-193).  stress is written as zeros.
    void calculateForces(const MPIComms&, double* posX, double* posY, double* posZ, double* forceX,
                         double* forceY, double* forceZ, double* stress, double* /*latVector*/,
                         double* /*rcpVector*/, double* atomcharge, int* intlabel, int* /*frozen*/,
                         int numatoms, Energy& eng)
    {
        require();
        akmc_energy e{};
        double s[6];
        akmc_dropin::check(akmc_forces(f_, numatoms, posX, posY, posZ, intlabel, atomcharge, forceX,
                                       forceY, forceZ, stress ? stress : s, &e),
                           "Field::calculateForces");
        store(e, eng);
    }

    // Field::calculateConfig: energy of a configuration (forces computed and dropped).
    void calculateConfig(const MPIComms& mpi, double* posX, double* posY, double* posZ,
                         double* latVector, double* rcpVector, double* atomcharge, int* intlabel,
                         int* frozen, int numatoms, Energy& eng)
    {
        fx_.assign((size_t)numatoms, 0.0);
        fy_.assign((size_t)numatoms, 0.0);
        fz_.assign((size_t)numatoms, 0.0);
        double stress[6];
        calculateForces(mpi, posX, posY, posZ, fx_.data(), fy_.data(), fz_.data(), stress, latVector,
                        rcpVector, atomcharge, intlabel, frozen, numatoms, eng);
    }

    void calculateEnergy(const MPIComms& mpi, double* posX, double* posY, double* posZ,
                         double* latVector, double* rcpVector, double* atomcharge, int* intlabel,
                         int* frozen, int numatoms, Energy& eng)
    {
        calculateConfig(mpi, posX, posY, posZ, latVector, rcpVector, atomcharge, intlabel, frozen,
                        numatoms, eng);
    }

    // Field::resetSimulationCellMinImage (metal/Field.cpp:1894-1920): fractional coordinates
    // s = r . rcp (columns of rcpVector), s -= rint(s), r = s . lat.
    void resetSimulationCellMinImage(const MPIComms&, double* posX, double* posY, double* posZ,
                                     double* latVector, double* rcpVector, int natoms)
    {
        for (int i = 0; i < natoms; i++) {
            double s[3];
            for (int d = 0; d < 3; d++) {
                s[d] = posX[i] * rcpVector[d] + posY[i] * rcpVector[3 + d] + posZ[i] * rcpVector[6 + d];
                s[d] -= std::rint(s[d]);
            }
            posX[i] = s[0] * latVector[0] + s[1] * latVector[3] + s[2] * latVector[6];
            posY[i] = s[0] * latVector[1] + s[1] * latVector[4] + s[2] * latVector[7];
            posZ[i] = s[0] * latVector[2] + s[1] * latVector[5] + s[2] * latVector[8];
        }
    }

    void print(const MPIComms&, std::ofstream& outStream) { print(outStream); }

    // The GPU path keeps no per-move state: these reference hooks have nothing to do.
    void tidy(const MPIComms&) {}
    void updatePhaseSum(void) {}
    void resetAtomMove(int) {}

    // The underlying C-ABI handle, for batched calls (akmc_batch_*, akmc_walkers_*).
    akmc_field* handle() const { return f_; }

private:
    akmc_field* f_ = nullptr;
    double lat_[9] = {0.0};
    std::vector<double> fx_, fy_, fz_;

    void require() const
    {
        if (!f_) throw std::runtime_error("Field: readPotential must come first");
    }

    static void store(const akmc_energy& e, Energy& eng)
    {
        eng.rcpEnergy = e.rcp;
        eng.realEnergy = e.real;
        eng.vdwEnergy = e.vdw;
        eng.manyEnergy = e.many;
        eng.totalEnergy = e.total;
    }

    void print(std::ofstream& out)
    {
        if (!f_) return;
        out << " force field on the GPU (" << akmc_version() << "): "
            << (akmc_field_family(f_) == AKMC_FAMILY_EAM ? "EAM" : "Buckingham + Ewald")
            << ", cutoff " << akmc_field_cutoff(f_) << " A" << std::endl;
        for (int i = 0; i < akmc_field_num_species(f_); i++) {
            char name[16];
            double mass = 0.0, charge = 0.0;
            akmc_field_species(f_, i, name, &mass, &charge);
            out << "   species " << i << " " << name << " mass " << mass << " charge " << charge
                << std::endl;
        }
    }
};
