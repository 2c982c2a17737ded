// Reference-format readers and Ewald set-up (host).
//
// The keyword loops follow the reference's Field::readPotential for each family
// (potentials/metal/Field.cpp:122-205, potentials/pair/Field.cpp:215-317): lines are
// lower-cased before the keyword test, `species N` reads N lines "name mass charge [Z]"
// (potentials/Species.cpp:31-70), `manybody N unit` reads N entries of a type line and a
// parameter line (potentials/metal/ManyBody.cpp:188-305), `twobody N ...` does the same
// for pair potentials (potentials/pair/TwoBody.cpp:56-266), `close` ends the file, and any
// other keyword is an error.  Forms outside this path (analytic many-body potentials,
// Morse/LJ/BHM/7-6, damped Coulomb, `noimage`) are rejected with AKMC_ERR_UNSUPPORTED.
#include "potentials.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace akmc {

namespace {

std::vector<std::string> split(const std::string& s)
{
    std::vector<std::string> w;
    std::istringstream ss(s);
    std::string x;
    while (ss >> x) w.push_back(x);
    return w;
}

std::string lower(std::string s)
{
    std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return std::tolower(c); });
    return s;
}

bool to_double(const std::string& s, double& v)
{
    const char* b = s.c_str();
    char* e = nullptr;
    v = std::strtod(b, &e);
    return e != b;
}

bool to_int(const std::string& s, int& v)
{
    const char* b = s.c_str();
    char* e = nullptr;
    long x = std::strtol(b, &e, 10);
    v = (int)x;
    return e != b;
}

// MetalPotential::readParameters (MetalPotential.cpp:363-386): whole lines, every word.
bool read_values(std::ifstream& in, std::vector<double>& v, int n)
{
    v.assign((size_t)n, 0.0);
    int id = 0;
    std::string line;
    while (id < n) {
        if (!std::getline(in, line)) return false;
        for (const auto& w : split(line)) {
            if (id >= n) return false;      // the reference would write past the table
            double x;
            if (!to_double(w, x)) return false;
            v[(size_t)id++] = x;
        }
    }
    return true;
}

// MetalPotential::calculateDerivativeMesh (MetalPotential.cpp:388-392); deriv[n-1] = 0.
std::vector<double> forward_difference(const std::vector<double>& p, double dr)
{
    std::vector<double> d(p.size(), 0.0);
    for (size_t i = 0; i + 1 < p.size(); i++) d[i] = (p[i + 1] - p[i]) / dr;
    return d;
}

// MetalPotential::readLEAM (MetalPotential.cpp:276-361).
akmc_status read_setfl(const std::string& file, EamTable& t, std::string& msg)
{
    std::ifstream in(file);
    if (!in.good()) { msg = "cannot open EAM table " + file; return AKMC_ERR_IO; }
    std::string line;
    for (int k = 0; k < 4; k++) std::getline(in, line);
    std::getline(in, line);
    auto w = split(line);
    if (w.size() < 5 || !to_int(w[0], t.n_embed) || !to_double(w[1], t.step_embed) ||
        !to_int(w[2], t.n_r) || !to_double(w[3], t.step_r) || !to_double(w[4], t.pot_cutoff) ||
        t.n_embed < 2 || t.n_r < 2 || !(t.step_embed > 0) || !(t.step_r > 0)) {
        msg = "malformed setfl header in " + file;
        return AKMC_ERR_PARSE;
    }
    std::getline(in, line);
    std::vector<double> rphi;
    if (!read_values(in, t.F, t.n_embed) || !read_values(in, t.rho, t.n_r) ||
        !read_values(in, rphi, t.n_r)) {
        msg = "truncated or malformed setfl tables in " + file;
        return AKMC_ERR_PARSE;
    }
    t.phi.resize((size_t)t.n_r);
    for (int i = 0; i < t.n_r; i++) t.phi[(size_t)i] = rphi[(size_t)i] / (i * t.step_r);  // NaN at 0
    t.dF = forward_difference(t.F, t.step_embed);
    t.drho = forward_difference(t.rho, t.step_r);
    t.dphi = forward_difference(t.phi, t.step_r);
    return AKMC_OK;
}

void dcell(const double* a, double* b)
{
    // Common/Utility.cpp:23-84: lengths, cosines, perpendicular widths, volume
    b[0] = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    b[1] = std::sqrt(a[3] * a[3] + a[4] * a[4] + a[5] * a[5]);
    b[2] = std::sqrt(a[6] * a[6] + a[7] * a[7] + a[8] * a[8]);
    b[3] = (a[0] * a[3] + a[1] * a[4] + a[2] * a[5]) / (b[0] * b[1]);
    b[4] = (a[0] * a[6] + a[1] * a[7] + a[2] * a[8]) / (b[0] * b[2]);
    b[5] = (a[3] * a[6] + a[4] * a[7] + a[5] * a[8]) / (b[1] * b[2]);
    const double axb1 = a[1] * a[5] - a[2] * a[4], axb2 = a[2] * a[3] - a[0] * a[5],
                 axb3 = a[0] * a[4] - a[1] * a[3];
    const double bxc1 = a[4] * a[8] - a[5] * a[7], bxc2 = a[5] * a[6] - a[3] * a[8],
                 bxc3 = a[3] * a[7] - a[4] * a[6];
    const double cxa1 = a[7] * a[2] - a[1] * a[8], cxa2 = a[0] * a[8] - a[2] * a[6],
                 cxa3 = a[1] * a[6] - a[0] * a[7];
    b[9] = std::fabs(a[0] * bxc1 + a[1] * bxc2 + a[2] * bxc3);
    b[6] = b[9] / std::sqrt(bxc1 * bxc1 + bxc2 * bxc2 + bxc3 * bxc3);
    b[7] = b[9] / std::sqrt(cxa1 * cxa1 + cxa2 * cxa2 + cxa3 * cxa3);
    b[8] = b[9] / std::sqrt(axb1 * axb1 + axb2 * axb2 + axb3 * axb3);
}

}  // namespace

void reciprocal_vectors(const double L[9], double R[9])
{
    // Basis::setRcpVec index layout (Common/Basis.cpp:987-1010)
    R[0] = L[4] * L[8] - L[7] * L[5];
    R[1] = L[6] * L[5] - L[3] * L[8];
    R[2] = L[3] * L[7] - L[6] * L[4];
    R[3] = L[7] * L[2] - L[1] * L[8];
    R[4] = L[0] * L[8] - L[6] * L[2];
    R[7] = L[6] * L[1] - L[0] * L[7];
    R[6] = L[1] * L[5] - L[4] * L[2];
    R[5] = L[2] * L[3] - L[5] * L[0];
    R[8] = L[0] * L[4] - L[3] * L[1];
    const double det = L[0] * R[0] + L[1] * R[3] + L[2] * R[6];
    const double f = std::fabs(det) > 0.0 ? 1.0 / det : 1.0;
    for (int i = 0; i < 9; i++) R[i] *= f;
}

akmc_status read_potentials(const std::string& path, Potentials& P, std::string& msg)
{
    std::ifstream in(path);
    if (!in.good()) { msg = "cannot open potentials file " + path; return AKMC_ERR_IO; }
    std::vector<std::string> lines;
    std::string l;
    while (std::getline(in, l)) lines.push_back(l);
    return read_potential_lines(lines, path, P, msg);
}

akmc_status read_potentials_text(const std::string& text, Potentials& P, std::string& msg)
{
    std::istringstream in(text);
    std::vector<std::string> lines;
    std::string l;
    while (std::getline(in, l)) lines.push_back(l);
    return read_potential_lines(lines, "potentials text", P, msg);
}

akmc_status read_potential_lines(const std::vector<std::string>& lines, const std::string& path,
                                 Potentials& P, std::string& msg)
{
    // family: the first family-specific keyword decides which reference Field reads it
    P.family = 0;
    for (const auto& l : lines) {
        auto w = split(lower(l));
        if (w.empty()) continue;
        if (w[0] == "many" || w[0] == "manybody") { P.family = AKMC_FAMILY_EAM; break; }
        if (w[0] == "twobody" || w[0] == "ewald") { P.family = AKMC_FAMILY_IONIC; break; }
        if (w[0] == "close") break;
    }
    if (P.family == 0) { msg = "no manybody, twobody or ewald block in " + path; return AKMC_ERR_PARSE; }
    P.verlet_shell = P.family == AKMC_FAMILY_EAM ? -0.5 : 1.0;

    size_t i = 0;
    auto next = [&](std::string& out) -> bool {
        if (i >= lines.size()) return false;
        out = lines[i++];
        return true;
    };
    bool closed = false;
    std::string line;
    while (next(line)) {
        auto w = split(lower(line));
        if (w.empty()) continue;
        const std::string& k = w[0];
        if (k == "cutoff") {
            if (w.size() < 2 || !to_double(w[1], P.cutoff)) { msg = "bad cutoff line"; return AKMC_ERR_PARSE; }
        } else if (k == "nbrlist") {
            P.use_nbrlist = true;
            if (w.size() < 2 || !to_double(w[1], P.verlet_shell)) { msg = "bad nbrlist line"; return AKMC_ERR_PARSE; }
        } else if (k == "noimage") {
            msg = "the noimage convention is not on this path";
            return AKMC_ERR_UNSUPPORTED;
        } else if (k == "species") {
            int n = 0;
            if (w.size() < 2 || !to_int(w[1], n) || n < 1 || n > kMaxSpecies) {
                msg = "bad species count";
                return AKMC_ERR_PARSE;
            }
            for (int s = 0; s < n; s++) {
                std::string sl;
                if (!next(sl)) { msg = "truncated species block"; return AKMC_ERR_PARSE; }
                auto sw = split(sl);
                SpeciesRec r;
                if (sw.size() < 3 || !to_double(sw[1], r.mass) || !to_double(sw[2], r.charge)) {
                    msg = "bad species line: " + sl;
                    return AKMC_ERR_PARSE;
                }
                r.name = sw[0];
                P.species.push_back(r);
            }
        } else if (P.family == AKMC_FAMILY_EAM && (k == "many" || k == "manybody")) {
            int n = 0;
            if (w.size() < 3 || !to_int(w[1], n) || n < 1) { msg = "bad manybody line"; return AKMC_ERR_PARSE; }
            for (int p = 0; p < n; p++) {
                std::string tl, pl;
                if (!next(tl) || !next(pl)) { msg = "truncated manybody block"; return AKMC_ERR_PARSE; }
                auto tw = split(lower(tl));
                if (tw.empty() || tw[0] == "close") { msg = "wrong number of many-body potentials"; return AKMC_ERR_PARSE; }
                if (tw[0] != "eam") { msg = "many-body form not on this path: " + tw[0]; return AKMC_ERR_UNSUPPORTED; }
                auto pw = split(pl);
                if (pw.size() < 3) { msg = "bad eam line: " + pl; return AKMC_ERR_PARSE; }
                std::string fmt = pw.size() > 3 ? pw[3] : "lammps";
                if (fmt != "lammps") { msg = "EAM format not on this path: " + fmt; return AKMC_ERR_UNSUPPORTED; }
                EamTable t;
                t.atA = pw[0];
                t.atB = pw[1];
                t.file = pw[2];
                akmc_status st = read_setfl(t.file, t, msg);
                if (st) return st;
                P.eam.push_back(std::move(t));
            }
        } else if (P.family == AKMC_FAMILY_IONIC && k == "twobody") {
            int n = 0;
            if (w.size() < 2 || !to_int(w[1], n) || n < 1) { msg = "bad twobody line"; return AKMC_ERR_PARSE; }
            P.cfact = kCtoev;
            for (int p = 0; p < n; p++) {
                std::string tl, pl;
                if (!next(tl)) { msg = "truncated twobody block"; return AKMC_ERR_PARSE; }
                auto tw = split(lower(tl));
                if (tw.empty() || tw[0] == "close") { msg = "wrong number of two-body potentials"; return AKMC_ERR_PARSE; }
                if (tw[0] != "buck") { msg = "two-body form not on this path: " + tw[0]; return AKMC_ERR_UNSUPPORTED; }
                if (!next(pl)) { msg = "truncated twobody block"; return AKMC_ERR_PARSE; }
                auto pw = split(pl);
                BuckRec b;
                if (pw.size() < 5 || !to_double(pw[2], b.A) || !to_double(pw[3], b.rho) ||
                    !to_double(pw[4], b.C)) {
                    msg = "bad buck line: " + pl;
                    return AKMC_ERR_PARSE;
                }
                b.a = pw[0];
                b.b = pw[1];
                P.buck.push_back(b);
            }
        } else if (P.family == AKMC_FAMILY_IONIC && k == "ewald") {
            if (w.size() >= 3 && w[1] == "precis") {
                P.do_ewald = 1;
                if (!to_double(w[2], P.precis)) { msg = "bad ewald precis"; return AKMC_ERR_PARSE; }
            } else if (w.size() >= 2 && w[1] == "none") {
                P.do_ewald = 0;
            } else if (w.size() >= 2 && w[1] == "damp") {
                msg = "damped shifted Coulomb is not on this path";
                return AKMC_ERR_UNSUPPORTED;
            }
        } else if (k == "close") {
            closed = true;
            break;
        } else {
            msg = "unrecognised key word used in potentials file " + k;
            return AKMC_ERR_PARSE;
        }
    }
    (void)closed;
    const int ns = (int)P.species.size();
    if (ns == 0) { msg = "no species block"; return AKMC_ERR_PARSE; }
    if (P.family == AKMC_FAMILY_EAM) {
        if (P.eam.empty()) { msg = "no EAM potential"; return AKMC_ERR_PARSE; }
        if (P.eam.size() > 127) { msg = "too many EAM potentials"; return AKMC_ERR_UNSUPPORTED; }
        const EamTable& t0 = P.eam[0];
        for (const EamTable& t : P.eam)
            if (t.n_r != t0.n_r || t.n_embed != t0.n_embed || t.step_r != t0.step_r ||
                t.step_embed != t0.step_embed || t.pot_cutoff != t0.pot_cutoff) {
                msg = "the EAM tables of one field must share their r and rho grids and cutoff";
                return AKMC_ERR_UNSUPPORTED;
            }
        // ManyBody::calculateEAMEnergyMesh (ManyBody.cpp:937-1000), default -1
        P.eam_mesh.assign((size_t)ns * ns, -1);
        for (size_t k = 0; k < P.eam.size(); k++)
            for (int a = 0; a < ns; a++)
                for (int b = 0; b < ns; b++)
                    if (P.species[a].name == P.eam[k].atA && P.species[b].name == P.eam[k].atB) {
                        P.eam_mesh[(size_t)b * ns + a] = (int)k;
                        P.eam_mesh[(size_t)a * ns + b] = (int)k;
                    }
    } else {
        if (P.buck.empty()) {
            // no short-range entries: all pairs carry a zero Buckingham
            BuckRec z;
            z.A = 0.0; z.rho = 1.0; z.C = 0.0;
            P.buck.push_back(z);
        }
        // TwoBody::calculateEnergyMesh (TwoBody.cpp:480-576): default 0, so an unlisted
        // species pair silently uses potential 0
        P.buck_mesh.assign((size_t)ns * ns, 0);
        for (int a = 0; a < ns; a++)
            for (int b = 0; b < ns; b++)
                for (size_t k = 0; k < P.buck.size(); k++)
                    if (P.species[a].name == P.buck[k].a && P.species[b].name == P.buck[k].b) {
                        P.buck_mesh[(size_t)b * ns + a] = (int)k;
                        P.buck_mesh[(size_t)a * ns + b] = (int)k;
                    }
    }
    return AKMC_OK;
}

// Field::setup eta (pair/Field.cpp:129-133), Ewald::setEwaldImage (Ewald.cpp:88-120) and
// Ewald::findGvector (Ewald.cpp:188-319).  k-vectors are kept as integer triples: for an
// orthorhombic cell k = 2 pi (nx/Lx, ny/Ly, nz/Lz), which is what the reference's
// x = nx*rcp[0] + ny*rcp[1] + nz*rcp[2] (times 2 pi) evaluates to.
akmc_status ewald_setup(double precis, double cutoff, const double lat[9], const double rcp[9],
                        EwaldSet& E, std::string& msg)
{
    const double eps = std::fmin(std::fabs(precis), 0.5);
    const double tol = std::sqrt(std::fabs(std::log(eps * cutoff)));
    E.eta = std::sqrt(std::fabs(std::log(eps * cutoff * tol))) / cutoff;
    const double eta = E.eta;
    double cel[10];
    dcell(lat, cel);
    const double volume = cel[9];
    const double tol1 = std::sqrt(-std::log(eps * cutoff * std::pow(2.0 * tol * eta, 2)));
    if (!std::isfinite(tol1)) { msg = "Ewald precision gives no k-space cutoff"; return AKMC_ERR_ARG; }
    for (int d = 0; d < 3; d++) E.gcell[d] = (int)std::rint(0.25 + cel[d] * eta * tol1 / kPi);
    double rc[10];
    dcell(rcp, rc);
    const double kc = std::fmin(std::fmin(E.gcell[0] * rc[6], E.gcell[1] * rc[7]), E.gcell[2] * rc[8]);
    const double kcsq = kc * kc;
    const double etasq = eta * eta, gsqfct = 1.0 / (4.0 * etasq);
    const double gfct0 = kCtoev * kPi / (etasq * volume);
    E.nx.clear(); E.ny.clear(); E.nz.clear(); E.g0.clear();
    for (int nx = 0; nx <= E.gcell[0]; nx++)
        for (int ny = -E.gcell[1]; ny <= E.gcell[1]; ny++)
            for (int nz = -E.gcell[2]; nz <= E.gcell[2]; nz++) {
                const double x = nx * rcp[0] + ny * rcp[1] + nz * rcp[2];
                const double y = nx * rcp[3] + ny * rcp[4] + nz * rcp[5];
                const double z = nx * rcp[6] + ny * rcp[7] + nz * rcp[8];
                const double gsq = x * x + y * y + z * z;
                if (gsq < kcsq && gsq > 1.0e-8) {
                    const double kx = x * kTwoPi, ky = y * kTwoPi, kz = z * kTwoPi;
                    const double xg = (kx * kx + ky * ky + kz * kz) * gsqfct;
                    const double gzz = std::exp(-xg) / xg;
                    E.nx.push_back(nx);
                    E.ny.push_back(ny);
                    E.nz.push_back(nz);
                    E.g0.push_back(kx < 1.0e-8 ? gzz * gfct0 : gzz * gfct0 * 2.0);
                }
            }
    return AKMC_OK;
}

}  // namespace akmc
