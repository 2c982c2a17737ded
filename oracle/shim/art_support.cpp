// Support code for the reference's ART saddle search (optim/ART.cpp, compiled unchanged):
// the three SaddleSearch members ART::findSaddlePoint calls, whose own source file
// (optim/SaddleSearch.cpp) needs MPI, and a stand-in for LAPACK's dstev_, which is absent
// here.  Used by both ART builds: on the reference's own Field (ref_art.cpp) and on the
// drop-in Field of this project (tests/cpp/art_dropin.cpp).  Test infrastructure only.
//
// Every atom is active (the reference's global region, regionStyle 1), and instead of a
// random displacement the search starts from a given one (art_support_set_seed): the atoms
// are moved by it and the initial Lanczos vector is its unit vector -- what
// SaddleSearch::makeGaussDisplacement (optim/SaddleSearch.cpp:423-490) does with the
// displacement it draws.  dstev_ (the lowest eigenpair of the Lanczos tridiagonal matrix,
// optim/ART.cpp:764-793) is a cyclic Jacobi eigensolver written for this harness.
#include <algorithm>
#include <cmath>
#include <fstream>
#include <string>
#include <vector>

#include "ART.h"
#include "art_support.h"

namespace {
const double* g_seed = nullptr;      // the starting displacement of the next search, [n][3]

void place_seed(Basis& bas, int vectorSize, double*& rVector)
{
    rVector = alloc_dvector(vectorSize, "ART::rVector", 0.0);
    double norm = 0.0;
    for (int i = 0; i < vectorSize; i++) norm += g_seed[i] * g_seed[i];
    norm = std::sqrt(norm);
    for (int i = 0; i < vectorSize; i++) rVector[i] = g_seed[i] / norm;
    bas.displaceAtoms(g_seed);
}
}  // namespace

SaddleSearch::SaddleSearch() {}
SaddleSearch::~SaddleSearch() {}

void SaddleSearch::constructActiveRegion(const MPIComms&, Basis& bas, const Species&, const JobControl&,
                                         double* centre, std::ofstream&)
{
    bas.numFrozenAtoms = 0;
    for (int i = 0; i < bas.numberOfAtoms; i++) bas.frozen[i] = 0;
    vectorSize = 3 * bas.numberOfAtoms;
    centre[0] = centre[1] = centre[2] = 0.0;
}

void SaddleSearch::makeGaussDisplacement(const MPIComms&, Basis& bas, double*, double, double, std::ofstream&)
{
    place_seed(bas, vectorSize, rVector);
}

void SaddleSearch::makeRandomDisplacement(const MPIComms&, Basis& bas, double, std::ofstream&)
{
    place_seed(bas, vectorSize, rVector);
}

// Eigenvalues (ascending, in d) and eigenvectors (columns of z, n x n, column-major as
// LAPACK returns them) of the symmetric tridiagonal matrix with diagonal d and sub-diagonal
// e: cyclic Jacobi rotations on the dense matrix until the off-diagonal mass is below
// 1e-30 of the total.  Only jobz = 'V' is supported; info = 0.
extern "C" int dstev_(char* jobz, int* n_in, double* d, double* e, double* z, int* ldz, double*, int* info)
{
    const int n = *n_in, ld = *ldz;
    *info = 0;
    if (*jobz != 'V' || n < 1 || ld < n) {
        *info = -1;
        return 0;
    }
    std::vector<double> A((size_t)n * n, 0.0), V((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++) {
        A[(size_t)i * n + i] = d[i];
        if (i + 1 < n) A[(size_t)i * n + i + 1] = A[(size_t)(i + 1) * n + i] = e[i];
        V[(size_t)i * n + i] = 1.0;
    }
    auto a = [&](int r, int c) -> double& { return A[(size_t)r * n + c]; };
    double total = 0.0;
    for (double x : A) total += x * x;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0;
        for (int p = 0; p < n; p++)
            for (int q = p + 1; q < n; q++) off += a(p, q) * a(p, q);
        if (off <= 1e-30 * total) break;
        for (int p = 0; p < n; p++) {
            for (int q = p + 1; q < n; q++) {
                if (a(p, q) == 0.0) continue;
                // rotation that zeroes a(p, q): tan(2 theta) = 2 a_pq / (a_qq - a_pp)
                const double theta = 0.5 * std::atan2(2.0 * a(p, q), a(q, q) - a(p, p));
                const double c = std::cos(theta), s = std::sin(theta);
                for (int k = 0; k < n; k++) {             // columns p, q: A <- A J
                    const double akp = a(k, p), akq = a(k, q);
                    a(k, p) = c * akp - s * akq;
                    a(k, q) = s * akp + c * akq;
                }
                for (int k = 0; k < n; k++) {             // rows p, q: A <- J^T A
                    const double apk = a(p, k), aqk = a(q, k);
                    a(p, k) = c * apk - s * aqk;
                    a(q, k) = s * apk + c * aqk;
                }
                for (int k = 0; k < n; k++) {             // eigenvectors: V <- V J
                    const double vkp = V[(size_t)k * n + p], vkq = V[(size_t)k * n + q];
                    V[(size_t)k * n + p] = c * vkp - s * vkq;
                    V[(size_t)k * n + q] = s * vkp + c * vkq;
                }
            }
        }
    }
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int x, int y) { return a(x, x) < a(y, y); });
    std::vector<double> ev(n);
    for (int i = 0; i < n; i++) ev[i] = a(order[i], order[i]);
    for (int i = 0; i < n; i++) {
        d[i] = ev[i];
        for (int k = 0; k < n; k++) z[(size_t)i * ld + k] = V[(size_t)k * n + order[i]];
    }
    return 0;
}

void art_support_set_seed(const double* seed) { g_seed = seed; }
