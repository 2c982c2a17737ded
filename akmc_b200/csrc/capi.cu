// C-ABI of the AKMC force path: field lifetime, batch planning and the force calls.
//
// akmc_field mirrors the reference's Field object (one per potential file): it owns the
// parsed potential, the device tables and Ewald k-set of its setup cell, a stream and
// pinned staging for the host-buffer call, and a cached batch of one system.
// akmc_batch is the device-resident plan for many independent systems: per-system cell
// grids, work-item windows and every scratch buffer, so that akmc_batch_forces
// allocates nothing and can be replayed or captured.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "host_internal.h"

using namespace akmc;

namespace {
thread_local std::string g_last_error;
}  // namespace

namespace akmc {
akmc_status fail(akmc_status code, const std::string& m)
{
    g_last_error = m;
    return code;
}
const char* const kKernelNames[K_COUNT] = {"cell_sort", "eam_density", "eam_force",
                                           "structure_factor", "ionic_force", "energy_reduce"};
}  // namespace akmc

namespace {

bool orthorhombic(const double* lat)
{
    return lat[1] == 0.0 && lat[2] == 0.0 && lat[3] == 0.0 && lat[5] == 0.0 && lat[6] == 0.0 &&
           lat[7] == 0.0 && lat[0] > 0.0 && lat[4] > 0.0 && lat[8] > 0.0;
}

// Field::setup image check: metal/Field.cpp:42-61, pair/Field.cpp:98-107.
akmc_status cutoff_check(const akmc_field* f, double min_dim)
{
    const Potentials& P = f->pot;
    if (P.cutoff < 1.0) return fail(AKMC_ERR_CUTOFF, "short range cutoff is too small");
    double radius = P.cutoff;
    if (P.family == AKMC_FAMILY_IONIC) radius = P.cutoff + P.verlet_shell;
    else if (P.use_nbrlist) radius = P.cutoff + P.verlet_shell;
    if (radius > min_dim / 2)
        return fail(AKMC_ERR_CUTOFF, "short range cutoff too large for simulation box: cutoff " +
                                         std::to_string(P.cutoff) + " minimum dimension " +
                                         std::to_string(min_dim));
    return AKMC_OK;
}

std::vector<float4> pack_rows(const EamTable& t)
{
    std::vector<float4> rows(2 * (size_t)t.n_r);
    for (int i = 0; i < t.n_r; i++) {
        const bool last = i + 1 >= t.n_r;
        auto d = [&](const std::vector<double>& v) {
            return last ? 0.0 : v[(size_t)i + 1] - v[(size_t)i];
        };
        rows[2 * (size_t)i] = make_float4((float)t.phi[i], (float)d(t.phi), (float)t.dphi[i],
                                          (float)d(t.dphi));
        rows[2 * (size_t)i + 1] = make_float4((float)t.drho[i], (float)d(t.drho), (float)t.rho[i],
                                              (float)d(t.rho));
    }
    return rows;
}

template <class T>
akmc_status upload(DevBuf<T>& b, const std::vector<T>& v)
{
    AKMC_CUDA(b.alloc(v.size()));
    if (!v.empty()) AKMC_CUDA(cudaMemcpy(b.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
    return AKMC_OK;
}

void free_host(akmc_field* f)
{
    if (f->h_pos) cudaFreeHost(f->h_pos);
    if (f->h_force) cudaFreeHost(f->h_force);
    if (f->h_energy) cudaFreeHost(f->h_energy);
    if (f->h_status) cudaFreeHost(f->h_status);
    if (f->h_label) cudaFreeHost(f->h_label);
    if (f->h_charge) cudaFreeHost(f->h_charge);
    f->h_pos = f->h_force = f->h_energy = f->h_charge = nullptr;
    f->h_status = f->h_label = nullptr;
}

// Cell grid and work-item window of one orthorhombic system: cells at least one cutoff
// wide (so the 27-cell stencil holds every neighbour), at most max_cells cells, and the
// per-pair minimum image in every dimension with fewer than 3 cells.  Returns the
// number of cells.
int plan_system(int n, const double* L, double rc, int max_cells, int atom_begin,
                int cell_begin, int item_base, int home_chunk, SysGeom& g)
{
    std::memset(&g, 0, sizeof(g));
    g.atom_begin = atom_begin;
    g.n_atoms = n;
    g.cell_begin = cell_begin;
    int nc[3];
    for (int d = 0; d < 3; d++) nc[d] = std::max(1, (int)std::floor(L[d] / rc));
    while ((long long)nc[0] * nc[1] * nc[2] > max_cells) {
        const int d = (nc[0] >= nc[1] && nc[0] >= nc[2]) ? 0 : (nc[1] >= nc[2] ? 1 : 2);
        nc[d]--;
    }
    int mi = 0;
    for (int d = 0; d < 3; d++) {
        g.nc[d] = nc[d];
        g.L[d] = L[d];
        g.invL[d] = 1.0 / L[d];
        g.cell_w_inv[d] = nc[d] / L[d];
        if (nc[d] < 3) mi |= 1 << d;
    }
    g.mi_mask = mi;
    const int ncell = nc[0] * nc[1] * nc[2];
    g.item_base = item_base;
    g.item_cap = ncell + (n + home_chunk - 1) / home_chunk;
    return ncell;
}

// erfc(x) exp(x^2) on [lo, hi] for the far-pair terms of the mixed ionic pass: the degree-
// kErfcxDeg Chebyshev interpolant (values at the Chebyshev points of the first kind, FP64,
// the function from std::erfc and std::exp), converted to monomials in t in [-1, 1] by the
// recurrence T_{k+1} = 2 t T_k - T_{k-1}.  Accepted (erfcx_on = 1) if its largest relative
// error on 4001 points of the range, evaluated as the kernel does from FP32 coefficients
// in FP64, is below 1e-9 plus the coefficients' FP32 rounding.
void fit_erfcx(double lo, double hi, IonicDev& p)
{
    constexpr int N = kErfcxDeg + 1;
    p.erfcx_on = 0;
    if (!(hi > lo) || !(lo > 0.0)) return;
    const double mid = 0.5 * (hi + lo), half = 0.5 * (hi - lo);
    auto fn = [](double x) { return std::erfc(x) * std::exp(x * x); };
    double c[N] = {0.0};
    for (int j = 0; j < N; j++) {
        const double th = kPi * (j + 0.5) / N;
        const double v = fn(mid + half * std::cos(th));
        for (int k = 0; k < N; k++) c[k] += 2.0 / N * v * std::cos(k * th);
    }
    c[0] *= 0.5;
    // monomial coefficients: sum_k c_k T_k(t) = sum_k m_k t^k
    double m[N] = {0.0}, Tm[N] = {0.0}, T0[N] = {0.0}, T1[N] = {0.0};
    T0[0] = 1.0;
    T1[1] = 1.0;
    for (int i = 0; i < N; i++) m[i] += c[0] * T0[i];
    for (int i = 0; i < N; i++) m[i] += c[1] * T1[i];
    for (int k = 2; k < N; k++) {
        for (int i = 0; i < N; i++) Tm[i] = -T0[i] + (i > 0 ? 2.0 * T1[i - 1] : 0.0);
        for (int i = 0; i < N; i++) m[i] += c[k] * Tm[i];
        for (int i = 0; i < N; i++) { T0[i] = T1[i]; T1[i] = Tm[i]; }
    }
    const float c0lo = (float)(m[0] - (double)(float)m[0]);
    double err = 0.0;
    for (int q = 0; q <= 4000; q++) {
        const double x = lo + (hi - lo) * q / 4000.0;
        const double t = (x - mid) / half;
        double v = (float)m[N - 1];
        for (int k = N - 2; k >= 1; k--) v = v * t + (float)m[k];
        v = (v * t + c0lo) + (float)m[0];
        err = std::max(err, std::fabs(v / fn(x) - 1.0));
    }
    if (!(err < 1.0e-9 + 2.0e-7)) return;
    for (int k = 0; k < N; k++) p.erfcx_c[k] = (float)m[k];
    p.erfcx_c0lo = c0lo;
    p.erfcx_t1 = (float)(1.0 / half);
    p.erfcx_t0 = (float)(-mid / half);
    p.erfcx_on = 1;
}

// Launch one kernel, bracketed by timing events when the batch is being profiled.
template <class Fn>
akmc_status timed(akmc_batch* b, int k, cudaStream_t s, Fn&& launch)
{
    cudaEvent_t a = nullptr, e = nullptr;
    if (b->timer.on) {
        a = b->timer.take();
        e = b->timer.take();
        AKMC_CUDA(cudaEventRecord(a, s));
    }
    AKMC_CUDA(launch());
    if (b->timer.on) {
        AKMC_CUDA(cudaEventRecord(e, s));
        b->timer.pending.push_back({k, a, e});
    }
    return AKMC_OK;
}

}  // namespace

akmc_status akmc::run_batch(akmc_batch* b, double* pos, double* force, double* energy, int* status,
                            cudaStream_t s, const int* active, cudaEvent_t wrapped)
{
    akmc_field* f = b->field;
    BatchDev v = b->view;
    v.active = active;
    const double rc2 = f->pot.cutoff * f->pot.cutoff;
    const int fam = f->pot.family;
    const int prec = f->precision;
    akmc_status st;
    // Work queues pay where systems are switched off or reuse their lists (few queued items
    // out of many planned); a call where every system scans its cells takes one CTA per
    // planned item.  The cell kernel fills this call's queues from zero.
    if (!(active || v.skin > 0.0)) {
        v.work = nullptr;
        v.chunks = nullptr;
    }
    if (v.work) AKMC_CUDA(cudaMemsetAsync(v.counters, 0, sizeof(int) * kCounters, s));
    // whole-cell ionic batches in mixed precision need no cell order (see the pair kernels)
    const bool whole = fam == AKMC_FAMILY_IONIC && v.whole_cell_n > 0 && prec != AKMC_PREC_FP64;
    if ((st = timed(b, K_CELL, s, [&] {
             return whole ? launch_wrap_whole_cell(v, pos, status, s)
                          : launch_cell_sort(v, pos, status, fam, b->max_cells, s);
         })))
        return st;
    if (wrapped) AKMC_CUDA(cudaEventRecord(wrapped, s));
    if (fam == AKMC_FAMILY_EAM) {
        if ((st = timed(b, K_EAM_DENSITY, s, [&] { return launch_eam_density(v, f->eam, rc2, status, prec, s); })) ||
            (st = timed(b, K_EAM_FORCE, s, [&] { return launch_eam_force(v, f->eam, rc2, force, status, prec, s); })) ||
            (energy && (st = timed(b, K_ENERGY, s, [&] { return launch_energy_reduce(v, fam, nullptr, energy, s); }))))
            return st;
    } else {
        if (f->ionic.nk > 0 &&
            (st = timed(b, K_STRUCTURE, s, [&] { return launch_structure_factor(v, f->ionic, prec, s); })))
            return st;
        // the whole-cell kernel sums each system's energies itself (its last CTA to finish)
        if ((st = timed(b, K_IONIC_FORCE, s, [&] {
                 return launch_ionic_force(v, f->ionic, rc2, force, whole ? energy : nullptr, status, prec, s);
             })) ||
            (energy && !whole &&
             (st = timed(b, K_ENERGY, s, [&] { return launch_energy_reduce(v, fam, &f->ionic, energy, s); }))))
            return st;
    }
    return AKMC_OK;
}

extern "C" {

const char* akmc_last_error(void) { return g_last_error.c_str(); }

const char* akmc_version(void) { return "akmc_b200 0.1 (sm_100a)"; }

akmc_status akmc_field_set_list_density(akmc_field* f, double rho)
{
    if (!f || !(rho >= 0.0)) return fail(AKMC_ERR_ARG, "bad list density");
    f->list_density = rho;
    if (f->single) {                   // the host path's batch is re-created with it
        akmc_batch_destroy(f->single);
        f->single = nullptr;
        f->single_n = -1;
    }
    return AKMC_OK;
}

int akmc_checks_enabled(void)
{
#ifdef AKMC_CHECKS
    return 1;
#else
    return 0;
#endif
}

akmc_status akmc_checks_read(int* hits, int* first, int clear)
{
#ifdef AKMC_CHECKS
    if (!hits || !first) return fail(AKMC_ERR_ARG, "null argument");
    int buf[2 * kCheckCodes];
    cudaError_t (*readers[3])(int*) = {checks_read_cells, checks_read_pair, checks_read_walkers};
    cudaError_t (*clears[3])() = {checks_clear_cells, checks_clear_pair, checks_clear_walkers};
    for (int f = 0; f < AKMC_CHECK_FILES; f++) {
        AKMC_CUDA(readers[f](buf));
        for (int c = 0; c < kCheckCodes; c++) {
            hits[f * kCheckCodes + c] = buf[c];
            first[f * kCheckCodes + c] = buf[kCheckCodes + c];
        }
        if (clear) AKMC_CUDA(clears[f]());
    }
    return AKMC_OK;
#else
    (void)hits;
    (void)first;
    (void)clear;
    return fail(AKMC_ERR_UNSUPPORTED, "this library was built without bounds checks (build --checks)");
#endif
}

akmc_status akmc_field_create(const char* path, akmc_field** out)
{
    if (!path || !out) return fail(AKMC_ERR_ARG, "null argument");
    *out = nullptr;
    auto f = std::make_unique<akmc_field>();
    std::string msg;
    akmc_status st = read_potentials(path, f->pot, msg);
    if (st) return fail(st, msg);
    *out = f.release();
    return AKMC_OK;
}

akmc_status akmc_field_create_from_text(const char* text, akmc_field** out)
{
    if (!text || !out) return fail(AKMC_ERR_ARG, "null argument");
    *out = nullptr;
    auto f = std::make_unique<akmc_field>();
    std::string msg;
    akmc_status st = read_potentials_text(text, f->pot, msg);
    if (st) return fail(st, msg);
    *out = f.release();
    return AKMC_OK;
}

akmc_status akmc_field_setup(akmc_field* f, const double lat[9], const double rcp_in[9],
                             int max_atoms)
{
    if (!f || !lat || max_atoms < 1) return fail(AKMC_ERR_ARG, "bad setup arguments");
    if (!orthorhombic(lat)) return fail(AKMC_ERR_UNSUPPORTED, "only orthorhombic cells are supported");
    std::memcpy(f->lat, lat, sizeof(double) * 9);
    if (rcp_in) std::memcpy(f->rcp, rcp_in, sizeof(double) * 9);
    else reciprocal_vectors(lat, f->rcp);
    const double min_dim = std::min(std::min(lat[0], lat[4]), lat[8]);
    akmc_status st = cutoff_check(f, min_dim);
    if (st) return st;

    AKMC_CUDA(cudaGetDevice(&f->device));
    AKMC_CUDA(configure_cell_kernels());
    AKMC_CUDA(configure_pair_kernels());
    const Potentials& P = f->pot;
    const int ns = (int)P.species.size();
    if (P.family == AKMC_FAMILY_EAM) {
        // every table, one after the other (they share one grid)
        const EamTable& t = P.eam[0];
        std::vector<float4> rows;
        std::vector<double> phi, dphi, rho, drho, F, dF;
        for (const EamTable& q : P.eam) {
            const std::vector<float4> r = pack_rows(q);
            rows.insert(rows.end(), r.begin(), r.end());
            phi.insert(phi.end(), q.phi.begin(), q.phi.end());
            dphi.insert(dphi.end(), q.dphi.begin(), q.dphi.end());
            rho.insert(rho.end(), q.rho.begin(), q.rho.end());
            drho.insert(drho.end(), q.drho.begin(), q.drho.end());
            F.insert(F.end(), q.F.begin(), q.F.end());
            dF.insert(dF.end(), q.dF.begin(), q.dF.end());
        }
        if ((st = upload(f->eam_rows, rows))) return st;
        if ((st = upload(f->eam_phi, phi)) || (st = upload(f->eam_dphi, dphi)) ||
            (st = upload(f->eam_rho, rho)) || (st = upload(f->eam_drho, drho)) ||
            (st = upload(f->eam_F, F)) || (st = upload(f->eam_dF, dF)))
            return st;
        EamDev& e = f->eam;
        std::memset(&e, 0, sizeof(e));
        e.ns = ns;
        e.ntab = (int)P.eam.size();
        for (int a = 0; a < ns; a++) {
            for (int b = 0; b < ns; b++) {
                e.mesh[a * ns + b] = (signed char)P.eam_mesh[(size_t)a * ns + b];
                e.pair_ok[a * ns + b] = P.eam_mesh[(size_t)a * ns + b] >= 0;
            }
            e.dens_ok[a] = P.eam_mesh[(size_t)a * ns + a] >= 0;
            e.embed_ok[a] = P.eam_mesh[(size_t)a * ns + a] >= 0;
        }
        e.rows = f->eam_rows.p;
        e.phi = f->eam_phi.p; e.dphi = f->eam_dphi.p;
        e.rho = f->eam_rho.p; e.drho = f->eam_drho.p;
        e.F = f->eam_F.p; e.dF = f->eam_dF.p;
        e.n_r = t.n_r; e.n_embed = t.n_embed;
        e.step_r = t.step_r; e.inv_step_r = 1.0 / t.step_r;
        e.step_embed = t.step_embed; e.inv_step_embed = 1.0 / t.step_embed;
        e.pot_cutoff = t.pot_cutoff;
    } else {
        IonicDev& p = f->ionic;
        std::memset(&p, 0, sizeof(p));
        p.ns = ns;
        for (int a = 0; a < ns; a++)
            for (int b = 0; b < ns; b++) {
                const BuckRec& r = P.buck[(size_t)P.buck_mesh[(size_t)a * ns + b]];
                p.buckA[a * ns + b] = r.A;
                p.buckInvRho[a * ns + b] = 1.0 / r.rho;
                p.buckC[a * ns + b] = r.C;
            }
        p.cfact = P.cfact;
        for (int k = 0; k < kMaxSpecies * kMaxSpecies; k++) {
            p.buckAf[k] = (float)p.buckA[k];
            p.buckInvRhof[k] = (float)p.buckInvRho[k];
            p.buckCf[k] = (float)p.buckC[k];
        }
        p.r_split2 = f->r_split * f->r_split;
        if (P.do_ewald == 1) {
            std::string msg;
            if ((st = ewald_setup(P.precis, P.cutoff, f->lat, f->rcp, f->ewald, msg))) return fail(st, msg);
            std::vector<int4> ki(f->ewald.nx.size());
            for (size_t k = 0; k < ki.size(); k++)
                ki[k] = make_int4(f->ewald.nx[k], f->ewald.ny[k], f->ewald.nz[k], 0);
            if ((st = upload(f->kint, ki)) || (st = upload(f->g0, f->ewald.g0))) return st;
            p.eta = f->ewald.eta;
            p.nk = (int)ki.size();
            p.kint = f->kint.p;
            std::vector<double4> kd(ki.size());
            std::vector<float4> kf(ki.size());
            for (size_t k = 0; k < ki.size(); k++) {
                kd[k] = make_double4(ki[k].x, ki[k].y, ki[k].z, f->ewald.g0[k]);
                kf[k] = make_float4((float)ki[k].x, (float)ki[k].y, (float)ki[k].z, (float)f->ewald.g0[k]);
            }
            if ((st = upload(f->kd, kd)) || (st = upload(f->kf, kf))) return st;
            p.kd = f->kd.p;
            p.kf = f->kf.p;
            // phase-table slots of every k-vector (see IonicDev)
            p.gx = f->ewald.gcell[0];
            p.gy = f->ewald.gcell[1];
            p.gz = f->ewald.gcell[2];
            p.ntab = (p.gx + 1) + (2 * p.gy + 1) + (2 * p.gz + 1);
            std::vector<int4> kt(ki.size());
            for (size_t k = 0; k < ki.size(); k++)
                kt[k] = make_int4(ki[k].x, (p.gx + 1) + ki[k].y + p.gy,
                                  (p.gx + 1) + (2 * p.gy + 1) + ki[k].z + p.gz, 0);
            if ((st = upload(f->kt, kt))) return st;
            p.kt = f->kt.p;
            std::vector<int4> grp;
            for (size_t k = 0; k < ki.size();) {
                size_t e = k + 1;
                while (e < ki.size() && e - k < (size_t)kSkGroup && ki[e].x == ki[k].x && ki[e].y == ki[k].y &&
                       ki[e].z == ki[e - 1].z + 1)
                    e++;
                grp.push_back(make_int4((int)k, (int)(e - k), kt[k].x | (kt[k].y << 16), kt[k].z));
                k = e;
            }
            if ((st = upload(f->kgrp, grp))) return st;
            p.kgrp = f->kgrp.p;
            p.ngrp = (int)grp.size();
            p.inv_eta = 1.0 / p.eta;
            fit_erfcx(p.eta * std::min(f->r_split, P.cutoff), p.eta * P.cutoff * (1.0 + 1.0e-5), p);
            p.etaf = (float)p.eta;
            p.eta3f = (float)(p.eta * p.eta * p.eta);
            p.inv_etaf = (float)(1.0 / p.eta);
            p.g0 = f->g0.p;
        } else {
            // `ewald none`: no Coulomb terms at all
            p.eta = 0.0;
            p.cfact = 0.0;
            p.nk = 0;
        }
    }
    // host-buffer path resources
    free_host(f);
    f->max_atoms = max_atoms;
    if (!f->stream) AKMC_CUDA(cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking));
    AKMC_CUDA(cudaMallocHost(&f->h_pos, sizeof(double) * 3 * (size_t)max_atoms));
    AKMC_CUDA(cudaMallocHost(&f->h_force, sizeof(double) * 3 * (size_t)max_atoms));
    AKMC_CUDA(cudaMallocHost(&f->h_energy, sizeof(double) * 5));
    AKMC_CUDA(cudaMallocHost(&f->h_status, sizeof(int)));
    AKMC_CUDA(cudaMallocHost(&f->h_label, sizeof(int) * (size_t)max_atoms));
    AKMC_CUDA(cudaMallocHost(&f->h_charge, sizeof(double) * (size_t)max_atoms));
    AKMC_CUDA(f->d_pos.alloc(3 * (size_t)max_atoms));
    AKMC_CUDA(f->d_force.alloc(3 * (size_t)max_atoms));
    AKMC_CUDA(f->d_energy.alloc(5));
    AKMC_CUDA(f->d_status.alloc(1));
    if (f->single) { akmc_batch_destroy(f->single); f->single = nullptr; f->single_n = -1; }
    f->ready = true;
    return AKMC_OK;
}

akmc_status akmc_field_destroy(akmc_field* f)
{
    if (!f) return AKMC_OK;
    if (f->single) akmc_batch_destroy(f->single);
    free_host(f);
    if (f->stream) cudaStreamDestroy(f->stream);
    delete f;
    return AKMC_OK;
}

akmc_status akmc_field_set_precision(akmc_field* f, int mode)
{
    if (!f || (mode != AKMC_PREC_MIXED && mode != AKMC_PREC_FP64)) return fail(AKMC_ERR_ARG, "bad precision mode");
    f->precision = mode;
    return AKMC_OK;
}

int akmc_field_family(const akmc_field* f) { return f ? f->pot.family : 0; }

int akmc_field_num_species(const akmc_field* f) { return f ? (int)f->pot.species.size() : 0; }

akmc_status akmc_field_species(const akmc_field* f, int i, char* name, double* mass, double* charge)
{
    if (!f || i < 0 || i >= (int)f->pot.species.size()) return fail(AKMC_ERR_ARG, "bad species index");
    const SpeciesRec& s = f->pot.species[(size_t)i];
    if (name) {
        std::strncpy(name, s.name.c_str(), 15);
        name[15] = 0;
    }
    if (mass) *mass = s.mass;
    if (charge) *charge = s.charge;
    return AKMC_OK;
}

double akmc_field_cutoff(const akmc_field* f) { return f ? f->pot.cutoff : 0.0; }

akmc_status akmc_field_ewald(const akmc_field* f, double* eta, int* nk, int gcell[3])
{
    if (!f || f->pot.family != AKMC_FAMILY_IONIC) return fail(AKMC_ERR_ARG, "not an ionic field");
    if (!f->ready) return fail(AKMC_ERR_STATE, "field not set up");
    if (eta) *eta = f->ewald.eta;
    if (nk) *nk = f->ionic.nk;
    if (gcell) for (int d = 0; d < 3; d++) gcell[d] = f->ewald.gcell[d];
    return AKMC_OK;
}

akmc_status akmc_batch_create(akmc_field* f, int nsys, const int* natoms, const double* box,
                              const int* label, const double* charge, akmc_batch** out)
{
    return akmc_batch_create_skin(f, nsys, natoms, box, label, charge, 0.0, out);
}

akmc_status akmc_batch_create_skin(akmc_field* f, int nsys, const int* natoms, const double* box,
                                   const int* label, const double* charge, double skin,
                                   akmc_batch** out)
{
    if (!f || !out || nsys < 1 || !natoms || !box || !label) return fail(AKMC_ERR_ARG, "bad batch arguments");
    if (!f->ready) return fail(AKMC_ERR_STATE, "akmc_field_setup must come first");
    if (!(skin >= 0.0)) return fail(AKMC_ERR_ARG, "skin must be >= 0");
    *out = nullptr;
    const Potentials& P = f->pot;
    if (P.family != AKMC_FAMILY_EAM) skin = 0.0;           // list reuse is an EAM-path feature
    const double rc = P.cutoff;
    const double rc_list = rc + skin;                       // cells and lists cover cutoff + skin
    const int ns = (int)P.species.size();
    auto b = std::make_unique<akmc_batch>();
    b->field = f;
    b->nsys = nsys;
    b->natoms.assign(natoms, natoms + nsys);
    b->box.assign(box, box + 3 * (size_t)nsys);
    std::vector<SysGeom> geo((size_t)nsys);
    int atom = 0, cell = 0, item = 0, max_n = 0, max_cells = 0;
    // Work items are planned for the smallest home chunk (the largest item count); the
    // chunk actually used is set below and can be changed by the autotuner.
    const int home_chunk = kMinHomeChunk;
    for (int s = 0; s < nsys; s++) {
        const int n = natoms[s];
        if (n < 1) return fail(AKMC_ERR_ARG, "every system needs at least one atom");
        const double* L = box + 3 * (size_t)s;
        if (!(L[0] > 0 && L[1] > 0 && L[2] > 0)) return fail(AKMC_ERR_ARG, "box lengths must be positive");
        if (P.family == AKMC_FAMILY_IONIC &&
            (L[0] != f->lat[0] || L[1] != f->lat[4] || L[2] != f->lat[8]))
            return fail(AKMC_ERR_ARG, "ionic batches share the setup cell (one Ewald k-set)");
        akmc_status st = cutoff_check(f, std::min(std::min(L[0], L[1]), L[2]));
        if (st) return st;
        if (skin > 0.0 && rc_list > 0.5 * std::min(std::min(L[0], L[1]), L[2]))
            return fail(AKMC_ERR_CUTOFF, "cutoff + skin exceeds half the smallest box length");
        SysGeom& g = geo[(size_t)s];
        const int ncell = plan_system(n, L, rc_list, kMaxCellsPerSystem, atom, cell, item, home_chunk, g);
        b->ncell.push_back(ncell);
        atom += n;
        cell += ncell;
        item += g.item_cap;
        max_n = std::max(max_n, n);
        max_cells = std::max(max_cells, ncell);
    }
    for (int i = 0; i < atom; i++)
        if (label[i] < 0 || label[i] >= ns) return fail(AKMC_ERR_ARG, "species label out of range");
    b->n_total = atom;
    b->total_cells = cell;
    b->total_items = item;
    b->max_cells = max_cells;
    AKMC_CUDA(b->geom.alloc((size_t)nsys));
    AKMC_CUDA(cudaMemcpy(b->geom.p, geo.data(), sizeof(SysGeom) * nsys, cudaMemcpyHostToDevice));
    // every cell of every system starts out empty at the system's first atom: the length of
    // a system's last cell is read against the next system's first cell, which must hold
    // that system's first atom even before the cell kernel has sorted it (a system that is
    // skipped, or that takes another system's order)
    {
        std::vector<int> cs0((size_t)cell + 1, atom);
        for (int s = 0; s < nsys; s++)
            for (int c = 0; c < b->ncell[(size_t)s]; c++) cs0[(size_t)geo[(size_t)s].cell_begin + c] = geo[(size_t)s].atom_begin;
        AKMC_CUDA(b->cell_start.alloc((size_t)cell + 1));
        AKMC_CUDA(cudaMemcpy(b->cell_start.p, cs0.data(), sizeof(int) * ((size_t)cell + 1), cudaMemcpyHostToDevice));
    }
    AKMC_CUDA(b->perm.alloc((size_t)atom));
    AKMC_CUDA(b->keys.alloc((size_t)atom));
    AKMC_CUDA(b->slots.alloc((size_t)atom));
    AKMC_CUDA(b->order.alloc((size_t)atom));
    AKMC_CUDA(b->slabel.alloc((size_t)atom));
    AKMC_CUDA(b->spos.alloc((size_t)atom));
    AKMC_CUDA(b->eatom.alloc((size_t)atom));
    AKMC_CUDA(b->items.alloc((size_t)item));
    AKMC_CUDA(b->n_items.alloc((size_t)nsys));
    AKMC_CUDA(b->label.alloc((size_t)atom));
    AKMC_CUDA(cudaMemcpy(b->label.p, label, sizeof(int) * atom, cudaMemcpyHostToDevice));
    AKMC_CUDA(b->charge.alloc((size_t)atom));
    std::vector<double> q((size_t)atom, 0.0);
    for (int i = 0; i < atom; i++)
        q[(size_t)i] = charge ? charge[i] : P.species[(size_t)label[i]].charge;
    AKMC_CUDA(cudaMemcpy(b->charge.p, q.data(), sizeof(double) * atom, cudaMemcpyHostToDevice));
    if (P.family == AKMC_FAMILY_EAM) AKMC_CUDA(b->sextra.alloc((size_t)atom));
    // EAM neighbour list of the force pass: capacity from the densest system, 1.5 x its
    // mean neighbour count inside the cutoff plus 16; indices are 16-bit offsets inside a
    // system, so every system must hold < 65536 atoms (otherwise the force pass rescans).
    int nbr_cap = 0;
    if (P.family == AKMC_FAMILY_EAM && max_n < 65536) {
        double dens = f->list_density;     // the caller's floor (clustered atoms), else 0
        for (int s = 0; s < nsys; s++) {
            const double* L = box + 3 * (size_t)s;
            dens = std::max(dens, natoms[s] / (L[0] * L[1] * L[2]));
        }
        const double mean = dens * 4.0 / 3.0 * kPi * rc_list * rc_list * rc_list;
        nbr_cap = ((int)std::ceil(1.5 * mean + 16.0) + 7) / 8 * 8;
        nbr_cap = std::min(nbr_cap, max_n);
        AKMC_CUDA(b->nbr.alloc((size_t)nbr_cap * atom));
        AKMC_CUDA(b->nbr_count.alloc((size_t)atom));
        AKMC_CUDA(b->frec.alloc((size_t)atom));
    }
    int sk_chunks = 1, ktiles = 1;
    const int nk = f->ionic.nk;
    if (P.family == AKMC_FAMILY_IONIC && nk > 0) {
        sk_chunks = (max_n + kSkAtomChunk - 1) / kSkAtomChunk;
        ktiles = (nk + kSkThreads - 1) / kSkThreads;
        AKMC_CUDA(b->skpart.alloc((size_t)nsys * sk_chunks * nk));
        AKMC_CUDA(b->sk.alloc((size_t)nsys * nk));
        AKMC_CUDA(b->skf.alloc((size_t)nsys * nk));
        AKMC_CUDA(b->sk_counter.alloc((size_t)nsys * ktiles));
        AKMC_CUDA(cudaMemset(b->sk_counter.p, 0, sizeof(int) * (size_t)nsys * ktiles));
        AKMC_CUDA(cudaMemset(b->sk.p, 0, sizeof(double2) * (size_t)nsys * nk));
    }
    BatchDev& v = b->view;
    v.nsys = nsys;
    v.n_total = atom;
    v.total_cells = cell;
    v.total_items = item;
    v.geom = b->geom.p;
    v.cell_start = b->cell_start.p;
    v.perm = b->perm.p;
    v.keys = b->keys.p;
    v.slots = b->slots.p;
    v.order = b->order.p;
    v.spos = b->spos.p;
    v.sextra = b->sextra.p;
    v.eatom = b->eatom.p;
    v.items = b->items.p;
    v.n_items = b->n_items.p;
    v.label = b->label.p;
    v.charge = b->charge.p;
    v.slabel = b->slabel.p;
    v.skpart = b->skpart.p;
    v.sk = b->sk.p;
    v.sk_counter = b->sk_counter.p;
    v.skf = b->skf.p;
    v.home_chunk = home_chunk;
    v.nbr = b->nbr.p;
    v.nbr_count = b->nbr_count.p;
    v.frec = b->frec.p;
    v.nbr_cap = nbr_cap;
    v.sk_chunks = sk_chunks;
    v.stage_cap = std::min(kStageCap, ((max_n + 31) / 32) * 32);
    v.whole_cell_n = 0;
    if (P.family == AKMC_FAMILY_IONIC && max_n <= kWholeCellMaxAtoms) {
        bool whole = true;
        for (int s2 = 0; s2 < nsys; s2++) whole = whole && geo[(size_t)s2].mi_mask == 7;
        if (whole) {
            v.whole_cell_n = max_n;
            AKMC_CUDA(b->wc_counter.alloc((size_t)nsys));
            AKMC_CUDA(cudaMemset(b->wc_counter.p, 0, sizeof(int) * nsys));
            v.wc_counter = b->wc_counter.p;
        }
    }
    // work queues: items up to the home chunk 8 plan, atom chunks of every system
    int work_cap = 0, chunk_cap = 0;
    for (int s2 = 0; s2 < nsys; s2++) {
        work_cap += b->ncell[(size_t)s2] + (natoms[s2] + 7) / 8;
        chunk_cap += (natoms[s2] + kChunkAtoms - 1) / kChunkAtoms;
    }
    AKMC_CUDA(b->work.alloc((size_t)work_cap));
    AKMC_CUDA(b->chunks.alloc((size_t)chunk_cap));
    AKMC_CUDA(b->counters.alloc((size_t)kCounters));
    AKMC_CUDA(cudaMemset(b->counters.p, 0, sizeof(int) * kCounters));
    v.work = b->work.p;
    v.chunks = b->chunks.p;
    v.counters = b->counters.p;
    v.ticket = nullptr;
    v.chunk_cap = chunk_cap;
    AKMC_CUDA(b->list_mode.alloc((size_t)nsys));
    AKMC_CUDA(b->list_ok.alloc((size_t)nsys));
    AKMC_CUDA(cudaMemset(b->list_ok.p, 0, sizeof(int) * nsys));
    if (skin > 0.0) AKMC_CUDA(b->ref_pos.alloc(3 * (size_t)atom));
    v.skin = skin;
    v.ref_pos = b->ref_pos.p;
    v.list_mode = b->list_mode.p;
    v.list_ok = b->list_ok.p;
    b->geo = geo;
    // default home chunk before any tuning: small batches get small items so that a few
    // thousand atoms still spread over every SM; large batches take 32
    const int hc0 = atom >= 64 * 1024 ? 32 : (atom >= 32 * 1024 ? 16 : 8);
    akmc_status st = akmc_batch_set_home_chunk(b.get(), hc0);
    if (st) return st;
    *out = b.release();
    return AKMC_OK;
}

namespace {

// The work-item plan of every system for its own home chunk (per_system[s]; 8, 16 or 32).
akmc_status plan_items(akmc_batch* b, const int* per_system, int uniform)
{
    int item = 0;
    for (int s = 0; s < b->nsys; s++) {
        const int hc = per_system ? per_system[s] : uniform;
        if (hc != 8 && hc != 16 && hc != 32) return fail(AKMC_ERR_ARG, "home chunk must be 8, 16 or 32");
        SysGeom& g = b->geo[(size_t)s];
        g.home_chunk = hc;
        g.item_base = item;
        g.item_cap = b->ncell[(size_t)s] + (g.n_atoms + hc - 1) / hc;
        item += g.item_cap;
    }
    // kernels of an earlier call may still read the plan: finish them first
    AKMC_CUDA(cudaDeviceSynchronize());
    AKMC_CUDA(cudaMemcpy(b->geom.p, b->geo.data(), sizeof(SysGeom) * b->nsys, cudaMemcpyHostToDevice));
    b->total_items = item;
    b->view.total_items = item;
    b->view.home_chunk = per_system ? 0 : uniform;
    return AKMC_OK;
}

}  // namespace

akmc_status akmc_batch_set_home_chunk(akmc_batch* b, int hc)
{
    if (!b || (hc != 8 && hc != 16 && hc != 32)) return fail(AKMC_ERR_ARG, "home chunk must be 8, 16 or 32");
    return plan_items(b, nullptr, hc);
}

akmc_status akmc_batch_set_system_chunks(akmc_batch* b, const int* chunks)
{
    if (!b || !chunks) return fail(AKMC_ERR_ARG, "null argument");
    return plan_items(b, chunks, 0);
}

int akmc_batch_total_items(const akmc_batch* b) { return b ? b->total_items : 0; }

int akmc_batch_home_chunk(const akmc_batch* b) { return b ? b->view.home_chunk : 0; }

akmc_status akmc_batch_autotune(akmc_batch* b, double* pos, double* force, double* energy,
                                int* status, void* stream, int* chosen)
{
    if (!b || !pos || !force || !energy || !status) return fail(AKMC_ERR_ARG, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    const int cand[3] = {8, 16, 32};
    float best = 1e30f;
    int best_hc = b->view.home_chunk;
    cudaEvent_t e0, e1;
    AKMC_CUDA(cudaEventCreate(&e0));
    AKMC_CUDA(cudaEventCreate(&e1));
    const bool was_on = b->timer.on;
    b->timer.on = false;
    akmc_status st = AKMC_OK;
    for (int c = 0; c < 3 && !st; c++) {
        if ((st = akmc_batch_set_home_chunk(b, cand[c]))) break;
        // with a skin, every timed call rebuilds its lists: the work-item size matters only there
        auto fresh = [&]() { if (b->view.skin > 0.0) cudaMemsetAsync(b->list_ok.p, 0, sizeof(int) * b->nsys, s); };
        fresh();
        if ((st = run_batch(b, pos, force, energy, status, s))) break;      // warm-up
        cudaEventRecord(e0, s);
        for (int r = 0; r < 3 && !st; r++) {
            fresh();
            st = run_batch(b, pos, force, energy, status, s);
        }
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) { best = ms; best_hc = cand[c]; }
    }
    b->timer.on = was_on;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    if ((st = akmc_batch_set_home_chunk(b, best_hc))) return st;
    if (chosen) *chosen = best_hc;
    return AKMC_OK;
}


akmc_status akmc_batch_autotune_classes(akmc_batch* b, double* pos, double* force, double* energy, int* status,
                                        void* stream, int* n_classes, int* class_cells, int* class_chunk,
                                        float* class_ms, int max_classes)
{
    if (!b || !pos || !force || !energy || !status || !n_classes) return fail(AKMC_ERR_ARG, "null argument");
    // 1. the best uniform chunk, the starting point
    int hc0 = 0;
    akmc_status st = akmc_batch_autotune(b, pos, force, energy, status, stream, &hc0);
    if (st) return st;
    // 2. size classes: systems with the same cell grid do the same work per item
    std::vector<int> key((size_t)b->nsys), classes;
    for (int s = 0; s < b->nsys; s++) {
        key[(size_t)s] = b->ncell[(size_t)s];
        if (std::find(classes.begin(), classes.end(), key[(size_t)s]) == classes.end()) classes.push_back(key[(size_t)s]);
    }
    std::sort(classes.begin(), classes.end());
    std::vector<int> chunk((size_t)b->nsys, hc0);
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t e0, e1;
    AKMC_CUDA(cudaEventCreate(&e0));
    AKMC_CUDA(cudaEventCreate(&e1));
    const bool was_on = b->timer.on;
    b->timer.on = false;
    auto fresh = [&]() { if (b->view.skin > 0.0) cudaMemsetAsync(b->list_ok.p, 0, sizeof(int) * b->nsys, s); };
    auto time_plan = [&](float* ms) -> akmc_status {
        akmc_status q;
        if ((q = akmc_batch_set_system_chunks(b, chunk.data()))) return q;
        fresh();
        if ((q = run_batch(b, pos, force, energy, status, s))) return q;     // warm-up
        cudaEventRecord(e0, s);
        for (int r = 0; r < 3; r++) {
            fresh();
            if ((q = run_batch(b, pos, force, energy, status, s))) return q;
        }
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(ms, e0, e1);
        return AKMC_OK;
    };
    // 3. one pass of coordinate descent: each class tries 8, 16 and 32 with the others fixed
    std::vector<float> best_ms(classes.size(), 0.f);
    for (size_t c = 0; c < classes.size() && !st; c++) {
        const int cand[3] = {8, 16, 32};
        float best = 1e30f;
        int best_hc = hc0;
        for (int k = 0; k < 3 && !st; k++) {
            for (int q = 0; q < b->nsys; q++)
                if (key[(size_t)q] == classes[c]) chunk[(size_t)q] = cand[k];
            float ms = 0.f;
            st = time_plan(&ms);
            if (!st && ms < best) { best = ms; best_hc = cand[k]; }
        }
        for (int q = 0; q < b->nsys; q++)
            if (key[(size_t)q] == classes[c]) chunk[(size_t)q] = best_hc;
        best_ms[c] = best;
    }
    b->timer.on = was_on;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    if ((st = akmc_batch_set_system_chunks(b, chunk.data()))) return st;
    *n_classes = (int)classes.size();
    for (size_t c = 0; c < classes.size() && (int)c < max_classes; c++) {
        if (class_cells) class_cells[c] = classes[c];
        if (class_chunk)
            for (int q = 0; q < b->nsys; q++)
                if (key[(size_t)q] == classes[c]) { class_chunk[c] = chunk[(size_t)q]; break; }
        if (class_ms) class_ms[c] = best_ms[c] / 3.0f;
    }
    return AKMC_OK;
}

akmc_status akmc_batch_destroy(akmc_batch* b)
{
    if (b) {
        if (b->side) cudaStreamDestroy(b->side);
        if (b->ev_wrapped) cudaEventDestroy(b->ev_wrapped);
        if (b->ev_side) cudaEventDestroy(b->ev_side);
    }
    delete b;
    return AKMC_OK;
}

int akmc_batch_launches(const akmc_batch* b)
{
    if (!b) return 0;
    if (b->field->pot.family != AKMC_FAMILY_IONIC) return 4;
    // ionic: cell kernel (or the whole-cell wrap), structure factors when there are k-vectors,
    // the pair pass, and the energy reduction unless the whole-cell pass sums the energies
    const bool whole = b->view.whole_cell_n > 0 && b->field->precision != AKMC_PREC_FP64;
    return 2 + (b->field->ionic.nk > 0 ? 1 : 0) + (whole ? 0 : 1);
}

akmc_status akmc_batch_profile(akmc_batch* b, int enable)
{
    if (!b) return fail(AKMC_ERR_ARG, "null batch");
    b->timer.drain();
    b->timer.on = enable != 0;
    return AKMC_OK;
}

int akmc_batch_kernel_times(akmc_batch* b, double* ms, int* launches, const char** names, int max)
{
    if (!b) return 0;
    b->timer.drain();
    const int n = std::min<int>(max, K_COUNT);
    for (int k = 0; k < n; k++) {
        if (ms) ms[k] = b->timer.ms[k];
        if (launches) launches[k] = b->timer.count[k];
        if (names) names[k] = kKernelNames[k];
        b->timer.ms[k] = 0.0;
        b->timer.count[k] = 0;
    }
    return n;
}

akmc_status akmc_batch_forces_host(akmc_batch* b, double* pos, double* force, double* energy,
                                   int* status, void* stream)
{
    if (!b || !pos || !force || !energy || !status) return fail(AKMC_ERR_ARG, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    const size_t n3 = 3 * (size_t)b->n_total;
    if (!b->h_pos_dev.p) {
        AKMC_CUDA(b->h_pos_dev.alloc(n3));
        AKMC_CUDA(b->h_force_dev.alloc(n3));
        AKMC_CUDA(b->h_energy_dev.alloc(5 * (size_t)b->nsys));
        AKMC_CUDA(b->h_status_dev.alloc((size_t)b->nsys));
    }
    if (!b->side) {
        AKMC_CUDA(cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking));
        AKMC_CUDA(cudaEventCreateWithFlags(&b->ev_wrapped, cudaEventDisableTiming));
        AKMC_CUDA(cudaEventCreateWithFlags(&b->ev_side, cudaEventDisableTiming));
    }
    AKMC_CUDA(cudaMemcpyAsync(b->h_pos_dev.p, pos, sizeof(double) * n3, cudaMemcpyHostToDevice, s));
    akmc_status st = run_batch(b, b->h_pos_dev.p, b->h_force_dev.p, b->h_energy_dev.p, b->h_status_dev.p, s,
                               nullptr, b->ev_wrapped);
    if (st) return st;
    // the wrapped positions are final after the first kernel: read back on the side stream
    // while the force passes run; the call's stream waits for it before returning
    AKMC_CUDA(cudaStreamWaitEvent(b->side, b->ev_wrapped, 0));
    AKMC_CUDA(cudaMemcpyAsync(pos, b->h_pos_dev.p, sizeof(double) * n3, cudaMemcpyDeviceToHost, b->side));
    AKMC_CUDA(cudaEventRecord(b->ev_side, b->side));
    AKMC_CUDA(cudaMemcpyAsync(force, b->h_force_dev.p, sizeof(double) * n3, cudaMemcpyDeviceToHost, s));
    AKMC_CUDA(cudaMemcpyAsync(energy, b->h_energy_dev.p, sizeof(double) * 5 * b->nsys, cudaMemcpyDeviceToHost, s));
    AKMC_CUDA(cudaMemcpyAsync(status, b->h_status_dev.p, sizeof(int) * b->nsys, cudaMemcpyDeviceToHost, s));
    AKMC_CUDA(cudaStreamWaitEvent(s, b->ev_side, 0));
    AKMC_CUDA(cudaStreamSynchronize(s));
    return AKMC_OK;
}

akmc_status akmc_batch_forces(akmc_batch* b, double* pos, double* force, double* energy,
                              int* status, void* stream)
{
    if (!b || !pos || !force || !energy || !status) return fail(AKMC_ERR_ARG, "null argument");
    return run_batch(b, pos, force, energy, status, (cudaStream_t)stream);
}

akmc_status akmc_batch_list_modes(akmc_batch* b, int* modes)
{
    if (!b || !modes) return fail(AKMC_ERR_ARG, "null argument");
    AKMC_CUDA(cudaDeviceSynchronize());
    AKMC_CUDA(cudaMemcpy(modes, b->list_mode.p, sizeof(int) * b->nsys, cudaMemcpyDeviceToHost));
    return AKMC_OK;
}

akmc_status akmc_batch_neighbours(akmc_batch* b, int* counts, int* nbrs, int max_per_atom)
{
    if (!b || !counts || !nbrs || max_per_atom < 1) return fail(AKMC_ERR_ARG, "bad neighbour arguments");
    if (!b->nbr.p) return fail(AKMC_ERR_STATE, "this batch keeps no neighbour list (EAM batches of < 65536-atom systems do)");
    const int n = b->n_total, cap = b->view.nbr_cap;
    std::vector<unsigned short> list((size_t)cap * n);
    std::vector<int> cnt((size_t)n), perm((size_t)n);
    AKMC_CUDA(cudaDeviceSynchronize());
    AKMC_CUDA(cudaMemcpy(list.data(), b->nbr.p, sizeof(unsigned short) * list.size(), cudaMemcpyDeviceToHost));
    AKMC_CUDA(cudaMemcpy(cnt.data(), b->nbr_count.p, sizeof(int) * n, cudaMemcpyDeviceToHost));
    AKMC_CUDA(cudaMemcpy(perm.data(), b->perm.p, sizeof(int) * n, cudaMemcpyDeviceToHost));
    std::vector<int> begin((size_t)b->nsys + 1, 0);
    for (int s = 0; s < b->nsys; s++) begin[(size_t)s + 1] = begin[(size_t)s] + b->natoms[(size_t)s];
    akmc_status st = AKMC_OK;
    int sys = 0;
    for (int i = 0; i < n; i++) {
        while (i >= begin[(size_t)sys + 1]) sys++;
        const int o = perm[(size_t)i];
        int* row = nbrs + (size_t)o * max_per_atom;
        const int c = cnt[(size_t)i];
        if (c > max_per_atom) st = AKMC_ERR_CAPACITY;
        const int m = std::min(c, max_per_atom);
        for (int k = 0; k < m; k++) row[k] = perm[(size_t)(begin[(size_t)sys] + list[(size_t)k * n + i])];
        std::sort(row, row + m);
        for (int k = m; k < max_per_atom; k++) row[k] = -1;
        counts[o] = c;
    }
    if (st) return fail(st, "a neighbour row exceeds max_per_atom");
    return AKMC_OK;
}

akmc_status akmc_forces(akmc_field* f, int n, double* px, double* py, double* pz,
                        const int* label, const double* charge, double* fx, double* fy,
                        double* fz, double stress[6], akmc_energy* out)
{
    if (!f || !px || !py || !pz || !label || !fx || !fy || !fz) return fail(AKMC_ERR_ARG, "null argument");
    if (!f->ready) return fail(AKMC_ERR_STATE, "akmc_field_setup must come first");
    if (n < 1 || n > f->max_atoms) return fail(AKMC_ERR_CAPACITY, "atom count outside 1..max_atoms");
    const int ns = (int)f->pot.species.size();
    for (int i = 0; i < n; i++) {
        if (label[i] < 0 || label[i] >= ns) return fail(AKMC_ERR_ARG, "species label out of range");
        f->h_label[i] = label[i];
        f->h_charge[i] = charge ? charge[i] : f->pot.species[(size_t)label[i]].charge;
    }
    AKMC_CUDA(cudaSetDevice(f->device));
    if (!f->single || f->single_n != n) {
        if (f->single) akmc_batch_destroy(f->single);
        f->single = nullptr;
        const double box[3] = {f->lat[0], f->lat[4], f->lat[8]};
        akmc_status st = akmc_batch_create(f, 1, &n, box, f->h_label, f->h_charge, &f->single);
        if (st) return st;
        f->single_n = n;
    } else {
        AKMC_CUDA(cudaMemcpyAsync(f->single->label.p, f->h_label, sizeof(int) * n,
                                  cudaMemcpyHostToDevice, f->stream));
        AKMC_CUDA(cudaMemcpyAsync(f->single->charge.p, f->h_charge, sizeof(double) * n,
                                  cudaMemcpyHostToDevice, f->stream));
    }
    for (int i = 0; i < n; i++) {
        f->h_pos[3 * i + 0] = px[i];
        f->h_pos[3 * i + 1] = py[i];
        f->h_pos[3 * i + 2] = pz[i];
    }
    const size_t bytes = sizeof(double) * 3 * (size_t)n;
    AKMC_CUDA(cudaMemcpyAsync(f->d_pos.p, f->h_pos, bytes, cudaMemcpyHostToDevice, f->stream));
    akmc_batch* sb = f->single;
    if (!sb->side) {
        AKMC_CUDA(cudaStreamCreateWithFlags(&sb->side, cudaStreamNonBlocking));
        AKMC_CUDA(cudaEventCreateWithFlags(&sb->ev_wrapped, cudaEventDisableTiming));
        AKMC_CUDA(cudaEventCreateWithFlags(&sb->ev_side, cudaEventDisableTiming));
    }
    akmc_status st = run_batch(sb, f->d_pos.p, f->d_force.p, f->d_energy.p, f->d_status.p, f->stream, nullptr,
                               sb->ev_wrapped);
    if (st) return st;
    // the wrapped positions go back while the force passes run (as akmc_batch_forces_host)
    AKMC_CUDA(cudaStreamWaitEvent(sb->side, sb->ev_wrapped, 0));
    AKMC_CUDA(cudaMemcpyAsync(f->h_pos, f->d_pos.p, bytes, cudaMemcpyDeviceToHost, sb->side));
    AKMC_CUDA(cudaEventRecord(sb->ev_side, sb->side));
    AKMC_CUDA(cudaMemcpyAsync(f->h_force, f->d_force.p, bytes, cudaMemcpyDeviceToHost, f->stream));
    AKMC_CUDA(cudaMemcpyAsync(f->h_energy, f->d_energy.p, sizeof(double) * 5, cudaMemcpyDeviceToHost, f->stream));
    AKMC_CUDA(cudaMemcpyAsync(f->h_status, f->d_status.p, sizeof(int), cudaMemcpyDeviceToHost, f->stream));
    AKMC_CUDA(cudaStreamWaitEvent(f->stream, sb->ev_side, 0));
    AKMC_CUDA(cudaStreamSynchronize(f->stream));
    for (int i = 0; i < n; i++) {
        px[i] = f->h_pos[3 * i + 0];
        py[i] = f->h_pos[3 * i + 1];
        pz[i] = f->h_pos[3 * i + 2];
        fx[i] = f->h_force[3 * i + 0];
        fy[i] = f->h_force[3 * i + 1];
        fz[i] = f->h_force[3 * i + 2];
    }
    if (stress) for (int k = 0; k < 6; k++) stress[k] = 0.0;
    if (out) {
        out->total = f->h_energy[0];
        out->rcp = f->h_energy[1];
        out->real = f->h_energy[2];
        out->vdw = f->h_energy[3];
        out->many = f->h_energy[4];
    }
    if (*f->h_status != AKMC_OK) return fail(*f->h_status, "kernel reported a range or value error");
    return AKMC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------
// Allocation-free EAM call: the batch scratch of one system, carved out of a fixed
// static device array instead of cudaMalloc'd buffers.
// ---------------------------------------------------------------------------------
namespace {

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr int kNaAtoms = AKMC_NOALLOC_MAX_ATOMS;
constexpr int kNaCells = AKMC_NOALLOC_MAX_CELLS;
constexpr int kNaItems = kNaCells + (kNaAtoms + kHomeChunk - 1) / kHomeChunk;
constexpr size_t kNaGeom = 0;
constexpr size_t kNaCellStart = align256(kNaGeom + sizeof(SysGeom));
constexpr size_t kNaItemsOff = align256(kNaCellStart + sizeof(int) * (kNaCells + 1));
constexpr size_t kNaNItems = align256(kNaItemsOff + sizeof(WorkItem) * kNaItems);
constexpr size_t kNaSpos = align256(kNaNItems + sizeof(int));
constexpr size_t kNaSextra = align256(kNaSpos + sizeof(double4) * kNaAtoms);
constexpr size_t kNaEatom = align256(kNaSextra + sizeof(double2) * kNaAtoms);
constexpr size_t kNaInts = align256(kNaEatom + sizeof(double2) * kNaAtoms);  // 5 int arrays
constexpr size_t kNaBytes = align256(kNaInts + 5 * sizeof(int) * (size_t)kNaAtoms);

}  // namespace

// The scratch of akmc_eam_forces_noalloc (about 0.42 MB), held by every device that
// loads this library.  Host code must not use this name as a device address: its device
// address comes from cudaGetSymbolAddress, per device, below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

namespace {

constexpr int kNaMaxDevices = 64;
unsigned char* g_noalloc_addr[kNaMaxDevices] = {nullptr};
std::mutex g_noalloc_mutex;

// Device address of the scratch array on the current device (looked up once per device).
akmc_status noalloc_scratch(int dev, unsigned char** out)
{
    if (dev < 0 || dev >= kNaMaxDevices) return fail(AKMC_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(AKMC_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_noalloc_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_noalloc_addr[dev];
    return AKMC_OK;
}

// Per-call initialisation inside the array: the system geometry and the end offset of
// the cell list (the scan in K1 writes every other entry).
__global__ void noalloc_prepare_kernel(SysGeom g, SysGeom* geom, int* cell_start, int ncell)
{
    if (threadIdx.x == 0) {
        *geom = g;
        cell_start[ncell] = g.n_atoms;
    }
}

}  // namespace

extern "C" akmc_status akmc_eam_forces_noalloc(akmc_field* f, int n, const double box[3],
                                               double* pos, const int* label, double* force,
                                               double* energy, int* status, void* stream)
{
    if (!f || !box || !pos || !label || !force || !energy || !status) return fail(AKMC_ERR_ARG, "null argument");
    if (!f->ready) return fail(AKMC_ERR_STATE, "akmc_field_setup must come first");
    if (f->pot.family != AKMC_FAMILY_EAM) return fail(AKMC_ERR_UNSUPPORTED, "the allocation-free call is EAM only");
    if (n < 1 || n > kNaAtoms)
        return fail(AKMC_ERR_CAPACITY, "allocation-free call: atom count outside 1.." + std::to_string(kNaAtoms));
    if (!(box[0] > 0 && box[1] > 0 && box[2] > 0)) return fail(AKMC_ERR_ARG, "box lengths must be positive");
    akmc_status st = cutoff_check(f, std::min(std::min(box[0], box[1]), box[2]));
    if (st) return st;
    SysGeom g;
    const int ncell = plan_system(n, box, f->pot.cutoff, kMaxCellsPerSystem, 0, 0, 0, kHomeChunk, g);
    if (ncell > kNaCells)
        return fail(AKMC_ERR_CAPACITY, "allocation-free call: cell grid larger than " + std::to_string(kNaCells));
    int dev = 0;
    AKMC_CUDA(cudaGetDevice(&dev));
    if (dev != f->device) return fail(AKMC_ERR_STATE, "current device differs from the field's device");
    unsigned char* base = nullptr;
    if ((st = noalloc_scratch(dev, &base))) return st;

    BatchDev v{};
    v.nsys = 1;
    v.n_total = n;
    v.total_cells = ncell;
    v.total_items = g.item_cap;
    v.geom = reinterpret_cast<SysGeom*>(base + kNaGeom);
    v.cell_start = reinterpret_cast<int*>(base + kNaCellStart);
    v.items = reinterpret_cast<WorkItem*>(base + kNaItemsOff);
    v.n_items = reinterpret_cast<int*>(base + kNaNItems);
    v.spos = reinterpret_cast<double4*>(base + kNaSpos);
    v.sextra = reinterpret_cast<double2*>(base + kNaSextra);
    v.eatom = reinterpret_cast<double2*>(base + kNaEatom);
    int* ints = reinterpret_cast<int*>(base + kNaInts);
    v.perm = ints;
    v.keys = ints + kNaAtoms;
    v.slots = ints + 2 * kNaAtoms;
    v.order = ints + 3 * kNaAtoms;
    v.slabel = ints + 4 * kNaAtoms;
    v.label = label;
    v.label_check = (int)f->pot.species.size();   // caller labels: checked on the device
    v.charge = nullptr;                   // read by the ionic family only
    v.sk_chunks = 1;
    v.stage_cap = std::min(kStageCap, ((n + 31) / 32) * 32);

    cudaStream_t s = (cudaStream_t)stream;
    const double rc2 = f->pot.cutoff * f->pot.cutoff;
    noalloc_prepare_kernel<<<1, 32, 0, s>>>(g, const_cast<SysGeom*>(v.geom), v.cell_start, ncell);
    AKMC_CUDA(cudaGetLastError());
    AKMC_CUDA(launch_cell_sort(v, pos, status, AKMC_FAMILY_EAM, ncell, s));
    AKMC_CUDA(launch_eam_density(v, f->eam, rc2, status, f->precision, s));
    AKMC_CUDA(launch_eam_force(v, f->eam, rc2, force, status, f->precision, s));
    AKMC_CUDA(launch_energy_reduce(v, AKMC_FAMILY_EAM, nullptr, energy, s));
    return AKMC_OK;
}

namespace akmc {

akmc_status batch_create_images(akmc_field* f, int n_groups, int n_images, const int* natoms,
                                const double* box, const int* label, const double* charge, double skin,
                                akmc_batch** out)
{
    if (!f || !out || n_groups < 1 || n_images < 1 || !natoms || !box || !label)
        return fail(AKMC_ERR_ARG, "bad image batch arguments");
    size_t atoms = 0;
    for (int k = 0; k < n_groups; k++) atoms += (size_t)std::max(natoms[k], 0);
    std::vector<int> nat, lab;
    std::vector<double> bx, q;
    for (int m = 0; m < n_images; m++) {
        nat.insert(nat.end(), natoms, natoms + n_groups);
        bx.insert(bx.end(), box, box + 3 * (size_t)n_groups);
        lab.insert(lab.end(), label, label + atoms);
        if (charge) q.insert(q.end(), charge, charge + atoms);
    }
    akmc_status st = akmc_batch_create_skin(f, n_groups * n_images, nat.data(), bx.data(), lab.data(),
                                            charge ? q.data() : nullptr, skin, out);
    if (st) return st;
    (*out)->view.n_images = n_images;
    (*out)->view.n_groups = n_groups;
    return AKMC_OK;
}

}  // namespace akmc
