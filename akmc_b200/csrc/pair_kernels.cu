// Pair kernels of the AKMC force path (sm_100a).
//
//   K2 eam_density  rho_i = sum_j rho(r_ij); F(rho_i), F'(rho_i); writes the neighbour
//        list (the reference criterion rsq <= rc^2, j != i, minimum image)
//        calculateAtomRho (potentials/metal/Field.cpp:1782-1853), ManyBody::embed
//        (potentials/metal/ManyBody.cpp:554-619)
//   K3 eam_force    F_i = -sum_j [phi'(r) + (F'_i + F'_j) rho'(r)] (r_i - r_j)/r,
//        E_pair = sum_{i<j} phi, thread per atom over the K2 list: realSpaceForceImage
//        pass 2 (metal/Field.cpp:371-449), calculateManyBodyPairForce /
//        calculateManyBodyForce (ManyBody.cpp:621-831)
//   K4+K6 ionic_force  Ewald real space erfc(eta r)/r + Buckingham
//        (pair/Field.cpp:660-842, TwoBody.h:203-215, hfunc1 pair/Field.cpp:2218-2236),
//        fused with the reciprocal-space force of the same atom (Ewald.cpp:636-646)
//   K5 structure_factor  C_k = sum q cos(k.r), S_k = sum q sin(k.r) (Ewald.cpp:585-611)
//   K7 energy_reduce  per-system FP64 energies, Ewald self term (pair/Field.cpp:704-720)
//
// Work decomposition of K2/K4 (and of the cell-scan EAM force pass kept for the
// allocation-free call): one CTA per work item (<= home_chunk home atoms of one cell,
// built by K1).  The CTA stages the neighbour cells in shared memory as FP32 coordinates
// relative to the home cell centre (periodic shift folded in) plus the atom index, 16
// bytes per candidate.  Each warp then takes one home atom at a time: lanes screen 32
// candidates at once in FP32 against a slightly enlarged cutoff, survivors are compacted
// into per-warp queues (ballot + popc), and full warps of queued pairs redo the
// separation in FP64 from the sorted positions (the exact reference test rsq <= rc^2
// decides) before evaluating the pair terms.  Lane partial sums are reduced with warp
// shuffles in a fixed order, so results are bitwise reproducible.
//
// Precision (AKMC_PREC_MIXED): separations, r and all force accumulations FP64; EAM table
// interpolation FP32; ionic pair terms FP32 beyond r_split and FP64 inside it (the nearest
// shells carry the largest forces); structure factors from FP64 per-atom terms, reciprocal
// force terms in FP32 from FP64-tabulated phases.  AKMC_PREC_FP64: every term FP64.  The FP32 screen only
// preselects: it accepts every pair within rc*(1 + 5e-4), far beyond its rounding error.
#include "akmc_internal.h"

namespace akmc {

AKMC_CHECKS_FILE(pair)

namespace {

constexpr unsigned kFull = 0xffffffffu;
// Entries of a warp's phase table in the reciprocal loop (the warp's compaction queues of the
// cell-scan kernel hold 64 float2; larger k-sets take the direct FP32 phases).
constexpr int kWarpTab = 64;
static_assert(kWarpTab <= kMaxPhaseTable, "warp phase table");
constexpr float kTwoOverRootPiF = 1.128379167095512f;
// FP32 screen: rc^2 * (1 + 1e-3); FP32 relative coordinates err by < 1e-5 A
constexpr double kScreenSlack = 1.0e-3;

__device__ __forceinline__ void set_status(int* st, int code) { atomicCAS(st, 0, code); }

// Programmatic dependent launch: see akmc_internal.h.
__device__ __forceinline__ void wait_for_prior_grid() { pdl_wait(); }

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Read-only load of a 32-byte record as two 16-byte read-only loads.
__device__ __forceinline__ double4 ldg4(const double4* p)
{
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ double warp_sum(double v)
{
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// r and 1/r from r^2: FP32 reciprocal square root as the seed, then one Newton-Raphson
// step y <- y (3 - x y^2) / 2 in FP64, which squares the relative error (~1e-7 -> ~1e-14).
__device__ __forceinline__ void refined_sqrt(double rsq, double& r, double& inv_r)
{
    double y = (double)rsqrtf((float)rsq);
    y = y * (1.5 - 0.5 * rsq * y * y);
    inv_r = y;
    r = rsq * y;
}

// u - rint(u) with the 1.5 * 2^52 rounding constant (FP64 adds only; exact for |u| < 2^51,
// ties to even like rint).
__device__ __forceinline__ double frac_nearest(double u)
{
    const double M = 6755399441055744.0;
    return u - ((u + M) - M);
}

// Minimum image of a separation d: d - L*rint(d/L), the reference's fold
// (metal/Field.cpp:397-414), rint by the 1.5 * 2^52 rounding constant (measured faster
// on this kernel than a compare-and-select fold).
__device__ __forceinline__ double fold(double d, double L, double iL)
{
    const double M = 6755399441055744.0;
    const double n = (d * iL + M) - M;
    return fma(-n, L, d);
}

// FP32 fold for the screen (|d| < L): compare, select and add; ties at |d| = L/2 stay
// unshifted as rint leaves them.
__device__ __forceinline__ float foldf(float d, float L, float hL)
{
    return fabsf(d) > hL ? d - copysignf(L, d) : d;
}

// ---------------------------------------------------------------------------------
// neighbour ranges of one home cell
// ---------------------------------------------------------------------------------
struct RangeSet {
    int n, total, home_range, home_start;
    int start[27];
    int prefix[28];
    double shift[27][3];
    double centre[3];
};

// Built by warp 0.  Dimensions with fewer than 3 cells take every cell once and use
// the per-pair minimum image; others take the home cell and its two neighbours with the
// periodic shift folded into the staged coordinates.
__device__ void build_ranges(const BatchDev& b, const SysGeom& g, int cell, RangeSet& rs)
{
    const int lane = threadIdx.x & 31;
    const int c = cell - g.cell_begin;
    const int nc0 = g.nc[0], nc1 = g.nc[1], nc2 = g.nc[2];
    const int h[3] = {c % nc0, (c / nc0) % nc1, c / (nc0 * nc1)};
    const int nc[3] = {nc0, nc1, nc2};
    int cnt[3];
    #pragma unroll
    for (int d = 0; d < 3; d++) cnt[d] = (g.mi_mask >> d & 1) ? nc[d] : 3;
    const int ncomb = cnt[0] * cnt[1] * cnt[2];
    int len = 0, st = 0;
    bool home = false;
    if (lane < ncomb) {
        const int o[3] = {lane % cnt[0], (lane / cnt[0]) % cnt[1], lane / (cnt[0] * cnt[1])};
        int cc[3];
        double sh[3];
        #pragma unroll
        for (int d = 0; d < 3; d++) {
            sh[d] = 0.0;
            if (g.mi_mask >> d & 1) {
                cc[d] = o[d];
            } else {
                cc[d] = h[d] + o[d] - 1;
                if (cc[d] < 0) { cc[d] += nc[d]; sh[d] = -g.L[d]; }
                else if (cc[d] >= nc[d]) { cc[d] -= nc[d]; sh[d] = g.L[d]; }
            }
        }
        const int nb = (cc[2] * nc1 + cc[1]) * nc0 + cc[0];
        st = b.cell_start[g.cell_begin + nb];
        len = b.cell_start[g.cell_begin + nb + 1] - st;
        home = (nb == c);
        rs.start[lane] = st;
        rs.shift[lane][0] = sh[0];
        rs.shift[lane][1] = sh[1];
        rs.shift[lane][2] = sh[2];
    }
    int incl = len;
    #pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        int y = __shfl_up_sync(kFull, incl, off);
        if (lane >= off) incl += y;
    }
    if (lane < ncomb) rs.prefix[lane] = incl - len;
    const unsigned hb = __ballot_sync(kFull, home);
    if (lane == 0) {
        rs.n = ncomb;
        rs.home_range = __ffs(hb) - 1;
        // reference point of the FP32 relative coordinates: the home cell centre in
        // shifted dimensions, the cell origin in minimum-image dimensions
        #pragma unroll
        for (int d = 0; d < 3; d++)
            rs.centre[d] = (g.mi_mask >> d & 1) ? 0.0 : (h[d] + 0.5) * g.L[d] / nc[d] - 0.5 * g.L[d];
    }
    if (lane == ncomb - 1) {
        rs.total = incl;
        rs.prefix[ncomb] = incl;
    }
    if (home) rs.home_start = st;
}

__device__ __forceinline__ int find_range(const RangeSet& rs, int f)
{
    int lo = 0, hi = rs.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (rs.prefix[mid] <= f) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int find_system_by_item(const BatchDev& b, int blk)
{
    int lo = 0, hi = b.nsys - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (b.geom[mid].item_base <= blk) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int find_system_by_atom(const BatchDev& b, int i)
{
    int lo = 0, hi = b.nsys - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (b.geom[mid].atom_begin <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// How a pass stages its candidates in shared memory and screens them.
//   kStageF32W:  float4 {x, y, z relative to the cell reference point, int w}; FP32 screen
//                with slack; every queued pair re-tested in FP64 from the sorted positions
//   kStageF64:   double4 {x, y, z (periodic shift applied), w} + int w; FP64 screen with
//                the exact test; queued pairs never touch global memory
//   kStageF32Q:  float4 {x, y, z relative, charge} + int (j << 4 | species); FP32 screen
//                that sorts pairs three ways (pass classify): definitely inside the cutoff
//                and beyond the near-pair radius -> queue 0, evaluated from the staged FP32
//                record alone; near pairs and pairs within a relative 1e-5 of the cutoff ->
//                queue 1, FP64 separation from the sorted positions, the exact test
//                rsq <= rc^2, FP64 terms
enum StageMode { kStageF32W = 0, kStageF64 = 1, kStageF32Q = 2 };

struct Geo {            // per-CTA copy of the system geometry used in the inner loops
    double L0, L1, L2, hL0, hL1, hL2, iL0, iL1, iL2;
    float Lf0, Lf1, Lf2, hLf0, hLf1, hLf2;
    int mi;
};

__device__ __forceinline__ Geo make_geo(const SysGeom& g, int mi)
{
    Geo G;
    G.L0 = g.L[0]; G.L1 = g.L[1]; G.L2 = g.L[2];
    G.hL0 = 0.5 * g.L[0]; G.hL1 = 0.5 * g.L[1]; G.hL2 = 0.5 * g.L[2];
    G.iL0 = g.invL[0]; G.iL1 = g.invL[1]; G.iL2 = g.invL[2];
    G.Lf0 = (float)g.L[0]; G.Lf1 = (float)g.L[1]; G.Lf2 = (float)g.L[2];
    G.hLf0 = 0.5f * G.Lf0; G.hLf1 = 0.5f * G.Lf1; G.hLf2 = 0.5f * G.Lf2;
    G.mi = mi;
    return G;
}

// FP64 minimum-image separation, folding the dimensions set in mi (7 for two wrapped
// positions; G.mi for a staged neighbour whose periodic shift is already applied).
__device__ __forceinline__ double displacement(const Geo& G, int mi, double hx, double hy,
                                               double hz, const double4& p, double& dx,
                                               double& dy, double& dz)
{
    dx = hx - p.x;
    dy = hy - p.y;
    dz = hz - p.z;
    if (mi & 1) dx = fold(dx, G.L0, G.iL0);
    if (mi & 2) dy = fold(dy, G.L1, G.iL1);
    if (mi & 4) dz = fold(dz, G.L2, G.iL2);
    return dx * dx + dy * dy + dz * dz;
}

// ---------------------------------------------------------------------------------
// passes
// ---------------------------------------------------------------------------------
template <int N>
struct AccN {
    double v[N];
    __device__ __forceinline__ void zero()
    {
        #pragma unroll
        for (int k = 0; k < N; k++) v[k] = 0.0;
    }
    // warp totals of every accumulator, valid in every lane
    __device__ __forceinline__ void reduce(double* out)
    {
        #pragma unroll
        for (int k = 0; k < N; k++) out[k] = warp_sum(v[k]);
    }
};

// Shared context every pass receives for a home atom.
struct Home {
    int i;          // sorted global index
    int a0;         // first atom of the system
    int* st;        // status word of the system
    int lrow;       // its neighbour-list row (i, or the same atom of its group's image 0)
};

// rho_j(r) of one pair (ManyBody::calculateManyBodyDensEnergy EAM branch,
// ManyBody.cpp:539-549): 0 for a species without a density table or beyond the table's
// cutoff, a status for r below the first bin.
template <bool kFp64>
__device__ __forceinline__ double eam_rho_term(const EamDev& P, double rsq, int lj, int* st)
{
    if (!P.dens_ok[lj]) return 0.0;
    const int k = P.ntab > 1 ? P.mesh[lj * P.ns + lj] : 0;     // the neighbour's own table
    double r, ir;
    if (kFp64) { r = sqrt(rsq); } else { refined_sqrt(rsq, r, ir); }
    if (r < 1.0e-8 || !(r < P.pot_cutoff)) return 0.0;
    const double tr = r * P.inv_step_r;
    const int idx = (int)tr;
    if (idx >= P.n_r - 1) { set_status(st, AKMC_ERR_TABLE_RANGE); return 0.0; }
    if (kFp64) {
        const double* rho = P.rho + (size_t)k * P.n_r;
        const double p0 = rho[idx], p1 = rho[idx + 1];
        return p0 + (p1 - p0) * (r - idx * P.step_r) * P.inv_step_r;
    }
    const float4 row = __ldg(&P.rows[2 * ((size_t)k * P.n_r + idx) + 1]);
    return (double)(row.z + row.w * (float)(tr - idx));
}

// derivEmbed of table k at rho (ManyBody.cpp:797-810, used per pair when a field holds more
// than one table); the reference exits when the index leaves the table, here a status and 0.
__device__ __forceinline__ double eam_dembed(const EamDev& P, int k, double rho, int* st)
{
    const int idx = (int)(rho * P.inv_step_embed);
    if (idx < 0 || idx >= P.n_embed - 1) {
        set_status(st, AKMC_ERR_EMBED_RANGE);
        return 0.0;
    }
    const double t = (rho - idx * P.step_embed) * P.inv_step_embed;
    const double* dF = P.dF + (size_t)k * P.n_embed;
    return dF[idx] + (dF[idx + 1] - dF[idx]) * t;
}

// ManyBody::embed EAM branch (ManyBody.cpp:598-615) for F and, once per atom, the
// derivEmbed interpolation the force pass needs (ManyBody.cpp:797-810).
__device__ __forceinline__ void eam_embed(const EamDev& P, int li, double rho, int i, int* st,
                                          double2* sextra, double2* eatom, double4* frec,
                                          const double4& hp)
{
    double F = 0.0, fp = 0.0;
    if (P.embed_ok[li]) {
        const int idx = (int)(rho * P.inv_step_embed);
        if (idx < 0 || idx >= P.n_embed - 1) {
            set_status(st, AKMC_ERR_EMBED_RANGE);
        } else {
            const size_t k = (size_t)P.mesh[li * P.ns + li] * P.n_embed;     // its own table
            const double t = (rho - idx * P.step_embed) * P.inv_step_embed;
            F = P.F[k + idx] + (P.F[k + idx + 1] - P.F[k + idx]) * t;
            fp = P.dF[k + idx] + (P.dF[k + idx + 1] - P.dF[k + idx]) * t;
        }
    }
    sextra[i] = make_double2(fp, rho);
    eatom[i].x = F;
    // the force pass's record: F' (one table), or the density itself (several tables: F' then
    // comes from each pair's table); NaN below the density floor
    if (frec) frec[i] = make_double4(hp.x, hp.y, hp.z, rho < 1.0e-8 ? __longlong_as_double(0x7ff8000000000000ll)
                                                                     : (P.ntab > 1 ? rho : fp));
}

// K2: EAM density, and the neighbour list of the force pass.  spos.w holds the species
// label.
template <bool kFp64>
struct EamDensityPass {
    static constexpr int kAcc = 1, kQueues = 1, kMinBlocks = 8, kThreads = kPairThreads;
    // ~13 % of candidates survive: screen in FP32 (16-byte staged records); accepted pairs
    // read their FP64 record from global memory
    static constexpr int kStage = kStageF32W;
    static constexpr bool kOverlapPrior = false;
    __device__ int stage_w(const BatchDev&, int j) const { return j; }
    using Acc = AccN<1>;
    EamDev P;
    double2* sextra;
    double2* eatom;
    unsigned short* nbr;
    int* nbr_count;
    int nbr_cap, n_total;
    double rc2_acc;      // the density sum takes pairs within the cutoff; the list, within cutoff + skin
    double4* frec;
    struct Ctx { int li; };

    __device__ Ctx home(const BatchDev& b, const Home& h) const { return Ctx{b.slabel[h.i]}; }
    __device__ int classify(float) const { return 0; }

    __device__ void pair(int, Acc& acc, const Home& h, const Ctx&, double, double, double,
                         double rsq, const double4& pj, int j, int slot) const
    {
        if (nbr) {
            if (AKMC_BAD(h.lrow < 0 || h.lrow >= n_total, 1, h.lrow)) return;
            if (slot < nbr_cap) nbr[(size_t)slot * n_total + h.lrow] = (unsigned short)(j - h.a0);
            else set_status(h.st, AKMC_ERR_CAPACITY);
        }
        if (!(rsq <= rc2_acc)) return;
        acc.v[0] += eam_rho_term<kFp64>(P, rsq, (int)pj.w, h.st);
    }

    __device__ void post(const BatchDev&, int, const Geo&, const double4&, const Home&, const Ctx&,
                         Acc&, float2*) const {}

    __device__ void finish(const BatchDev& b, const Home& h, const Ctx& cx, const double* a,
                           int listed) const
    {
        eam_embed(P, cx.li, a[0], h.i, h.st, sextra, eatom, frec, b.spos[h.i]);
        if (nbr && !AKMC_BAD(h.lrow < 0 || h.lrow >= n_total, 1, h.lrow)) nbr_count[h.lrow] = min(listed, nbr_cap);
    }
};

// EAM pair term shared by the cell-scan and the list force passes:
// g = (phi'(r) + (F'_i + F'_j) rho'(r)) / r and the pair energy phi(r).
// mb: both densities >= 1e-8 (ManyBody.cpp:730-731); fps = F'_i + F'_j.
// k: the pair's table.
template <bool kFp64>
__device__ __forceinline__ bool eam_pair_term_mb(const EamDev& P, int k, double rsq, bool mb, double fps,
                                                 int* st, double& g, double& phi)
{
    double r, ir;
    if (kFp64) { r = sqrt(rsq); ir = 1.0 / r; } else { refined_sqrt(rsq, r, ir); }
    if (r < 1.0e-8 || !(r < P.pot_cutoff)) return false;
    const double tr = r * P.inv_step_r;
    const int idx = (int)tr;
    if (idx >= P.n_r - 1) { set_status(st, AKMC_ERR_TABLE_RANGE); return false; }
    if (kFp64) {
        const size_t o = (size_t)k * P.n_r + idx;
        const double w = (r - idx * P.step_r) * P.inv_step_r;
        phi = P.phi[o] + (P.phi[o + 1] - P.phi[o]) * w;
        const double dphi = P.dphi[o] + (P.dphi[o + 1] - P.dphi[o]) * w;
        const double drho = P.drho[o] + (P.drho[o + 1] - P.drho[o]) * w;
        g = (dphi + (mb ? fps * drho : 0.0)) * ir;
    } else {
        const size_t o = 2 * ((size_t)k * P.n_r + idx);
        const float ft = (float)(tr - idx);
        const float4 A = __ldg(&P.rows[o]);
        const float4 B = __ldg(&P.rows[o + 1]);
        const float phif = A.x + A.y * ft;
        const float dphi = A.z + A.w * ft;
        const float drho = B.x + B.y * ft;
        const float many = mb ? (float)fps * drho : 0.0f;
        phi = (double)phif;
        g = (double)(dphi + many) * ir;
    }
    return true;
}

template <bool kFp64>
__device__ __forceinline__ bool eam_pair_term(const EamDev& P, int k, double rsq, double fpi, double rhoi,
                                              double fpj, double rhoj, int* st, double& g,
                                              double& phi)
{
    const bool mb = !(rhoi < 1.0e-8 || rhoj < 1.0e-8);
    const double fps = P.ntab > 1 ? (mb ? eam_dembed(P, k, rhoi, st) + eam_dembed(P, k, rhoj, st) : 0.0) : fpi + fpj;
    return eam_pair_term_mb<kFp64>(P, k, rsq, mb, fps, st, g, phi);
}

// K3 (cell scan): EAM force and pair energy.  Used when the batch holds no neighbour
// list (the allocation-free call).
template <bool kFp64>
struct EamForcePass {
    static constexpr int kAcc = 4, kQueues = 1, kMinBlocks = 4, kThreads = kPairThreads;
    static constexpr int kStage = kStageF32W;
    static constexpr bool kOverlapPrior = false;
    __device__ int stage_w(const BatchDev&, int j) const { return j; }
    using Acc = AccN<4>;
    EamDev P;
    double* force;
    double2* eatom;
    struct Ctx { int li; double fpi, rhoi; };

    __device__ Ctx home(const BatchDev& b, const Home& h) const
    {
        const double2 e = b.sextra[h.i];
        return Ctx{b.slabel[h.i], e.x, e.y};
    }
    __device__ int classify(float) const { return 0; }

    __device__ void pair(int, Acc& acc, const Home& h, const Ctx& cx, double dx, double dy,
                         double dz, double rsq, const double4& pj, int j, int) const
    {
        const int lj = (int)pj.w;
        if (!P.pair_ok[cx.li * P.ns + lj]) return;
        const double2 ej = __ldg(&sextra_of(j));
        double g, phi;
        if (!eam_pair_term<kFp64>(P, P.mesh[cx.li * P.ns + lj], rsq, cx.fpi, cx.rhoi, ej.x, ej.y, h.st, g, phi))
            return;
        acc.v[0] -= g * dx;
        acc.v[1] -= g * dy;
        acc.v[2] -= g * dz;
        acc.v[3] += 0.5 * phi;
    }
    const double2* sextra;
    __device__ const double2& sextra_of(int j) const { return sextra[j]; }

    __device__ void post(const BatchDev&, int, const Geo&, const double4&, const Home&, const Ctx&,
                         Acc&, float2*) const {}

    __device__ void finish(const BatchDev& b, const Home& h, const Ctx&, const double* a, int) const
    {
        const int o = b.perm[h.i];
        if (AKMC_BAD(o < 0 || o >= b.n_total, 5, o)) return;
        force[3 * (size_t)o + 0] = a[0];
        force[3 * (size_t)o + 1] = a[1];
        force[3 * (size_t)o + 2] = a[2];
        eatom[h.i].y = a[3];
    }
};

// K4+K6: ionic real space (queue 0 = FP32 terms, queue 1 = FP64 terms) fused with the
// reciprocal-space force of the home atom.
struct IonicAcc {
    double v[5];     // fx, fy, fz, E_real (FP64 terms), E_vdw (FP64 terms)
    float w[2];      // E_real, E_vdw of the FP32 terms (lane partials of ~14 terms)
    __device__ __forceinline__ void zero()
    {
        #pragma unroll
        for (int k = 0; k < 5; k++) v[k] = 0.0;
        w[0] = w[1] = 0.0f;
    }
    __device__ __forceinline__ void reduce(double* out)
    {
        out[0] = warp_sum(v[0]);
        out[1] = warp_sum(v[1]);
        out[2] = warp_sum(v[2]);
        out[3] = warp_sum(v[3] + (double)w[0]);
        out[4] = warp_sum(v[4] + (double)w[1]);
    }
};

template <bool kFp64>
struct IonicPass {
    static constexpr int kAcc = 5, kQueues = kFp64 ? 1 : 2;
    // mixed: 8 warps share one staged neighbourhood; 4 CTAs x 8 warps per SM at 64
    // registers
    static constexpr int kThreads = kFp64 ? kPairThreads : 256;
    static constexpr int kMinBlocks = kFp64 ? 1 : 4;
    // FP64 terms: stage the FP64 records (36 bytes each) and screen in FP64, so queued pairs
    // never touch global memory; the staged int is the species label.  Mixed: FP32 screen,
    // far pairs (about 93 % of the ~45 % that survive) evaluated from the staged FP32 record
    static constexpr int kStage = kFp64 ? kStageF64 : kStageF32Q;
    // the real-space part runs while the structure-factor kernel finishes; post() waits
    static constexpr bool kOverlapPrior = true;
    __device__ int stage_w(const BatchDev& b, int j) const { return b.slabel[j]; }
    using Acc = IonicAcc;
    IonicDev P;
    const double2* sk;
    const float2* skf;
    const int* slabel;
    double* force;
    double2* eatom;
    float r_split2f;
    float rc2_lo, rc2_hi;    // rc^2 (1 -/+ 1e-5): FP32 squared distances between them go to the exact test
    struct Ctx { int li; double cqi; float cqf; double qi; };

    __device__ Ctx home(const BatchDev& b, const Home& h) const
    {
        const double q = b.spos[h.i].w;
        return Ctx{b.slabel[h.i], P.cfact * q, (float)(P.cfact * q), q};
    }
    // FP64 mode: every pair that passed the exact test is queue 0.  Mixed (FP32 squared
    // distance of the staged records, error < 1e-6 relative): -1 beyond the cutoff, 1 for
    // near pairs and pairs at the cutoff (exact test and FP64 terms), 0 for the rest
    __device__ int classify(float rsq) const
    {
        if (kFp64) return 0;
        if (!(rsq <= rc2_hi)) return -1;
        return (rsq < r_split2f || rsq > rc2_lo) ? 1 : 0;
    }

    // The FP32 terms of a pair: Ewald real space (hfunc1, pair/Field.cpp:2218-2236) and
    // Buckingham (TwoBody.h:203-215).  forc = (1/r) dE/dr, so the force on the home atom is
    // -forc (r_i - r_j); eng and evdw are the pair's real-space and short-range energies.
    __device__ __forceinline__ float4 buck32(int ab) const
    {
        return make_float4(P.buckAf[ab], P.buckInvRhof[ab], P.buckCf[ab], 0.0f);
    }

    // bk = {A, 1/rho, C, -} of the species pair
    __device__ __forceinline__ void terms32(const float4& bk, float cqf, float qj, float rsqf, float& forc_out,
                                            float& eng_out, float& evdw_out) const
    {
        const float ir = rsqrtf(rsqf);
        const float r = rsqf * ir;
        const float x = P.etaf * r;
        const float ix = ir * P.inv_etaf;
        const float qq = cqf * qj;
        float h0, h1;
        if (P.erfcx_on) {
            // erfc(x) = exp(-x^2) R(x), R the fitted polynomial (one exp for both terms)
            const float t = fminf(fmaxf(fmaf(x, P.erfcx_t1, P.erfcx_t0), -1.0f), 1.0f);
            float R = P.erfcx_c[kErfcxDeg];
            #pragma unroll
            for (int k = kErfcxDeg - 1; k >= 1; k--) R = fmaf(R, t, P.erfcx_c[k]);
            R = fmaf(R, t, P.erfcx_c0lo) + P.erfcx_c[0];    // the constant's rounding kept: no bias
            const float g = expf(-x * x);
            h0 = g * R * ix;
            h1 = (-h0 - kTwoOverRootPiF * g) * (ix * ix);
        } else {
            h0 = erfcf(x) * ix;
            h1 = (-h0 - kTwoOverRootPiF * expf(-x * x)) * (ix * ix);
        }
        float forc = h1 * qq * P.eta3f;
        const float irho = bk.y;
        const float e1 = bk.x * expf(-r * irho);
        const float f1 = e1 * irho * ir;
        const float ir2 = ir * ir;
        const float e2 = -bk.z * (ir2 * ir2 * ir2);
        const float f2 = 6.0f * e2 * ir2;
        forc_out = forc - (f1 + f2);
        eng_out = h0 * qq * P.etaf;
        evdw_out = e1 + e2;
    }

    // A far pair in FP32 from the staged records (mixed mode, queue 0), the force
    // accumulated in FP64.
    __device__ __forceinline__ void pair32(Acc& acc, const Ctx& cx, float dx, float dy, float dz, float rsqf,
                                           float qj, int lj) const
    {
        float forc, eng, evdw;
        terms32(buck32(cx.li * P.ns + lj), cx.cqf, qj, rsqf, forc, eng, evdw);
        const double fd = (double)forc;
        acc.v[0] -= fd * (double)dx;
        acc.v[1] -= fd * (double)dy;
        acc.v[2] -= fd * (double)dz;
        acc.w[0] += 0.5f * eng;
        acc.w[1] += 0.5f * evdw;
    }

    // The FP64 terms of a pair of species pair ab: forc = (1/r) dE/dr, eng its real-space
    // and es its short-range energy (cqi: the home atom's charge times the Coulomb factor).
    __device__ __forceinline__ void terms64(int ab, double cqi, double qj, double rsq, double& forc_out,
                                            double& eng_out, double& es_out) const
    {
        double r, ir;
        if (kFp64) { r = sqrt(rsq); ir = 1.0 / r; } else { refined_sqrt(rsq, r, ir); }
        const double qq = cqi * qj;
        const double x = P.eta * r;
        double forc = 0.0, eng = 0.0, es = 0.0;
        if (x != 0.0) {
            const double ix = ir * P.inv_eta;
            const double h0 = erfc(x) * ix;
            const double h1 = (-h0 - kTwoOverRootPi * exp(-x * x)) * (ix * ix);
            eng = h0 * qq * P.eta;
            forc = h1 * qq * (P.eta * P.eta * P.eta);
        }
        if (r >= 1.0e-8) {
            const double irho = P.buckInvRho[ab];
            const double e1 = P.buckA[ab] * exp(-r * irho);
            const double f1 = e1 * irho * ir;
            const double ir2 = ir * ir;
            const double e2 = -P.buckC[ab] * (ir2 * ir2 * ir2);
            const double f2 = 6.0 * e2 * ir2;
            es = e1 + e2;
            forc -= f1 + f2;
        }
        forc_out = forc;
        eng_out = eng;
        es_out = es;
    }

    // A pair in FP64 terms: every pair in FP64 mode; near pairs and pairs at the cutoff in
    // the mixed mode (queue 1).  j is the partner's species label, pj.w its charge.
    __device__ void pair(int, Acc& acc, const Home&, const Ctx& cx, double dx, double dy,
                         double dz, double rsq, const double4& pj, int j, int) const
    {
        double forc, eng, es;
        terms64(cx.li * P.ns + j, cx.cqi, pj.w, rsq, forc, eng, es);
        acc.v[0] -= forc * dx;
        acc.v[1] -= forc * dy;
        acc.v[2] -= forc * dz;
        acc.v[3] += 0.5 * eng;
        acc.v[4] += 0.5 * es;
    }

    // Reciprocal force on the home atom (Ewald.cpp:636-646): lanes stride over k.
    // F_i = sum_k g0_k q_i (sin(k.r_i) C_k - cos(k.r_i) S_k) k.
    // Mixed precision: the warp first tabulates the atom's 1-D phase factors
    // e^{2 pi i n s_d} (FP64 sincospi, one per table entry) in `tab`; the phase of
    // k = 2 pi (nx/Lx, ny/Ly, nz/Lz) is then the product of three entries (FP32 complex).
    __device__ void post(const BatchDev&, int s, const Geo& G, const double4& hp, const Home&,
                         const Ctx& cx, Acc& acc, float2* tab) const
    {
        const int lane = threadIdx.x & 31;
        const double sx = hp.x * G.iL0, sy = hp.y * G.iL1, sz = hp.z * G.iL2;
        if (!kFp64 && P.ntab <= kWarpTab) {
            const int oy = P.gx + 1, oz = oy + 2 * P.gy + 1;
            for (int l = lane; l < P.ntab; l += 32) {
                double u;
                if (l < oy) u = l * sx;
                else if (l < oz) u = (l - oy - P.gy) * sy;
                else u = (l - oz - P.gz) * sz;
                double sn, cn;
                sincospi(2.0 * u, &sn, &cn);
                tab[l] = make_float2((float)cn, (float)sn);
            }
            __syncwarp();
            wait_for_prior_grid();            // C_k, S_k come from the structure-factor kernel
            const float2* skk = skf + (size_t)s * P.nk;
            const float qf = (float)cx.qi;
            float ax = 0.0f, ay = 0.0f, az = 0.0f;
            for (int k = lane; k < P.nk; k += 32) {
                const int4 t = __ldg(&P.kt[k]);
                const float4 kf = __ldg(&P.kf[k]);
                const float2 cs = skk[k];
                const float2 X = tab[t.x], Y = tab[t.y], Z = tab[t.z];
                const float xyr = X.x * Y.x - X.y * Y.y, xyi = X.x * Y.y + X.y * Y.x;
                const float cn = xyr * Z.x - xyi * Z.y, sn = xyr * Z.y + xyi * Z.x;
                const float pf = kf.w * qf * (sn * cs.x - cn * cs.y);
                ax += pf * kf.x;
                ay += pf * kf.y;
                az += pf * kf.z;
            }
            __syncwarp();
            acc.v[0] += (double)ax * kTwoPi * G.iL0;
            acc.v[1] += (double)ay * kTwoPi * G.iL1;
            acc.v[2] += (double)az * kTwoPi * G.iL2;
            return;
        }
        wait_for_prior_grid();
        if (kFp64) {
            const double2* skk = sk + (size_t)s * P.nk;
            double ax = 0.0, ay = 0.0, az = 0.0;
            for (int k = lane; k < P.nk; k += 32) {
                const double4 kd = ldg4(&P.kd[k]);
                const double2 cs = skk[k];
                const double u = frac_nearest(kd.x * sx + kd.y * sy + kd.z * sz);
                double sn, cn;
                sincospi(2.0 * u, &sn, &cn);
                const double pf = kd.w * cx.qi * (sn * cs.x - cn * cs.y);
                ax += pf * kd.x;
                ay += pf * kd.y;
                az += pf * kd.z;
            }
            acc.v[0] += ax * kTwoPi * G.iL0;
            acc.v[1] += ay * kTwoPi * G.iL1;
            acc.v[2] += az * kTwoPi * G.iL2;
        } else {
            const float2* skk = skf + (size_t)s * P.nk;
            const float qf = (float)cx.qi;
            float ax = 0.0f, ay = 0.0f, az = 0.0f;
            for (int k = lane; k < P.nk; k += 32) {
                const double4 kd = ldg4(&P.kd[k]);
                const float4 kf = __ldg(&P.kf[k]);
                const float2 cs = skk[k];
                const double u = frac_nearest(kd.x * sx + kd.y * sy + kd.z * sz);
                float sn, cn;
                sincospif(2.0f * (float)u, &sn, &cn);
                const float pf = kf.w * qf * (sn * cs.x - cn * cs.y);
                ax += pf * kf.x;
                ay += pf * kf.y;
                az += pf * kf.z;
            }
            acc.v[0] += (double)ax * kTwoPi * G.iL0;
            acc.v[1] += (double)ay * kTwoPi * G.iL1;
            acc.v[2] += (double)az * kTwoPi * G.iL2;
        }
    }

    __device__ void finish(const BatchDev& b, const Home& h, const Ctx&, const double* a, int) const
    {
        const int o = b.perm[h.i];
        if (AKMC_BAD(o < 0 || o >= b.n_total, 5, o)) return;
        force[3 * (size_t)o + 0] = a[0];
        force[3 * (size_t)o + 1] = a[1];
        force[3 * (size_t)o + 2] = a[2];
        eatom[h.i] = make_double2(a[3], a[4]);
    }
};

// ---------------------------------------------------------------------------------
// the shared cell-scan kernel
// ---------------------------------------------------------------------------------
// One work item (home atoms of one cell against the cells around it) of a pair pass.
template <class Pass>
__device__ __forceinline__ void pair_item(const BatchDev& b, const Pass& pass, double rc2, int* status, int s,
                                          const WorkItem& it, float4* s_pos, double4* s_p64, int* s_w,
                                          RangeSet& rs, int (*s_q)[2][64], double (*s_acc)[Pass::kAcc],
                                          int* s_listed)
{
    constexpr int kWarps = Pass::kThreads / 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const SysGeom& gref = b.geom[s];
    const Geo G = make_geo(gref, gref.mi_mask);
    int* st = status + s;
    const int a0 = gref.atom_begin;
    const int lshift = list_shift(b, s);

    if (warp == 0) {
        const SysGeom g = gref;
        build_ranges(b, g, it.cell, rs);
    }
    for (int k = tid; k < kHomeChunk * Pass::kAcc; k += blockDim.x) (&s_acc[0][0])[k] = 0.0;
    for (int k = tid; k < kHomeChunk; k += blockDim.x) s_listed[k] = 0;
    __syncthreads();

    const int total = rs.total;
    const int cap = b.stage_cap;
    const bool single = total <= cap;
    const int self_base = rs.prefix[rs.home_range] - rs.home_start;
    const double c0 = rs.centre[0], c1 = rs.centre[1], c2 = rs.centre[2];
    const float rc2f = (float)(rc2 * (1.0 + kScreenSlack));

    for (int rb = 0; rb < total; rb += cap) {
        const int m = min(cap, total - rb);
        __syncthreads();
        for (int t = tid; t < m; t += blockDim.x) {
            const int f = rb + t;
            const int ri = find_range(rs, f);
            int j = rs.start[ri] + (f - rs.prefix[ri]);
            if (AKMC_BAD(j < gref.atom_begin || j >= gref.atom_begin + gref.n_atoms, 9, j)) j = gref.atom_begin;
            const double4 p = b.spos[j];
            const double x = p.x + rs.shift[ri][0], y = p.y + rs.shift[ri][1], z = p.z + rs.shift[ri][2];
            if (Pass::kStage == kStageF64) {
                s_p64[t] = make_double4(x, y, z, p.w);
                s_w[t] = pass.stage_w(b, j);
            } else if (Pass::kStage == kStageF32Q) {
                s_pos[t] = make_float4((float)(x - c0), (float)(y - c1), (float)(z - c2), (float)p.w);
                s_w[t] = (j << 4) | pass.stage_w(b, j);
            } else {
                s_pos[t] = make_float4((float)(x - c0), (float)(y - c1), (float)(z - c2),
                                       __int_as_float(pass.stage_w(b, j)));
            }
        }
        __syncthreads();

        for (int a = warp; a < it.count; a += kWarps) {
            const Home h{it.first + a, a0, st, it.first + a + lshift};
            const double4 hp = b.spos[h.i];
            constexpr bool kF64 = Pass::kStage == kStageF64;
            const float hx = kF64 ? 0.f : (float)(hp.x - c0);
            const float hy = kF64 ? 0.f : (float)(hp.y - c1);
            const float hz = kF64 ? 0.f : (float)(hp.z - c2);
            const auto cx = pass.home(b, h);
            const int self_t = self_base + h.i - rb;
            typename Pass::Acc acc;
            acc.zero();
            int qh[2] = {0, 0}, qt[2] = {0, 0};
            int listed = s_listed[a];

            // consume queued pairs of queue qi (lanes < nq): exact FP64 separation from the
            // sorted positions, the reference test rsq <= rc^2, then the pair terms
            auto consume = [&](int qi, int nq) {
                __syncwarp();
                if constexpr (Pass::kStage == kStageF32Q) {
                    if (qi == 0) {
                        // far pairs: the FP32 screen placed them inside the cutoff with a
                        // margin far beyond its rounding; terms from the staged record
                        if (lane < nq) {
                            const int tq = s_q[warp][0][(qh[0] + lane) & 63];
                            const float4 p = s_pos[tq];
                            float dx = hx - p.x, dy = hy - p.y, dz = hz - p.z;
                            if (G.mi & 1) dx = foldf(dx, G.Lf0, G.hLf0);
                            if (G.mi & 2) dy = foldf(dy, G.Lf1, G.hLf1);
                            if (G.mi & 4) dz = foldf(dz, G.Lf2, G.hLf2);
                            const float rsq = dx * dx + dy * dy + dz * dz;
                            pass.pair32(acc, cx, dx, dy, dz, rsq, p.w, s_w[tq] & 15);
                        }
                        qh[0] += nq;
                        __syncwarp();
                        return;
                    }
                }
                bool ok = false;
                double dx = 0.0, dy = 0.0, dz = 0.0, rsq = 0.0;
                double4 pj = make_double4(0.0, 0.0, 0.0, 0.0);
                int j = 0;
                if (lane < nq) {
                    const int tq = s_q[warp][qi][(qh[qi] + lane) & 63];
                    if (Pass::kStage == kStageF32Q) {
                        // near pairs and pairs at the cutoff: FP64 from the sorted positions
                        const int tag = s_w[tq];
                        j = tag & 15;
                        pj = ldg4(&b.spos[tag >> 4]);
                        rsq = displacement(G, 7, hp.x, hp.y, hp.z, pj, dx, dy, dz);
                    } else if (Pass::kStage == kStageF64) {
                        j = s_w[tq];
                        pj = s_p64[tq];
                        rsq = displacement(G, G.mi, hp.x, hp.y, hp.z, pj, dx, dy, dz);
                    } else {
                        j = __float_as_int(s_pos[tq].w);
                        pj = ldg4(&b.spos[j]);
                        rsq = displacement(G, 7, hp.x, hp.y, hp.z, pj, dx, dy, dz);
                    }
                    ok = rsq <= rc2;
                    if (ok && rsq < 1.0e-16) {
                        set_status(st, AKMC_ERR_NONFINITE);
                        ok = false;
                    }
                }
                const unsigned okm = __ballot_sync(kFull, ok);
                if (ok) pass.pair(qi, acc, h, cx, dx, dy, dz, rsq, pj, j, listed + __popc(okm & lanemask_lt()));
                qh[qi] += nq;
                listed += __popc(okm);
                __syncwarp();
            };

            for (int base = 0; base < m; base += 32) {
                const int t = base + lane;
                int cls = -1;
                if (t < m && t != self_t) {
                    if (Pass::kStage == kStageF64) {
                        double dx, dy, dz;
                        const double rsq = displacement(G, G.mi, hp.x, hp.y, hp.z, s_p64[t], dx, dy, dz);
                        if (rsq <= rc2) cls = pass.classify((float)rsq);
                    } else {
                        const float4 p = s_pos[t];
                        float dx = hx - p.x, dy = hy - p.y, dz = hz - p.z;
                        if (G.mi & 1) dx = foldf(dx, G.Lf0, G.hLf0);
                        if (G.mi & 2) dy = foldf(dy, G.Lf1, G.hLf1);
                        if (G.mi & 4) dz = foldf(dz, G.Lf2, G.hLf2);
                        const float rsq = dx * dx + dy * dy + dz * dz;
                        if (Pass::kStage == kStageF32Q) cls = pass.classify(rsq);
                        else if (rsq <= rc2f) cls = pass.classify(rsq);
                    }
                }
                if (Pass::kQueues == 1) {
                    const unsigned bal = __ballot_sync(kFull, cls == 0);
                    if (cls == 0) s_q[warp][0][(qt[0] + __popc(bal & lanemask_lt())) & 63] = t;
                    qt[0] += __popc(bal);
                } else {
                    const unsigned bf = __ballot_sync(kFull, cls == 0);
                    const unsigned bn = __ballot_sync(kFull, cls == 1);
                    const unsigned lt = lanemask_lt();
                    if (cls == 0) s_q[warp][0][(qt[0] + __popc(bf & lt)) & 63] = t;
                    else if (cls == 1) s_q[warp][1][(qt[1] + __popc(bn & lt)) & 63] = t;
                    qt[0] += __popc(bf);
                    qt[1] += __popc(bn);
                }
                #pragma unroll
                for (int qi = 0; qi < Pass::kQueues; qi++)
                    if (qt[qi] - qh[qi] >= 32) consume(qi, 32);
            }
            #pragma unroll
            for (int qi = 0; qi < Pass::kQueues; qi++)
                if (qt[qi] > qh[qi]) consume(qi, qt[qi] - qh[qi]);
            double tot[Pass::kAcc];
            if (single) {
                // the whole neighbourhood was staged at once: finish this atom here with
                // one reduction
                pass.post(b, s, G, hp, h, cx, acc, reinterpret_cast<float2*>(&s_q[warp][0][0]));
                acc.reduce(tot);
                if (lane == 0) pass.finish(b, h, cx, tot, listed);
                continue;
            }
            acc.reduce(tot);
            if (lane == 0) {
                #pragma unroll
                for (int k = 0; k < Pass::kAcc; k++) s_acc[a][k] += tot[k];
                s_listed[a] = listed;
            }
        }
    }
    if (single) return;
    __syncthreads();

    for (int a = warp; a < it.count; a += kWarps) {
        const Home h{it.first + a, a0, st, it.first + a + lshift};
        const double4 hp = b.spos[h.i];
        const auto cx = pass.home(b, h);
        typename Pass::Acc acc;
        acc.zero();
        pass.post(b, s, G, hp, h, cx, acc, reinterpret_cast<float2*>(&s_q[warp][0][0]));
        double tot[Pass::kAcc];
        acc.reduce(tot);
        if (lane == 0) {
            #pragma unroll
            for (int k = 0; k < Pass::kAcc; k++) tot[k] += s_acc[a][k];
            pass.finish(b, h, cx, tot, s_listed[a]);
        }
    }
}

// kQueued: persistent CTAs over the call's queued items; otherwise one CTA per planned item
// (two instances, so the direct one carries no queue code in its registers)
template <class Pass, bool kQueued>
__global__ void __launch_bounds__(Pass::kThreads, Pass::kMinBlocks)
pair_kernel(BatchDev b, Pass pass, double rc2, int* status)
{
    // staged candidates (stage_cap of them): FP32 screen -> float4 {relative x, y, z, w};
    // FP64 screen -> double4 {x, y, z, q} (periodic shift applied) and int w
    extern __shared__ __align__(16) unsigned char s_dyn[];
    float4* s_pos = reinterpret_cast<float4*>(s_dyn);
    double4* s_p64 = reinterpret_cast<double4*>(s_dyn);
    int* s_w = Pass::kStage == kStageF64 ? reinterpret_cast<int*>(s_p64 + b.stage_cap)
                                         : reinterpret_cast<int*>(s_pos + b.stage_cap);
    constexpr int kWarps = Pass::kThreads / 32;
    __shared__ RangeSet rs;
    __shared__ int s_q[kWarps][2][64];
    static_assert(sizeof(s_q[0]) >= kWarpTab * sizeof(float2), "the phase table lives in a warp's queues");
    __shared__ double s_acc[kHomeChunk][Pass::kAcc];
    __shared__ int s_listed[kHomeChunk];
    __shared__ int s_ticket;

    // the ionic pass waits in its reciprocal loop (the only reader of its predecessor's
    // output); every other pass waits here
    if (!Pass::kOverlapPrior) pdl_wait();
    pdl_release();
    if (kQueued) {
        // persistent CTAs: queued items by ticket, until the queue is empty
        const int n_work = b.counters[0];
        for (;;) {
            if (threadIdx.x == 0) s_ticket = atomicAdd(b.ticket, 1);
            __syncthreads();
            const int q = s_ticket;
            if (q >= n_work) break;
            const WorkItem it = b.items[b.work[q]];
            pair_item(b, pass, rc2, status, it.sys, it, s_pos, s_p64, s_w, rs, s_q, s_acc, s_listed);
            __syncthreads();              // shared state is rebuilt by the next item
        }
        return;
    }
    const int s = find_system_by_item(b, blockIdx.x);
    const SysGeom& gref = b.geom[s];
    const int local = blockIdx.x - gref.item_base;
    if (local >= b.n_items[s]) return;
    const WorkItem it = b.items[gref.item_base + local];
    pair_item(b, pass, rc2, status, s, it, s_pos, s_p64, s_w, rs, s_q, s_acc, s_listed);
}


// ---------------------------------------------------------------------------------
// K4+K6 for whole-cell systems (mixed precision): fewer than three cells in every
// dimension, so every atom of the system is a candidate of every other under the minimum
// image -- the rocksalt workload (L = 21.05 A, cutoff 10 A) and every small ionic cell.
// ---------------------------------------------------------------------------------
// One CTA takes 32 home atoms of one system, one per lane, and stages the whole system in
// shared memory (FP32 coordinates and charge, species byte).  Its warps take the candidates
// interleaved (warp w: j = w, w + 8, ...), in chunks of kWcChunk, in two stages:
//   screen: each candidate is read by one broadcast load for the 32 home atoms of the warp;
//     every lane forms its FP32 minimum-image distance and appends j to its own list of far
//     pairs -- beyond the near radius and inside the cutoff by a relative 1e-5 of rc^2, far
//     beyond the FP32 squared distance's error -- or of near pairs (inside the near radius,
//     or within 1e-5 of the cutoff);
//   evaluate: every lane walks its own far list (the lists of a warp differ in length by a
//     few per cent) and evaluates the FP32 pair terms of accepted pairs only; forces and
//     energies are summed in FP32 over kWcFlush entries and then folded into FP64.
// Near pairs are evaluated in FP64 from the sorted FP64 positions with the exact test
// rsq <= rc^2 (the reference's criterion), whenever a lane's near list fills and at the
// end.  The warps' partials are added in warp order, and the reciprocal-space force
// follows, warp per home atom, as in the cell-scan pass.  Results are bitwise reproducible
// (fixed orders throughout).
// The four sums of energy_reduce_kernel in one pass (fixed order: warp shuffles, then the
// warps' totals in warp order), valid in thread 0.
__device__ void block_sum4(double* v, double (*sh)[32])
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    #pragma unroll
    for (int k = 0; k < 4; k++) {
        v[k] = warp_sum(v[k]);
        if (lane == 0) sh[k][warp] = v[k];
    }
    __syncthreads();
    if (warp == 0) {
        #pragma unroll
        for (int k = 0; k < 4; k++) v[k] = warp_sum(lane < (int)(blockDim.x >> 5) ? sh[k][lane] : 0.0);
    }
}

constexpr int kWcWarps = 8;
constexpr int kWcNear = 16;          // listed near pairs per lane and warp before a flush
constexpr int kWcFlush = 8;          // pairs per FP32 partial
constexpr int kWcChunk = 128;        // candidates a warp screens before evaluating its lanes' lists
constexpr int kWcPer = 32 / kWcWarps;  // home atoms per warp in the reciprocal part
// 2 CTAs of 8 warps per SM (measured faster than 4 smaller ones: with 32-candidate chunks the
// lanes' list lengths differ more, relative to their means)
static_assert(kWcChunk * 32 * sizeof(unsigned short) >= 5 * 32 * sizeof(double),
              "a warp's far lists hold its partial sums at the end");

__global__ void __launch_bounds__(kWcWarps * 32, 2)
ionic_whole_cell_kernel(BatchDev b, IonicPass<false> pass, double rc2, int* status, double* energy)
{
    extern __shared__ __align__(16) unsigned char s_dyn[];
    __shared__ unsigned short s_near[kWcWarps][kWcNear][32];
    __shared__ float2 s_tab[kWcWarps][kWcPer][kWarpTab];
    __shared__ float4 s_buck[kMaxSpecies * kMaxSpecies];    // {A, 1/rho, C} per species pair
    pdl_release();                    // the sorted positions are complete (see the structure factor)
    const int s = blockIdx.y;
    if (!system_active(b, s)) return;
    const SysGeom& gref = b.geom[s];
    const int n = gref.n_atoms, a0 = gref.atom_begin;
    const int tile0 = blockIdx.x * 32;
    if (tile0 >= n) return;
    const IonicDev& P = pass.P;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    float4* s_pos = reinterpret_cast<float4*>(s_dyn);                       // x, y, z, charge
    unsigned char* s_lab = reinterpret_cast<unsigned char*>(s_pos + b.whole_cell_n);
    // far lists: entry e of lane l of warp w at s_far[(w * kWcChunk + e) * 32 + l]
    unsigned short* s_far = reinterpret_cast<unsigned short*>(s_lab + ((b.whole_cell_n + 15) & ~15));
    // stage the system: four records per thread in flight at a time
    for (int j0 = tid; j0 < n; j0 += 4 * blockDim.x) {
        double4 p[4];
        int l[4];
        #pragma unroll
        for (int u = 0; u < 4; u++) {
            const int j = j0 + u * blockDim.x;
            if (j < n) {
                p[u] = b.spos[a0 + j];
                l[u] = b.slabel[a0 + j];
            }
        }
        #pragma unroll
        for (int u = 0; u < 4; u++) {
            const int j = j0 + u * blockDim.x;
            if (j < n) {
                s_pos[j] = make_float4((float)p[u].x, (float)p[u].y, (float)p[u].z, (float)p[u].w);
                s_lab[j] = (unsigned char)l[u];
            }
        }
    }
    for (int k = tid; k < kMaxSpecies * kMaxSpecies; k += blockDim.x) s_buck[k] = pass.buck32(k);
    __syncthreads();

    const Geo G = make_geo(gref, 7);
    int* st = status + s;
    const bool mine = tile0 + lane < n;
    const int il = mine ? tile0 + lane : n - 1;       // lanes past the end repeat the last atom
    const float4 hp = s_pos[il];
    const int li = s_lab[il];
    const double qi = b.spos[a0 + il].w;
    const float cqf = (float)(P.cfact * qi);
    const IonicPass<false>::Ctx cx{li, P.cfact * qi, cqf, qi};
    const float rs2 = fmaxf(pass.r_split2f, 1.0e-12f);
    const float rc2_lo = pass.rc2_lo, rc2_hi = pass.rc2_hi;
    const int abase = li * P.ns;

    IonicAcc acc;                     // FP64 totals of the lane's home atom: fx, fy, fz, E_real, E_vdw
    acc.zero();
    int nn = 0;

    // the listed near pairs of this lane, in FP64 (queue 1 of the cell-scan pass)
    auto near_flush = [&]() {
        const int rounds = __reduce_max_sync(kFull, nn);
        if (rounds == 0) return;
        const double4 h64 = b.spos[a0 + il];
        for (int k = 0; k < rounds; k++) {
            if (k < nn) {
                const int j = s_near[warp][k][lane];
                if (AKMC_BAD(j >= n, 12, j)) continue;
                const double4 pj = ldg4(&b.spos[a0 + j]);
                double dx, dy, dz;
                const double rsq = displacement(G, 7, h64.x, h64.y, h64.z, pj, dx, dy, dz);
                if (rsq <= rc2) {
                    if (rsq < 1.0e-16) {
                        if (mine) set_status(st, AKMC_ERR_NONFINITE);
                    } else {
                        const Home h{a0 + il, a0, st, a0 + il};
                        pass.pair(1, acc, h, cx, dx, dy, dz, rsq, pj, s_lab[j], 0);
                    }
                }
            }
        }
        nn = 0;
        __syncwarp();
    };

    unsigned short* my_far = s_far + (size_t)warp * kWcChunk * 32 + lane;
    for (int m0 = 0; warp + kWcWarps * m0 < n; m0 += kWcChunk) {
        // screen a chunk: far pairs to this lane's far list, near pairs to its near list
        int nf = 0;
        for (int u0 = 0; u0 < kWcChunk; u0 += kWcFlush) {
            if (__any_sync(kFull, nn > kWcNear - kWcFlush)) near_flush();
            #pragma unroll
            for (int u = 0; u < kWcFlush; u++) {
                const int j = warp + kWcWarps * (m0 + u0 + u);
                const bool in = j < n;
                const float4 pj = s_pos[in ? j : il];
                const float dx = foldf(hp.x - pj.x, G.Lf0, G.hLf0);
                const float dy = foldf(hp.y - pj.y, G.Lf1, G.hLf1);
                const float dz = foldf(hp.z - pj.z, G.Lf2, G.hLf2);
                const float rsq = dx * dx + dy * dy + dz * dz;
                const bool far = in && rsq >= rs2 && rsq <= rc2_lo;
                if (far) my_far[32 * nf++] = (unsigned short)j;
                if (in && !far && rsq <= rc2_hi && j != il) s_near[warp][nn++][lane] = (unsigned short)j;
            }
        }
        __syncwarp();
        // evaluate this lane's far pairs; lanes past their list's end compute a masked self pair
        const int rounds = __reduce_max_sync(kFull, nf);
        for (int e0 = 0; e0 < rounds; e0 += kWcFlush) {
            float px = 0.f, py = 0.f, pz = 0.f, pr = 0.f, pv = 0.f;
            #pragma unroll
            for (int u = 0; u < kWcFlush; u++) {
                const bool ok = e0 + u < nf;
                const int j = ok ? my_far[32 * (e0 + u)] : il;
                const float4 pj = s_pos[j];
                const int lj = s_lab[j];
                const float dx = foldf(hp.x - pj.x, G.Lf0, G.hLf0);
                const float dy = foldf(hp.y - pj.y, G.Lf1, G.hLf1);
                const float dz = foldf(hp.z - pj.z, G.Lf2, G.hLf2);
                const float rsq = dx * dx + dy * dy + dz * dz;
                float forc, eng, evdw;
                pass.terms32(s_buck[abase + lj], cqf, pj.w, rsq, forc, eng, evdw);
                if (!ok) { forc = 0.f; eng = 0.f; evdw = 0.f; }
                px = fmaf(-forc, dx, px);
                py = fmaf(-forc, dy, py);
                pz = fmaf(-forc, dz, pz);
                pr += eng;
                pv += evdw;
            }
            acc.v[0] += (double)px; acc.v[1] += (double)py; acc.v[2] += (double)pz;
            acc.v[3] += 0.5 * (double)pr; acc.v[4] += 0.5 * (double)pv;
        }
        __syncwarp();
    }
    near_flush();

    // the warp's partial sums, in its own far-list space (no longer needed)
    double* my_part = reinterpret_cast<double*>(s_far + (size_t)warp * kWcChunk * 32);
    #pragma unroll
    for (int k = 0; k < 5; k++) my_part[k * 32 + lane] = acc.v[k];
    __syncthreads();

    // reciprocal space: each warp takes its kWcPer home atoms a = warp + 8 j together, lanes
    // over k, so that every k-vector's record and C_k, S_k are read once for all of them
    if (P.ntab <= kWarpTab) {
        const int oy = P.gx + 1, oz = oy + 2 * P.gy + 1;
        // phase tables e^{2 pi i n s_d}: one FP64 sincospi per (atom, dimension), the other
        // entries by the angle-addition recurrence in FP64, negative n as conjugates
        if (lane < 3 * kWcPer) {
            const int j = lane / 3, d = lane - 3 * j, a = warp + kWcWarps * j;
            if (tile0 + a < n) {
                const double4 h64 = b.spos[a0 + tile0 + a];
                const double u = d == 0 ? h64.x * G.iL0 : d == 1 ? h64.y * G.iL1 : h64.z * G.iL2;
                double sn, cn;
                sincospi(2.0 * u, &sn, &cn);
                const double2 w = make_double2(cn, sn);
                const int zero = d == 0 ? 0 : d == 1 ? oy + P.gy : oz + P.gz;
                const int top = d == 0 ? P.gx : d == 1 ? P.gy : P.gz;
                float2* row = s_tab[warp][j];
                double2 e = make_double2(1.0, 0.0);
                row[zero] = make_float2(1.0f, 0.0f);
                for (int m = 1; m <= top; m++) {
                    e = cmul(e, w);
                    row[zero + m] = make_float2((float)e.x, (float)e.y);
                    if (d != 0) row[zero - m] = make_float2((float)e.x, -(float)e.y);
                }
            }
        }
        __syncwarp();
        wait_for_prior_grid();                // C_k, S_k come from the structure-factor kernel
        const float2* skk = pass.skf + (size_t)s * P.nk;
        float qf[kWcPer], ax[kWcPer], ay[kWcPer], az[kWcPer];
        #pragma unroll
        for (int j = 0; j < kWcPer; j++) {
            const int a = warp + kWcWarps * j;
            qf[j] = tile0 + a < n ? (float)b.spos[a0 + tile0 + a].w : 0.0f;
            ax[j] = ay[j] = az[j] = 0.0f;
        }
        for (int k = lane; k < P.nk; k += 32) {
            const int4 t = __ldg(&P.kt[k]);
            const float4 kf = __ldg(&P.kf[k]);
            const float2 cs = skk[k];
            #pragma unroll
            for (int j = 0; j < kWcPer; j++) {
                const float2 X = s_tab[warp][j][t.x], Y = s_tab[warp][j][t.y], Z = s_tab[warp][j][t.z];
                const float xyr = X.x * Y.x - X.y * Y.y, xyi = X.x * Y.y + X.y * Y.x;
                const float cn = xyr * Z.x - xyi * Z.y, sn = xyr * Z.y + xyi * Z.x;
                const float pf = kf.w * qf[j] * (sn * cs.x - cn * cs.y);
                ax[j] += pf * kf.x;
                ay[j] += pf * kf.y;
                az[j] += pf * kf.z;
            }
        }
        #pragma unroll
        for (int j = 0; j < kWcPer; j++) {
            const int a = warp + kWcWarps * j;
            double tot[5];
            tot[0] = warp_sum((double)ax[j] * kTwoPi * G.iL0);
            tot[1] = warp_sum((double)ay[j] * kTwoPi * G.iL1);
            tot[2] = warp_sum((double)az[j] * kTwoPi * G.iL2);
            tot[3] = tot[4] = 0.0;
            if (lane == 0 && tile0 + a < n) {
                const int i = a0 + tile0 + a;
                const double q = b.spos[i].w;
                const IonicPass<false>::Ctx ca{s_lab[tile0 + a], P.cfact * q, (float)(P.cfact * q), q};
                const Home h{i, a0, st, i};
                #pragma unroll
                for (int k = 0; k < 5; k++) {
                    double v = 0.0;
                    #pragma unroll
                    for (int w = 0; w < kWcWarps; w++)
                        v += reinterpret_cast<const double*>(s_far + (size_t)w * kWcChunk * 32)[k * 32 + a];
                    tot[k] += v;
                }
                pass.finish(b, h, ca, tot, 0);
            }
        }
    } else {
        // larger k-sets: warp per home atom, as in the cell-scan pass
        for (int a = warp; a < 32 && tile0 + a < n; a += kWcWarps) {
            const int i = a0 + tile0 + a;
            const double4 h64 = b.spos[i];
            const IonicPass<false>::Ctx ca{s_lab[tile0 + a], P.cfact * h64.w, (float)(P.cfact * h64.w), h64.w};
            const Home h{i, a0, st, i};
            IonicAcc r;
            r.zero();
            pass.post(b, s, G, h64, h, ca, r, s_tab[warp][0]);
            double tot[5];
            r.reduce(tot);
            if (lane == 0) {
                #pragma unroll
                for (int k = 0; k < 5; k++) {
                    double v = 0.0;
                    #pragma unroll
                    for (int w = 0; w < kWcWarps; w++)
                        v += reinterpret_cast<const double*>(s_far + (size_t)w * kWcChunk * 32)[k * 32 + a];
                    tot[k] += v;
                }
                pass.finish(b, h, ca, tot, 0);
            }
        }
    }
    // the system's energy record, by its last CTA to finish (energy_reduce_kernel's sums, in
    // the same fixed order)
    if (energy == nullptr) return;
    __shared__ int s_ticket;
    __shared__ double s_red[4][32];
    __threadfence();
    __syncthreads();
    if (tid == 0) s_ticket = atomicAdd(&b.wc_counter[s], 1);
    __syncthreads();
    if (s_ticket != (n + 31) / 32 - 1) return;
    __threadfence();
    double v[4] = {0.0, 0.0, 0.0, 0.0};          // E_real, E_vdw, reciprocal sum, self term
    for (int i = tid; i < n; i += blockDim.x) {
        const double2 e = __ldcg(&b.eatom[a0 + i]);
        v[0] += e.x;
        v[1] += e.y;
        const double q = b.charge[a0 + i];
        v[3] += -kTwoOverRootPi * (0.5 * P.cfact * q * q) * P.eta;
    }
    for (int k = tid; k < P.nk; k += blockDim.x) {
        const double2 cs = b.sk[(size_t)s * P.nk + k];
        v[2] += P.g0[k] * (cs.x * cs.x + cs.y * cs.y);
    }
    block_sum4(v, s_red);
    if (tid == 0) {
        const double rcp = 0.5 * v[2], real = v[0] + v[3], vdw = v[1];
        double* out = energy + 5 * (size_t)s;
        out[0] = rcp + real + vdw;
        out[1] = rcp;
        out[2] = real;
        out[3] = vdw;
        out[4] = 0.0;
        b.wc_counter[s] = 0;
    }
}

// ---------------------------------------------------------------------------------
// K3 (list): EAM force, one thread per atom over the density pass's neighbour list
// ---------------------------------------------------------------------------------
constexpr int kListThreads = 128;
static_assert(kListThreads == kChunkAtoms, "a queued chunk is one CTA's atoms");

// An atom's list entries are summed in kParts partial sums -- entry k into partial k mod 4,
// each in list order -- combined as (p0 + p1) + (p2 + p3).  A call with many queued atoms gives
// every atom one thread, which keeps the four partials; a call with few (a handful of walkers
// still running) gives every atom four lanes, lane u keeping partial u, so that the atom's
// chain of dependent gathers is a quarter of its list -- with the same sums bit for bit.
constexpr int kParts = 4;

__device__ __forceinline__ double combine_parts(double p0, double p1, double p2, double p3)
{
    return (p0 + p1) + (p2 + p3);
}

// Wide mode: the four lanes of the atom hold p0..p3; every one of them gets the combined sum.
__device__ __forceinline__ double combine_lanes(double v)
{
    const unsigned m = 0xFu << ((threadIdx.x & 31) & ~(kParts - 1));
    v += __shfl_xor_sync(m, v, 1);
    v += __shfl_xor_sync(m, v, 2);
    return v;
}

// f(system, sorted atom, lane, wide) for the atoms of this call's queued chunks, or for every
// atom of a running system of the batch.  Wide (queued chunks x 4 <= CTAs of the launch): CTA c
// takes quarter c % 4 of chunk c / 4, four lanes per atom; otherwise persistent CTAs take whole
// chunks by stride, one thread per atom (lane 0).
template <class F>
__device__ __forceinline__ void for_each_queued_atom(const BatchDev& b, F&& f)
{
    if (b.chunks) {
        const int nch = b.counters[1];
        if (kParts * nch <= (int)gridDim.x) {
            const int c = blockIdx.x / kParts, q = blockIdx.x % kParts;
            if (c >= nch) return;
            const int2 ch = b.chunks[c];
            const SysGeom& g = b.geom[ch.x];
            const int local = ch.y + q * (kChunkAtoms / kParts) + (int)threadIdx.x / kParts;
            if (local < g.n_atoms) f(ch.x, g.atom_begin + local, (int)threadIdx.x % kParts, true);
            return;
        }
        for (int c = blockIdx.x; c < nch; c += gridDim.x) {
            const int2 ch = b.chunks[c];
            const SysGeom& g = b.geom[ch.x];
            const int local = ch.y + threadIdx.x;
            if (local < g.n_atoms) f(ch.x, g.atom_begin + local, 0, false);
        }
        return;
    }
    const int i = blockIdx.x * kListThreads + threadIdx.x;
    if (i >= b.n_total) return;
    const int s = find_system_by_atom(b, i);
    if (system_active(b, s)) f(s, i, 0, false);
}

// Walks the list entries of one atom for one thread: narrow, every entry, entry k into partial
// k mod 4 (term(u, j)); wide, the entries k = lane, lane + 4, ... into partial 0.  Gathers of
// four entries are in flight together.
// Sorted index of list entry k of a row (a0: the system's first atom, n: its atom count).
__device__ __forceinline__ int list_entry(const unsigned short* row, size_t st, int k, int a0, int n)
{
    int j = row[(size_t)k * st];
    if (AKMC_BAD(j >= n, 4, j)) j = 0;
    return a0 + j;
}

template <class Term>
__device__ __forceinline__ void walk_list(const BatchDev& b, const unsigned short* row, int a0, int n, int cnt,
                                          int lane, bool wide, Term&& term)
{
    const size_t st = b.n_total;
    if (AKMC_BAD(cnt < 0 || cnt > b.nbr_cap, 3, cnt)) return;
    if (wide) {
        int k = lane;
        for (; k + 3 * kParts < cnt; k += 4 * kParts) {
            int j[4];
            #pragma unroll
            for (int u = 0; u < 4; u++) j[u] = list_entry(row, st, k + u * kParts, a0, n);
            term.gather4(j);
            #pragma unroll
            for (int u = 0; u < 4; u++) term.add(0, u);
        }
        for (; k < cnt; k += kParts) term.single(0, list_entry(row, st, k, a0, n));
        return;
    }
    int k = 0;
    for (; k + 4 <= cnt; k += 4) {
        int j[4];
        #pragma unroll
        for (int u = 0; u < 4; u++) j[u] = list_entry(row, st, k + u, a0, n);
        term.gather4(j);
        #pragma unroll
        for (int u = 0; u < 4; u++) term.add(u, u);
    }
    if (k < cnt) term.single(0, list_entry(row, st, k, a0, n));
    if (k + 1 < cnt) term.single(1, list_entry(row, st, k + 1, a0, n));
    if (k + 2 < cnt) term.single(2, list_entry(row, st, k + 2, a0, n));
}

// kMulti: the field holds several EAM tables (an alloy): the pair's table per pair, and the
// records carry densities; otherwise table 0 and F' records.
template <bool kFp64, bool kMulti>
struct ForceTerms {
    const BatchDev& b;
    const EamDev& P;
    const Geo& G;
    double rc2, fpi;
    double4 hp;
    int li;
    bool one_species, mbi;
    int* st;
    double fx[kParts], fy[kParts], fz[kParts], ep[kParts];
    double4 rj[4];
    int lj[4];
    __device__ void gather4(const int (&j)[4])
    {
        #pragma unroll
        for (int u = 0; u < 4; u++) rj[u] = b.frec[j[u]];
        #pragma unroll
        for (int u = 0; u < 4; u++) lj[u] = one_species ? 0 : b.slabel[j[u]];
    }
    // rec: the neighbour's {x, y, z, F'} record (F' NaN: its density is below 1e-8)
    __device__ __forceinline__ void term(int p, const double4& rec, int l)
    {
        if (!P.pair_ok[li * P.ns + l]) return;
        double dx, dy, dz;
        const double rsq = displacement(G, 7, hp.x, hp.y, hp.z, rec, dx, dy, dz);
        if (!(rsq <= rc2)) return;
        double gg, phi;
        const bool mb = mbi && !isnan(rec.w);
        const int k = kMulti ? P.mesh[li * P.ns + l] : 0;
        // records carry F' (one table) or the density (several: F' from the pair's table)
        const double fps = !mb ? 0.0 : kMulti ? eam_dembed(P, k, fpi, st) + eam_dembed(P, k, rec.w, st)
                                              : fpi + rec.w;
        if (!eam_pair_term_mb<kFp64>(P, k, rsq, mb, fps, st, gg, phi)) return;
        fx[p] = fma(-gg, dx, fx[p]);
        fy[p] = fma(-gg, dy, fy[p]);
        fz[p] = fma(-gg, dz, fz[p]);
        ep[p] = fma(0.5, phi, ep[p]);
    }
    __device__ __forceinline__ void add(int p, int u) { term(p, rj[u], lj[u]); }
    __device__ __forceinline__ void single(int p, int j) { term(p, b.frec[j], one_species ? 0 : b.slabel[j]); }
};

template <bool kFp64, bool kMulti>
__device__ __forceinline__ void eam_force_list_atom(const BatchDev& b, const EamDev& P, double rc2,
                                                    double* __restrict__ force, int* __restrict__ status,
                                                    int s, int i, int lane, bool wide)
{
    const SysGeom& g = b.geom[s];
    const Geo G = make_geo(g, 7);             // positions are wrapped: fold every dimension
    // its own {x, y, z, F'} record (F' NaN below the density floor), the one its neighbours gather
    const double4 h = b.frec[i];
    const int il = i + list_shift(b, s);     // its list row
    ForceTerms<kFp64, kMulti> t{b, P, G, rc2, h.w, h, b.slabel[i], P.ns == 1, !isnan(h.w), status + s};
    #pragma unroll
    for (int p = 0; p < kParts; p++) t.fx[p] = t.fy[p] = t.fz[p] = t.ep[p] = 0.0;
    if (AKMC_BAD(il < 0 || il >= b.n_total, 2, il)) return;
    walk_list(b, b.nbr + il, g.atom_begin, g.n_atoms, b.nbr_count[il], lane, wide, t);
    double fx, fy, fz, ep;
    if (wide) {
        fx = combine_lanes(t.fx[0]);
        fy = combine_lanes(t.fy[0]);
        fz = combine_lanes(t.fz[0]);
        ep = combine_lanes(t.ep[0]);
        if (lane != 0) return;
    } else {
        fx = combine_parts(t.fx[0], t.fx[1], t.fx[2], t.fx[3]);
        fy = combine_parts(t.fy[0], t.fy[1], t.fy[2], t.fy[3]);
        fz = combine_parts(t.fz[0], t.fz[1], t.fz[2], t.fz[3]);
        ep = combine_parts(t.ep[0], t.ep[1], t.ep[2], t.ep[3]);
    }
    const int o = b.perm[i];
    if (AKMC_BAD(o < 0 || o >= b.n_total, 5, o)) return;
    force[3 * (size_t)o + 0] = fx;
    force[3 * (size_t)o + 1] = fy;
    force[3 * (size_t)o + 2] = fz;
    b.eatom[i].y = ep;
}

template <bool kFp64, bool kMulti>
__global__ void __launch_bounds__(kListThreads)
eam_force_list_kernel(BatchDev b, EamDev P, double rc2, double* __restrict__ force,
                      int* __restrict__ status)
{
    pdl_wait();
    pdl_release();
    for_each_queued_atom(b, [&](int s, int i, int lane, bool wide) {
        eam_force_list_atom<kFp64, kMulti>(b, P, rc2, force, status, s, i, lane, wide);
    });
}

template <bool kFp64>
struct DensityTerms {
    const BatchDev& b;
    const EamDev& P;
    const Geo& G;
    double rc2;
    double4 hp;
    int* st;
    double rho[kParts];
    double4 pj[4];
    __device__ void gather4(const int (&j)[4])
    {
        #pragma unroll
        for (int u = 0; u < 4; u++) pj[u] = b.spos[j[u]];
    }
    __device__ __forceinline__ void term(int p, const double4& q)
    {
        double dx, dy, dz;
        const double rsq = displacement(G, 7, hp.x, hp.y, hp.z, q, dx, dy, dz);
        if (!(rsq <= rc2)) return;
        if (rsq < 1.0e-16) {
            set_status(st, AKMC_ERR_NONFINITE);
            return;
        }
        rho[p] += eam_rho_term<kFp64>(P, rsq, (int)q.w, st);
    }
    __device__ __forceinline__ void add(int p, int u) { term(p, pj[u]); }
    __device__ __forceinline__ void single(int p, int j) { term(p, b.spos[j]); }
};

// K2 on a reused list (systems with list_mode 2): rho_i over the list entries within the
// cutoff, then the embedding.
template <bool kFp64>
__device__ __forceinline__ void eam_density_list_atom(const BatchDev& b, const EamDev& P, double rc2,
                                                      int* __restrict__ status, int s, int i, int lane,
                                                      bool wide)
{
    if (b.list_mode[s] != 2) return;
    const SysGeom& g = b.geom[s];
    const Geo G = make_geo(g, 7);
    const double4 hp = b.spos[i];
    const int il = i + list_shift(b, s);     // its list row
    DensityTerms<kFp64> t{b, P, G, rc2, hp, status + s};
    #pragma unroll
    for (int p = 0; p < kParts; p++) t.rho[p] = 0.0;
    if (AKMC_BAD(il < 0 || il >= b.n_total, 2, il)) return;
    walk_list(b, b.nbr + il, g.atom_begin, g.n_atoms, b.nbr_count[il], lane, wide, t);
    double rho;
    if (wide) {
        rho = combine_lanes(t.rho[0]);
        if (lane != 0) return;
    } else {
        rho = combine_parts(t.rho[0], t.rho[1], t.rho[2], t.rho[3]);
    }
    eam_embed(P, b.slabel[i], rho, i, status + s, b.sextra, b.eatom, b.frec, hp);
}

template <bool kFp64>
__global__ void __launch_bounds__(kListThreads)
eam_density_list_kernel(BatchDev b, EamDev P, double rc2, int* __restrict__ status)
{
    pdl_wait();
    pdl_release();
    for_each_queued_atom(b, [&](int s, int i, int lane, bool wide) {
        eam_density_list_atom<kFp64>(b, P, rc2, status, s, i, lane, wide);
    });
}

// ---------------------------------------------------------------------------------
// K5: structure factors, grid (k tiles, atom chunks, systems)
// ---------------------------------------------------------------------------------
template <bool kFp64>
__global__ void __launch_bounds__(kSkThreads)
structure_factor_kernel(BatchDev b, IonicDev P)
{
    __shared__ double4 s_at[kSkAtomChunk];
    __shared__ int s_ticket;
    pdl_wait();                    // sorted positions come from the cell kernel
    pdl_release();                 // the ionic force kernel may start its real-space part
    const int s = blockIdx.z, chunk = blockIdx.y, tile = blockIdx.x;
    if (!system_active(b, s)) return;        // uniform per system: no chunk takes a ticket
    const SysGeom& g = b.geom[s];
    const int a_begin = g.atom_begin + chunk * kSkAtomChunk;
    const int a_end = min(g.atom_begin + g.n_atoms, a_begin + kSkAtomChunk);
    const int na = max(0, a_end - a_begin);
    for (int t = threadIdx.x; t < na; t += blockDim.x) {
        const double4 p = b.spos[a_begin + t];
        s_at[t] = make_double4(p.x * g.invL[0], p.y * g.invL[1], p.z * g.invL[2], p.w);
    }
    __syncthreads();
    const int k = tile * kSkThreads + threadIdx.x;
    const int nk = P.nk;
    if (k < nk) {
        const double4 kd = ldg4(&P.kd[k]);
        double C = 0.0, S = 0.0;
        for (int j = 0; j < na; j++) {
            const double4 a = s_at[j];
            const double u = frac_nearest(kd.x * a.x + kd.y * a.y + kd.z * a.z);
            if (kFp64) {
                double sn, cn;
                sincospi(2.0 * u, &sn, &cn);
                C += a.w * cn;
                S += a.w * sn;
            } else {
                float sf, cf;
                sincospif(2.0f * (float)u, &sf, &cf);
                C += a.w * (double)cf;
                S += a.w * (double)sf;
            }
        }
        b.skpart[((size_t)s * b.sk_chunks + chunk) * nk + k] = make_double2(C, S);
    }
    // the last chunk to arrive for this (system, tile) sums the chunks in fixed order
    __threadfence();
    __syncthreads();
    const int ntiles = gridDim.x;
    int* counter = b.sk_counter + (size_t)s * ntiles + tile;
    if (threadIdx.x == 0) s_ticket = atomicAdd(counter, 1);
    __syncthreads();
    if (s_ticket == b.sk_chunks - 1) {
        __threadfence();
        if (k < nk) {
            double C = 0.0, S = 0.0;
            for (int c = 0; c < b.sk_chunks; c++) {
                const double2 v = __ldcg(&b.skpart[((size_t)s * b.sk_chunks + c) * nk + k]);
                C += v.x;
                S += v.y;
            }
            b.sk[(size_t)s * nk + k] = make_double2(C, S);
            b.skf[(size_t)s * nk + k] = make_float2((float)C, (float)S);
        }
        if (threadIdx.x == 0) *counter = 0;
    }
}

// K5 with phase tables (mixed precision): grid (atom chunks, systems).  The CTA
// tabulates e^{2 pi i n s_d} for its kSkAtomChunk atoms: one FP64 sincospi per atom and
// dimension, the other entries by the angle-addition recurrence e^{i(n+1)t} = e^{int} e^{it}
// (at most a dozen complex products, a few 1e-16 of drift), negative n as conjugates.  Then
// each four threads take a group of up to kSkGroup k-vectors of one (nx, ny) column, each
// thread a quarter of the chunk's atoms: per atom the X.Y product once, times the charge, then
// one Z entry and four FP64 FMAs per k-vector (FP64 terms: an FP32 phase per atom would put
// ~1e-5 of error into C_k and S_k, the sum of ~1000 terms, each rounded, and a few 1e-6 eV/A
// into every atom's force).  The four quarters are added by shuffles, (0 + 1) + (2 + 3).
// The last chunk of a system to finish sums the chunk partials in fixed order.
constexpr int kSkTabThreads = 640;     // 160 groups per pass, four threads each
constexpr int kMaxSkTable = 96;        // 64 atoms x 96 entries x 16 B = 96 KB of tables

__global__ void __launch_bounds__(kSkTabThreads)
structure_factor_tab_kernel(BatchDev b, IonicDev P)
{
    extern __shared__ __align__(16) double2 s_tab[];      // [kSkAtomChunk][ntab]
    __shared__ double s_q[kSkAtomChunk];
    __shared__ int s_ticket;
    pdl_wait();                    // sorted positions come from the cell kernel
    pdl_release();                 // the ionic force kernel may start its real-space part
    const int s = blockIdx.y, chunk = blockIdx.x;
    if (!system_active(b, s)) return;        // uniform per system: no chunk takes a ticket
    const SysGeom& g = b.geom[s];
    const int a_begin = g.atom_begin + chunk * kSkAtomChunk;
    const int a_end = min(g.atom_begin + g.n_atoms, a_begin + kSkAtomChunk);
    const int na = max(0, a_end - a_begin);
    const int nt = P.ntab, oy = P.gx + 1, oz = oy + 2 * P.gy + 1;
    for (int idx = threadIdx.x; idx < na * 3; idx += blockDim.x) {
        const int a = idx / 3, d = idx - 3 * a;
        const double4 p = b.spos[a_begin + a];
        const double u = d == 0 ? p.x * g.invL[0] : d == 1 ? p.y * g.invL[1] : p.z * g.invL[2];
        double sn, cn;
        sincospi(2.0 * u, &sn, &cn);
        const double2 w = make_double2(cn, sn);
        double2* row = s_tab + a * nt;
        const int zero = d == 0 ? 0 : d == 1 ? oy + P.gy : oz + P.gz;     // slot of n = 0
        const int top = d == 0 ? P.gx : d == 1 ? P.gy : P.gz;
        double2 e = make_double2(1.0, 0.0);
        row[zero] = e;
        for (int m = 1; m <= top; m++) {
            e = cmul(e, w);
            row[zero + m] = e;
            if (d != 0) row[zero - m] = make_double2(e.x, -e.y);
        }
        if (d == 0) s_q[a] = p.w;
    }
    __syncthreads();
    const int nk = P.nk, part = threadIdx.x & 3, groups = blockDim.x >> 2;
    for (int g0 = 0; g0 < P.ngrp; g0 += groups) {
        const int gi = g0 + (threadIdx.x >> 2);
        const bool on = gi < P.ngrp;
        const int4 gr = on ? __ldg(&P.kgrp[gi]) : make_int4(0, 0, 0, 0);
        const int cnt = gr.y, tx = gr.z & 0xffff, ty = gr.z >> 16, tz = gr.w;
        double C[kSkGroup], S[kSkGroup];
        #pragma unroll
        for (int r = 0; r < kSkGroup; r++) C[r] = S[r] = 0.0;
        if (on) {
            for (int a = part; a < na; a += 4) {
                const double2* row = s_tab + a * nt;
                const double2 xy = cmul(row[tx], row[ty]);
                const double q = s_q[a];
                const double pr = q * xy.x, pi = q * xy.y;
                #pragma unroll
                for (int r = 0; r < kSkGroup; r++) {
                    if (r < cnt) {
                        const double2 Z = row[tz + r];
                        C[r] = fma(pr, Z.x, C[r]);
                        C[r] = fma(-pi, Z.y, C[r]);
                        S[r] = fma(pr, Z.y, S[r]);
                        S[r] = fma(pi, Z.x, S[r]);
                    }
                }
            }
        }
        #pragma unroll
        for (int r = 0; r < kSkGroup; r++) {
            C[r] += __shfl_xor_sync(kFull, C[r], 1);
            S[r] += __shfl_xor_sync(kFull, S[r], 1);
            C[r] += __shfl_xor_sync(kFull, C[r], 2);
            S[r] += __shfl_xor_sync(kFull, S[r], 2);
        }
        if (on && part == 0) {
            #pragma unroll
            for (int r = 0; r < kSkGroup; r++)
                if (r < cnt) b.skpart[((size_t)s * b.sk_chunks + chunk) * nk + gr.x + r] = make_double2(C[r], S[r]);
        }
    }
    __threadfence();
    __syncthreads();
    int* counter = b.sk_counter + (size_t)s;
    if (threadIdx.x == 0) s_ticket = atomicAdd(counter, 1);
    __syncthreads();
    if (s_ticket == gridDim.x - 1) {
        __threadfence();
        for (int k = threadIdx.x; k < nk; k += blockDim.x) {
            double C = 0.0, S = 0.0;
            for (int c = 0; c < (int)gridDim.x; c++) {
                const double2 v = __ldcg(&b.skpart[((size_t)s * b.sk_chunks + c) * nk + k]);
                C += v.x;
                S += v.y;
            }
            b.sk[(size_t)s * nk + k] = make_double2(C, S);
            b.skf[(size_t)s * nk + k] = make_float2((float)C, (float)S);
        }
        if (threadIdx.x == 0) *counter = 0;
    }
}

// ---------------------------------------------------------------------------------
// K7: per-system energies in a fixed summation order
// ---------------------------------------------------------------------------------
constexpr int kReduceThreads = 256;

__global__ void __launch_bounds__(kReduceThreads)
energy_reduce_kernel(BatchDev b, int family, IonicDev P, double* energy)
{
    __shared__ double sh[4][32];
    pdl_wait();
    pdl_release();
    const int s = blockIdx.x;
    if (!system_active(b, s)) return;
    const SysGeom& g = b.geom[s];
    double e0 = 0.0, e1 = 0.0, erc = 0.0, eself = 0.0;
    for (int i = threadIdx.x; i < g.n_atoms; i += blockDim.x) {
        const double2 e = b.eatom[g.atom_begin + i];
        e0 += e.x;
        e1 += e.y;
        if (family == AKMC_FAMILY_IONIC) {
            const double q = b.charge[g.atom_begin + i];
            eself += -kTwoOverRootPi * (0.5 * P.cfact * q * q) * P.eta;
        }
    }
    if (family == AKMC_FAMILY_IONIC) {
        for (int k = threadIdx.x; k < P.nk; k += blockDim.x) {
            const double2 cs = b.sk[(size_t)s * P.nk + k];
            erc += P.g0[k] * (cs.x * cs.x + cs.y * cs.y);
        }
    }
    double v[4] = {e0, e1, erc, eself};
    block_sum4(v, sh);
    e0 = v[0];
    e1 = v[1];
    erc = v[2];
    eself = v[3];
    if (threadIdx.x == 0) {
        double* out = energy + 5 * (size_t)s;
        if (family == AKMC_FAMILY_IONIC) {
            const double rcp = 0.5 * erc, real = e0 + eself, vdw = e1;
            out[0] = rcp + real + vdw;
            out[1] = rcp;
            out[2] = real;
            out[3] = vdw;
            out[4] = 0.0;
        } else {
            out[0] = e0 + e1;
            out[1] = 0.0;
            out[2] = 0.0;
            out[3] = e1;
            out[4] = e0;
        }
    }
}

template <class Pass>
size_t pair_smem(int cap)
{
    if (Pass::kStage == kStageF64) return (size_t)cap * (sizeof(double4) + sizeof(int));
    if (Pass::kStage == kStageF32Q) return (size_t)cap * (sizeof(float4) + sizeof(int));
    return (size_t)cap * sizeof(float4);
}

// Persistent CTAs of a kernel: resident blocks per SM x SMs (at least 1).
template <class K>
int resident_grid(K kernel, int threads, size_t smem)
{
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    return sms * per_sm;
}

// One pair pass.  With work queues (b.work) the grid is the resident CTAs (at most one per
// planned item), which take the queued items by the ticket counter `ticket`; without, one
// CTA per planned item.  early: launch with programmatic stream serialisation, so the
// kernel may start while the previous kernel on the stream is still running (it waits
// before reading its output).  A pass that defers its wait (kOverlapPrior) must be launched
// late when its predecessor is not the structure-factor kernel.
template <class Pass>
cudaError_t launch_pair(BatchDev b, const Pass& p, double rc2, int* status, cudaStream_t s, int ticket,
                        bool early = true)
{
    if (b.total_items == 0) return cudaSuccess;
    cudaLaunchConfig_t cfg = {};
    const size_t smem = pair_smem<Pass>(b.stage_cap);
    int grid = b.total_items;
    if (b.work) {
        b.ticket = b.counters + ticket;
        grid = std::min(grid, resident_grid(pair_kernel<Pass, true>, Pass::kThreads, smem));
    }
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(Pass::kThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = early ? 1 : 0;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (b.work) return cudaLaunchKernelEx(&cfg, pair_kernel<Pass, true>, b, p, rc2, status);
    return cudaLaunchKernelEx(&cfg, pair_kernel<Pass, false>, b, p, rc2, status);
}

// Grid of a list kernel: resident CTAs (at most one per queued-chunk slot) with queues,
// one CTA per kListThreads atoms without.
template <class K>
int list_grid(const BatchDev& b, K kernel)
{
    if (b.chunks) return std::max(1, std::min(b.chunk_cap, resident_grid(kernel, kListThreads, 0)));
    return (b.n_total + kListThreads - 1) / kListThreads;
}

size_t whole_cell_smem(int n)
{
    return (size_t)n * sizeof(float4) + (((size_t)n + 15) & ~size_t(15)) +
           (size_t)kWcWarps * kWcChunk * 32 * sizeof(unsigned short);
}

template <class Pass>
cudaError_t allow_smem()
{
    const int bytes = (int)pair_smem<Pass>(kStageCap);
    cudaError_t e = cudaFuncSetAttribute(pair_kernel<Pass, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(pair_kernel<Pass, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

}  // namespace

cudaError_t configure_pair_kernels()
{
    cudaError_t e;
    if ((e = allow_smem<EamDensityPass<false>>()) != cudaSuccess) return e;
    if ((e = allow_smem<EamDensityPass<true>>()) != cudaSuccess) return e;
    if ((e = allow_smem<EamForcePass<false>>()) != cudaSuccess) return e;
    if ((e = allow_smem<EamForcePass<true>>()) != cudaSuccess) return e;
    if ((e = allow_smem<IonicPass<false>>()) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(structure_factor_tab_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(sizeof(double2) * kSkAtomChunk * kMaxSkTable))) != cudaSuccess)
        return e;
    if ((e = cudaFuncSetAttribute(ionic_whole_cell_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)whole_cell_smem(kWholeCellMaxAtoms))) != cudaSuccess)
        return e;
    return allow_smem<IonicPass<true>>();
}

cudaError_t launch_eam_density(const BatchDev& b, const EamDev& p, double rc2, int* status,
                               int precision, cudaStream_t s)
{
    // systems that rebuild their list scan the cells out to cutoff + skin; systems that
    // reuse one walk it
    const double rl = sqrt(rc2) + b.skin;
    const double rc2_list = b.skin > 0.0 ? rl * rl : rc2;
    cudaError_t e;
    if (precision == AKMC_PREC_FP64) {
        EamDensityPass<true> pass{p, b.sextra, b.eatom, b.nbr, b.nbr_count, b.nbr_cap, b.n_total, rc2, b.frec};
        e = launch_pair(b, pass, rc2_list, status, s, kTicketDensity);
    } else {
        EamDensityPass<false> pass{p, b.sextra, b.eatom, b.nbr, b.nbr_count, b.nbr_cap, b.n_total, rc2, b.frec};
        e = launch_pair(b, pass, rc2_list, status, s, kTicketDensity);
    }
    if (e != cudaSuccess || b.skin <= 0.0) return e;
    if (precision == AKMC_PREC_FP64) {
        const int blocks = list_grid(b, eam_density_list_kernel<true>);
        return launch_pdl(eam_density_list_kernel<true>, dim3(blocks), dim3(kListThreads), 0, s, b, p, rc2, status);
    }
    const int blocks = list_grid(b, eam_density_list_kernel<false>);
    return launch_pdl(eam_density_list_kernel<false>, dim3(blocks), dim3(kListThreads), 0, s, b, p, rc2, status);
}

cudaError_t launch_eam_force(const BatchDev& b, const EamDev& p, double rc2, double* force,
                             int* status, int precision, cudaStream_t s)
{
    if (b.nbr) {
        auto go = [&](auto kernel) {
            return launch_pdl(kernel, dim3(list_grid(b, kernel)), dim3(kListThreads), 0, s, b, p, rc2, force, status);
        };
        if (precision == AKMC_PREC_FP64)
            return p.ntab > 1 ? go(eam_force_list_kernel<true, true>) : go(eam_force_list_kernel<true, false>);
        return p.ntab > 1 ? go(eam_force_list_kernel<false, true>) : go(eam_force_list_kernel<false, false>);
    }
    if (precision == AKMC_PREC_FP64) {
        EamForcePass<true> pass{p, force, b.eatom, b.sextra};
        return launch_pair(b, pass, rc2, status, s, kTicketForce);
    }
    EamForcePass<false> pass{p, force, b.eatom, b.sextra};
    return launch_pair(b, pass, rc2, status, s, kTicketForce);
}

cudaError_t launch_structure_factor(const BatchDev& b, const IonicDev& p, int precision,
                                    cudaStream_t s)
{
    if (p.nk == 0) return cudaSuccess;
    if (precision != AKMC_PREC_FP64 && p.ntab <= kMaxSkTable) {
        const size_t smem = sizeof(double2) * (size_t)kSkAtomChunk * p.ntab;
        return launch_pdl(structure_factor_tab_kernel, dim3(b.sk_chunks, b.nsys), dim3(kSkTabThreads), smem, s, b, p);
    }
    dim3 grid((p.nk + kSkThreads - 1) / kSkThreads, b.sk_chunks, b.nsys);
    if (precision == AKMC_PREC_FP64)
        return launch_pdl(structure_factor_kernel<true>, grid, dim3(kSkThreads), 0, s, b, p);
    return launch_pdl(structure_factor_kernel<false>, grid, dim3(kSkThreads), 0, s, b, p);
}

cudaError_t launch_ionic_force(const BatchDev& b, const IonicDev& p, double rc2, double* force, double* energy,
                               int* status, int precision, cudaStream_t s)
{
    const float rs2 = (float)p.r_split2;
    const float lo = (float)(rc2 * (1.0 - 1.0e-5)), hi = (float)(rc2 * (1.0 + 1.0e-5));
    // the real-space part overlaps the structure-factor kernel and the reciprocal part
    // waits for it; without k-vectors the predecessor is the cell kernel: launch late
    if (precision == AKMC_PREC_FP64) {
        IonicPass<true> pass{p, b.sk, b.skf, b.slabel, force, b.eatom, rs2, lo, hi};
        return launch_pair(b, pass, rc2, status, s, kTicketIonic, p.nk > 0);
    }
    IonicPass<false> pass{p, b.sk, b.skf, b.slabel, force, b.eatom, rs2, lo, hi};
    if (b.whole_cell_n > 0) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((b.whole_cell_n + 31) / 32, b.nsys);
        cfg.blockDim = dim3(kWcWarps * 32);
        cfg.dynamicSmemBytes = whole_cell_smem(b.whole_cell_n);
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = p.nk > 0 ? 1 : 0;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        return cudaLaunchKernelEx(&cfg, ionic_whole_cell_kernel, b, pass, rc2, status, energy);
    }
    return launch_pair(b, pass, rc2, status, s, kTicketIonic, p.nk > 0);
}

cudaError_t launch_energy_reduce(const BatchDev& b, int family, const IonicDev* ip,
                                 double* energy, cudaStream_t s)
{
    IonicDev p{};
    if (ip) p = *ip;
    return launch_pdl(energy_reduce_kernel, dim3(b.nsys), dim3(kReduceThreads), 0, s, b, family, p, energy);
}

}  // namespace akmc
