// Pair kernels of the AKMC force path (sm_100a).
//
//   K2 eam_density  rho_i = sum_j rho(r_ij); F(rho_i), F'(rho_i)
//        calculateAtomRho (potentials/metal/Field.cpp:1782-1853), ManyBody::embed
//        (potentials/metal/ManyBody.cpp:554-619)
//   K3 eam_force    F_i = -sum_j [phi'(r) + (F'_i + F'_j) rho'(r)] (r_i - r_j)/r,
//        E_pair = sum_{i<j} phi: realSpaceForceImage pass 2 (metal/Field.cpp:371-449),
//        calculateManyBodyPairForce / calculateManyBodyForce (ManyBody.cpp:621-831)
//   K4+K6 ionic_force  Ewald real space erfc(eta r)/r + Buckingham
//        (pair/Field.cpp:660-842, TwoBody.h:203-215, hfunc1 pair/Field.cpp:2218-2236),
//        fused with the reciprocal-space force of the same atom (Ewald.cpp:636-646)
//   K5 structure_factor  C_k = sum q cos(k.r), S_k = sum q sin(k.r) (Ewald.cpp:585-611)
//   K7 energy_reduce  per-system FP64 energies, Ewald self term (pair/Field.cpp:704-720)
//
// Work decomposition of K2/K3/K4: one CTA per work item (<= 32 home atoms of one cell,
// built by K1).  The CTA stages the positions of the neighbour cells (shifted to the
// home cell's periodic image) in shared memory, then each warp takes one home atom at a
// time: lanes test 32 candidates at once in FP64, accepted pairs are compacted into a
// per-warp queue (ballot + popc), and the pair terms run on full warps of queued pairs.
// Lane partial sums are FP64 and reduced with warp shuffles in a fixed order, so the
// result is bitwise reproducible.
//
// Precision (AKMC_PREC_MIXED): geometry, r and all accumulations FP64; EAM table
// interpolation FP32; ionic pair terms FP32 beyond r_split and FP64 inside it (the few
// nearest shells carry the largest forces); reciprocal phases reduced in FP64 before an
// FP32 sincospi.  AKMC_PREC_FP64: every term FP64.
#include "akmc_internal.h"

namespace akmc {

namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ void set_status(int* st, int code) { atomicCAS(st, 0, code); }

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

// ---------------------------------------------------------------------------------
// neighbour ranges of one home cell
// ---------------------------------------------------------------------------------
struct RangeSet {
    int n, total, home_range, home_start;
    int start[27];
    int prefix[28];
    double shift[27][3];
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

__device__ __forceinline__ int find_system(const BatchDev& b, int blk)
{
    int lo = 0, hi = b.nsys - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (b.geom[mid].item_base <= blk) lo = mid; else hi = mid - 1;
    }
    return lo;
}

struct Geo {            // per-CTA copy of the system geometry used in the inner loops
    double L0, L1, L2, iL0, iL1, iL2;
    int mi;
};

__device__ __forceinline__ double displacement(const Geo& G, double hx, double hy, double hz,
                                               const double4& p, double& dx, double& dy,
                                               double& dz)
{
    dx = hx - p.x;
    dy = hy - p.y;
    dz = hz - p.z;
    if (G.mi & 1) dx = fma(-rint(dx * G.iL0), G.L0, dx);
    if (G.mi & 2) dy = fma(-rint(dy * G.iL1), G.L1, dy);
    if (G.mi & 4) dz = fma(-rint(dz * G.iL2), G.L2, dz);
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
    __device__ __forceinline__ void reduce()
    {
        #pragma unroll
        for (int k = 0; k < N; k++) v[k] = warp_sum(v[k]);
    }
};

// K2: EAM density.  spos.w holds the species label.
template <bool kFp64>
struct EamDensityPass {
    static constexpr int kAcc = 1, kQueues = 1, kExtraBytes = 0;
    EamDev P;
    double2* sextra;
    double2* eatom;
    struct Ctx { int li; int* st; };

    __device__ Ctx home(const BatchDev& b, int i, int* st) const { return Ctx{b.slabel[i], st}; }
    __device__ int classify(double) const { return 0; }
    __device__ void stage_extra(const BatchDev&, void*, int, int) const {}

    __device__ void pair(int, AccN<1>& acc, const Ctx& cx, double, double, double, double rsq,
                         const double4& pj, const void*, int) const
    {
        const int lj = (int)pj.w;
        if (!P.dens_ok[lj]) return;
        double r, ir;
        if (kFp64) { r = sqrt(rsq); } else { refined_sqrt(rsq, r, ir); }
        if (r < 1.0e-8 || !(r < P.pot_cutoff)) return;
        const double tr = r * P.inv_step_r;
        const int idx = (int)tr;
        if (idx >= P.n_r - 1) { set_status(cx.st, AKMC_ERR_TABLE_RANGE); return; }
        if (kFp64) {
            const double p0 = P.rho[idx], p1 = P.rho[idx + 1];
            acc.v[0] += p0 + (p1 - p0) * (r - idx * P.step_r) * P.inv_step_r;
        } else {
            const float4 row = __ldg(&P.rows[2 * idx + 1]);
            acc.v[0] += (double)(row.z + row.w * (float)(tr - idx));
        }
    }

    __device__ void post(const BatchDev&, int, const Geo&, const double4&, const Ctx&,
                         AccN<1>&) const {}

    // ManyBody::embed EAM branch (ManyBody.cpp:598-615) for F and, once per atom, the
    // derivEmbed interpolation the force pass needs (ManyBody.cpp:797-810).
    __device__ void finish(const BatchDev&, int i, const Ctx& cx, const double* a) const
    {
        const double rho = a[0];
        double F = 0.0, fp = 0.0;
        if (P.embed_ok[cx.li]) {
            const int idx = (int)(rho * P.inv_step_embed);
            if (idx < 0 || idx >= P.n_embed - 1) {
                set_status(cx.st, AKMC_ERR_EMBED_RANGE);
            } else {
                const double t = (rho - idx * P.step_embed) * P.inv_step_embed;
                F = P.F[idx] + (P.F[idx + 1] - P.F[idx]) * t;
                fp = P.dF[idx] + (P.dF[idx + 1] - P.dF[idx]) * t;
            }
        }
        sextra[i] = make_double2(fp, rho);
        eatom[i].x = F;
    }
};

// K3: EAM force and pair energy.  Staged extra per candidate: {F'(rho_j), rho_j}.
template <bool kFp64>
struct EamForcePass {
    static constexpr int kAcc = 4, kQueues = 1, kExtraBytes = sizeof(double2);
    EamDev P;
    double* force;
    double2* eatom;
    struct Ctx { int li; double fpi, rhoi; int* st; };

    __device__ Ctx home(const BatchDev& b, int i, int* st) const
    {
        const double2 e = b.sextra[i];
        return Ctx{b.slabel[i], e.x, e.y, st};
    }
    __device__ int classify(double) const { return 0; }
    __device__ void stage_extra(const BatchDev& b, void* ext, int t, int j) const
    {
        reinterpret_cast<double2*>(ext)[t] = b.sextra[j];
    }

    __device__ void pair(int, AccN<4>& acc, const Ctx& cx, double dx, double dy, double dz,
                         double rsq, const double4& pj, const void* ext, int t) const
    {
        const int lj = (int)pj.w;
        if (!P.pair_ok[cx.li * P.ns + lj]) return;
        double r, ir;
        if (kFp64) { r = sqrt(rsq); ir = 1.0 / r; } else { refined_sqrt(rsq, r, ir); }
        if (r < 1.0e-8 || !(r < P.pot_cutoff)) return;
        const double tr = r * P.inv_step_r;
        const int idx = (int)tr;
        if (idx >= P.n_r - 1) { set_status(cx.st, AKMC_ERR_TABLE_RANGE); return; }
        const double2 ej = reinterpret_cast<const double2*>(ext)[t];
        const bool mb = !(cx.rhoi < 1.0e-8 || ej.y < 1.0e-8);     // ManyBody.cpp:730-731
        double g, phi;
        if (kFp64) {
            const double w = (r - idx * P.step_r) * P.inv_step_r;
            phi = P.phi[idx] + (P.phi[idx + 1] - P.phi[idx]) * w;
            const double dphi = P.dphi[idx] + (P.dphi[idx + 1] - P.dphi[idx]) * w;
            const double drho = P.drho[idx] + (P.drho[idx + 1] - P.drho[idx]) * w;
            g = (dphi + (mb ? (cx.fpi + ej.x) * drho : 0.0)) * ir;
        } else {
            const float ft = (float)(tr - idx);
            const float4 A = __ldg(&P.rows[2 * idx]);
            const float4 B = __ldg(&P.rows[2 * idx + 1]);
            const float phif = A.x + A.y * ft;
            const float dphi = A.z + A.w * ft;
            const float drho = B.x + B.y * ft;
            const float many = mb ? (float)(cx.fpi + ej.x) * drho : 0.0f;
            phi = (double)phif;
            g = (double)(dphi + many) * ir;
        }
        acc.v[0] -= g * dx;
        acc.v[1] -= g * dy;
        acc.v[2] -= g * dz;
        acc.v[3] += 0.5 * phi;
    }

    __device__ void post(const BatchDev&, int, const Geo&, const double4&, const Ctx&,
                         AccN<4>&) const {}

    __device__ void finish(const BatchDev& b, int i, const Ctx&, const double* a) const
    {
        const int o = b.perm[i];
        force[3 * (size_t)o + 0] = a[0];
        force[3 * (size_t)o + 1] = a[1];
        force[3 * (size_t)o + 2] = a[2];
        eatom[i].y = a[3];
    }
};

// K4+K6: ionic real space (queue 0 = FP32 terms, queue 1 = FP64 terms) fused with the
// reciprocal-space force of the home atom.  Staged extra per candidate: species label.
template <bool kFp64>
struct IonicPass {
    static constexpr int kAcc = 5, kQueues = kFp64 ? 1 : 2, kExtraBytes = sizeof(int);
    IonicDev P;
    const double2* sk;
    double* force;
    double2* eatom;
    struct Ctx { int li; double qi; int* st; };

    __device__ Ctx home(const BatchDev& b, int i, int* st) const
    {
        return Ctx{b.slabel[i], b.spos[i].w, st};
    }
    __device__ int classify(double rsq) const { return kFp64 ? 0 : (rsq < P.r_split2 ? 1 : 0); }
    __device__ void stage_extra(const BatchDev& b, void* ext, int t, int j) const
    {
        reinterpret_cast<int*>(ext)[t] = b.slabel[j];
    }

    __device__ void pair(int q, AccN<5>& acc, const Ctx& cx, double dx, double dy, double dz,
                         double rsq, const double4& pj, const void* ext, int t) const
    {
        const int lj = reinterpret_cast<const int*>(ext)[t];
        const int ab = cx.li * P.ns + lj;
        const double qq = P.cfact * cx.qi * pj.w;
        if (kFp64 || q == 1) {
            const double r = sqrt(rsq);
            const double x = P.eta * r;
            double forc = 0.0, eng = 0.0, es = 0.0;
            if (x != 0.0) {
                const double h0 = erfc(x) / x;
                const double xsq = x * x;
                const double h1 = (-h0 - kTwoOverRootPi * exp(-xsq)) / xsq;
                eng = h0 * qq * P.eta;
                forc = h1 * qq * (P.eta * P.eta * P.eta);
            }
            if (r >= 1.0e-8) {
                const double e1 = P.buckA[ab] * exp(-r * P.buckInvRho[ab]);
                const double f1 = e1 * P.buckInvRho[ab] / r;
                const double e2 = -P.buckC[ab] / (rsq * rsq * rsq);
                const double f2 = 6.0 * e2 / rsq;
                es = e1 + e2;
                forc -= f1 + f2;
            }
            acc.v[0] -= forc * dx;
            acc.v[1] -= forc * dy;
            acc.v[2] -= forc * dz;
            acc.v[3] += 0.5 * eng;
            acc.v[4] += 0.5 * es;
        } else {
            const float rsqf = (float)rsq;
            const float ir = rsqrtf(rsqf);
            const float r = rsqf * ir;
            const float eta = (float)P.eta;
            const float x = eta * r;
            const float h0 = erfcf(x) / x;
            const float xsq = x * x;
            const float h1 = (-h0 - (float)kTwoOverRootPi * expf(-xsq)) / xsq;
            const float qqf = (float)qq;
            const float eng = h0 * qqf * eta;
            float forc = h1 * qqf * (eta * eta * eta);
            const float irho = (float)P.buckInvRho[ab];
            const float e1 = (float)P.buckA[ab] * expf(-r * irho);
            const float f1 = e1 * irho * ir;
            const float ir2 = ir * ir;
            const float e2 = -(float)P.buckC[ab] * (ir2 * ir2 * ir2);
            const float f2 = 6.0f * e2 * ir2;
            forc -= f1 + f2;
            const double fd = (double)forc;
            acc.v[0] -= fd * dx;
            acc.v[1] -= fd * dy;
            acc.v[2] -= fd * dz;
            acc.v[3] += 0.5 * (double)eng;
            acc.v[4] += 0.5 * (double)(e1 + e2);
        }
    }

    // Reciprocal force on the home atom (Ewald.cpp:636-646): lanes stride over k.
    __device__ void post(const BatchDev& b, int s, const Geo& G, const double4& hp,
                         const Ctx& cx, AccN<5>& acc) const
    {
        const int lane = threadIdx.x & 31;
        const double sx = hp.x * G.iL0, sy = hp.y * G.iL1, sz = hp.z * G.iL2;
        const double2* skk = sk + (size_t)s * P.nk;
        double ax = 0.0, ay = 0.0, az = 0.0;
        for (int k = lane; k < P.nk; k += 32) {
            const int4 n = __ldg(&P.kint[k]);
            const double2 cs = skk[k];
            const double g0 = __ldg(&P.g0[k]);
            double u = n.x * sx + n.y * sy + n.z * sz;
            u -= rint(u);
            double sn, cn;
            if (kFp64) {
                sincospi(2.0 * u, &sn, &cn);
            } else {
                float sf, cf;
                sincospif(2.0f * (float)u, &sf, &cf);
                sn = sf;
                cn = cf;
            }
            const double pf = -g0 * cx.qi * (-sn * cs.x + cn * cs.y);
            ax += pf * (double)n.x;
            ay += pf * (double)n.y;
            az += pf * (double)n.z;
        }
        acc.v[0] += ax * kTwoPi * G.iL0;
        acc.v[1] += ay * kTwoPi * G.iL1;
        acc.v[2] += az * kTwoPi * G.iL2;
    }

    __device__ void finish(const BatchDev& b, int i, const Ctx&, const double* a) const
    {
        const int o = b.perm[i];
        force[3 * (size_t)o + 0] = a[0];
        force[3 * (size_t)o + 1] = a[1];
        force[3 * (size_t)o + 2] = a[2];
        eatom[i] = make_double2(a[3], a[4]);
    }
};

// ---------------------------------------------------------------------------------
// the shared pair kernel
// ---------------------------------------------------------------------------------
template <class Pass>
__global__ void __launch_bounds__(kPairThreads)
pair_kernel(BatchDev b, Pass pass, double rc2, int* status)
{
    extern __shared__ __align__(16) unsigned char dyn[];
    double4* s_pos = reinterpret_cast<double4*>(dyn);
    void* s_ext = reinterpret_cast<void*>(s_pos + b.stage_cap);

    __shared__ RangeSet rs;
    __shared__ int s_q[kPairWarps][2][64];
    __shared__ double s_acc[kHomeChunk][Pass::kAcc];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int s = find_system(b, blockIdx.x);
    const SysGeom& gref = b.geom[s];
    const int local = blockIdx.x - gref.item_base;
    if (local >= b.n_items[s]) return;
    const WorkItem it = b.items[gref.item_base + local];
    Geo G;
    G.L0 = gref.L[0]; G.L1 = gref.L[1]; G.L2 = gref.L[2];
    G.iL0 = gref.invL[0]; G.iL1 = gref.invL[1]; G.iL2 = gref.invL[2];
    G.mi = gref.mi_mask;
    int* st = status + s;

    if (warp == 0) {
        const SysGeom g = gref;
        build_ranges(b, g, it.cell, rs);
    }
    for (int k = tid; k < kHomeChunk * Pass::kAcc; k += blockDim.x) (&s_acc[0][0])[k] = 0.0;
    __syncthreads();

    const int total = rs.total;
    const int cap = b.stage_cap;
    const int self_base = rs.prefix[rs.home_range] - rs.home_start;

    for (int rb = 0; rb < total; rb += cap) {
        const int m = min(cap, total - rb);
        __syncthreads();
        for (int t = tid; t < m; t += blockDim.x) {
            const int f = rb + t;
            const int ri = find_range(rs, f);
            const int j = rs.start[ri] + (f - rs.prefix[ri]);
            double4 p = b.spos[j];
            p.x += rs.shift[ri][0];
            p.y += rs.shift[ri][1];
            p.z += rs.shift[ri][2];
            s_pos[t] = p;
            pass.stage_extra(b, s_ext, t, j);
        }
        __syncthreads();

        for (int a = warp; a < it.count; a += kPairWarps) {
            const int i = it.first + a;
            const double4 hp = b.spos[i];
            const auto cx = pass.home(b, i, st);
            const int self_t = self_base + i - rb;
            AccN<Pass::kAcc> acc;
            acc.zero();
            int qh[2] = {0, 0}, qt[2] = {0, 0};

            for (int base = 0; base < m; base += 32) {
                const int t = base + lane;
                int cls = -1;
                if (t < m && t != self_t) {
                    double dx, dy, dz;
                    const double rsq = displacement(G, hp.x, hp.y, hp.z, s_pos[t], dx, dy, dz);
                    if (rsq <= rc2) {
                        if (rsq < 1.0e-16) set_status(st, AKMC_ERR_NONFINITE);
                        else cls = pass.classify(rsq);
                    }
                }
                #pragma unroll
                for (int qi = 0; qi < Pass::kQueues; qi++) {
                    const unsigned bal = __ballot_sync(kFull, cls == qi);
                    if (cls == qi) s_q[warp][qi][(qt[qi] + __popc(bal & lanemask_lt())) & 63] = t;
                    qt[qi] += __popc(bal);
                    if (qt[qi] - qh[qi] >= 32) {
                        __syncwarp();
                        const int tq = s_q[warp][qi][(qh[qi] + lane) & 63];
                        double dx, dy, dz;
                        const double4 pj = s_pos[tq];
                        const double rsq = displacement(G, hp.x, hp.y, hp.z, pj, dx, dy, dz);
                        pass.pair(qi, acc, cx, dx, dy, dz, rsq, pj, s_ext, tq);
                        qh[qi] += 32;
                        __syncwarp();
                    }
                }
            }
            #pragma unroll
            for (int qi = 0; qi < Pass::kQueues; qi++) {
                const int left = qt[qi] - qh[qi];
                if (left > 0) {
                    __syncwarp();
                    if (lane < left) {
                        const int tq = s_q[warp][qi][(qh[qi] + lane) & 63];
                        double dx, dy, dz;
                        const double4 pj = s_pos[tq];
                        const double rsq = displacement(G, hp.x, hp.y, hp.z, pj, dx, dy, dz);
                        pass.pair(qi, acc, cx, dx, dy, dz, rsq, pj, s_ext, tq);
                    }
                    __syncwarp();
                }
            }
            acc.reduce();
            if (lane == 0) {
                #pragma unroll
                for (int k = 0; k < Pass::kAcc; k++) s_acc[a][k] += acc.v[k];
            }
        }
    }
    __syncthreads();

    for (int a = warp; a < it.count; a += kPairWarps) {
        const int i = it.first + a;
        const double4 hp = b.spos[i];
        const auto cx = pass.home(b, i, st);
        AccN<Pass::kAcc> acc;
        acc.zero();
        pass.post(b, s, G, hp, cx, acc);
        acc.reduce();
        if (lane == 0) {
            double tot[Pass::kAcc];
            #pragma unroll
            for (int k = 0; k < Pass::kAcc; k++) tot[k] = s_acc[a][k] + acc.v[k];
            pass.finish(b, i, cx, tot);
        }
    }
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
    const int s = blockIdx.z, chunk = blockIdx.y, tile = blockIdx.x;
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
        const int4 n = __ldg(&P.kint[k]);
        const double nx = n.x, ny = n.y, nz = n.z;
        double C = 0.0, S = 0.0;
        for (int j = 0; j < na; j++) {
            const double4 a = s_at[j];
            double u = nx * a.x + ny * a.y + nz * a.z;
            u -= rint(u);
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
        }
        if (threadIdx.x == 0) *counter = 0;
    }
}

// ---------------------------------------------------------------------------------
// K7: per-system energies in a fixed summation order
// ---------------------------------------------------------------------------------
constexpr int kReduceThreads = 256;

__device__ double block_sum(double v, double* sh)
{
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double r = 0.0;
    if (warp == 0) {
        r = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
        r = warp_sum(r);
    }
    __syncthreads();
    return r;   // valid in thread 0
}

__global__ void __launch_bounds__(kReduceThreads)
energy_reduce_kernel(BatchDev b, int family, IonicDev P, double* energy)
{
    __shared__ double sh[32];
    const int s = blockIdx.x;
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
    e0 = block_sum(e0, sh);
    e1 = block_sum(e1, sh);
    erc = block_sum(erc, sh);
    eself = block_sum(eself, sh);
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
size_t pair_smem(int cap) { return (size_t)cap * (sizeof(double4) + Pass::kExtraBytes); }

template <class Pass>
cudaError_t launch_pair(const BatchDev& b, const Pass& p, double rc2, int* status, cudaStream_t s)
{
    if (b.total_items == 0) return cudaSuccess;
    pair_kernel<Pass><<<b.total_items, kPairThreads, pair_smem<Pass>(b.stage_cap), s>>>(b, p, rc2, status);
    return cudaGetLastError();
}

template <class Pass>
cudaError_t allow_smem()
{
    return cudaFuncSetAttribute(pair_kernel<Pass>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)pair_smem<Pass>(kStageCap));
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
    return allow_smem<IonicPass<true>>();
}

cudaError_t launch_eam_density(const BatchDev& b, const EamDev& p, double rc2, int* status,
                               int precision, cudaStream_t s)
{
    if (precision == AKMC_PREC_FP64) {
        EamDensityPass<true> pass{p, b.sextra, b.eatom};
        return launch_pair(b, pass, rc2, status, s);
    }
    EamDensityPass<false> pass{p, b.sextra, b.eatom};
    return launch_pair(b, pass, rc2, status, s);
}

cudaError_t launch_eam_force(const BatchDev& b, const EamDev& p, double rc2, double* force,
                             int* status, int precision, cudaStream_t s)
{
    if (precision == AKMC_PREC_FP64) {
        EamForcePass<true> pass{p, force, b.eatom};
        return launch_pair(b, pass, rc2, status, s);
    }
    EamForcePass<false> pass{p, force, b.eatom};
    return launch_pair(b, pass, rc2, status, s);
}

cudaError_t launch_structure_factor(const BatchDev& b, const IonicDev& p, int precision,
                                    cudaStream_t s)
{
    if (p.nk == 0) return cudaSuccess;
    dim3 grid((p.nk + kSkThreads - 1) / kSkThreads, b.sk_chunks, b.nsys);
    if (precision == AKMC_PREC_FP64)
        structure_factor_kernel<true><<<grid, kSkThreads, 0, s>>>(b, p);
    else
        structure_factor_kernel<false><<<grid, kSkThreads, 0, s>>>(b, p);
    return cudaGetLastError();
}

cudaError_t launch_ionic_force(const BatchDev& b, const IonicDev& p, double rc2, double* force,
                               int* status, int precision, cudaStream_t s)
{
    if (precision == AKMC_PREC_FP64) {
        IonicPass<true> pass{p, b.sk, force, b.eatom};
        return launch_pair(b, pass, rc2, status, s);
    }
    IonicPass<false> pass{p, b.sk, force, b.eatom};
    return launch_pair(b, pass, rc2, status, s);
}

cudaError_t launch_energy_reduce(const BatchDev& b, int family, const IonicDev* ip,
                                 double* energy, cudaStream_t s)
{
    IonicDev p{};
    if (ip) p = *ip;
    energy_reduce_kernel<<<b.nsys, kReduceThreads, 0, s>>>(b, family, p, energy);
    return cudaGetLastError();
}

}  // namespace akmc
