// Learned proposal directions for saddle searches (sm_100a): per-atom structural
// descriptors from the EAM neighbour list, and a small MLP mapping them to a displacement
// vector, with its training kernels.
//
// The reference has no learned component: its searches start from random displacements
// (SaddleSearch.cpp:356-421).  The model here proposes the starting displacement of a
// Dimer walker; random displacement stays as the fallback.
//
// Descriptors (64 per atom, FP32, from neighbours within kDescRc = 5 A, minimum image):
//   32 radial  G2_m = sum_j exp(-eta_r (r_ij - mu_m)^2) fc(r_ij), mu_m = 0.5 + m * 4.5/31;
//   32 angular G4   = 2^(1-zeta) sum_{j<k} (1 + lambda cos theta_ijk)^zeta
//                     exp(-eta (r_ij^2 + r_ik^2 + r_jk^2)) fc(r_ij) fc(r_ik) fc(r_jk)
//     (Behler, J. Chem. Phys. 134, 074106 (2011)), eta in {0.01, 0.03, 0.07, 0.15} A^-2,
//     zeta in {1, 2, 4, 8}, lambda in {+1, -1};  fc(r) = (cos(pi r / rc) + 1) / 2.
// MLP: 64 -> 128 -> 128 -> 128 -> 3, SiLU on the hidden layers; standardised inputs, inputs,
// weights and hidden activations rounded to BF16 (nearest even), FP32 accumulation, FP32
// biases.  Parameters are one FP32 vector W1 b1 W2 b2 W3 b3 W4 b4 (W stored [in][out]); the
// kernels round the weights to BF16 as they stage them in shared memory.
#include <cuda_bf16.h>

#include "host_internal.h"
#include "philox.h"

namespace akmc {

namespace {

constexpr float kDescRc = 5.0f;
constexpr int kNRad = 32;
constexpr int kNDesc = 64;
constexpr int kMaxDescNbr = 192;         // neighbours within kDescRc kept per atom
constexpr int kDescWarps = 4;

constexpr int kH = 128;
// parameter offsets
constexpr int kOW1 = 0, kOB1 = kOW1 + 64 * kH;
constexpr int kOW2 = kOB1 + kH, kOB2 = kOW2 + kH * kH;
constexpr int kOW3 = kOB2 + kH, kOB3 = kOW3 + kH * kH;
constexpr int kOW4 = kOB3 + kH, kOB4 = kOW4 + kH * 3;
constexpr int kNParams = kOB4 + 3;       // 41731
constexpr int kNParamsPad = 41736;       // bf16 staging, 16-byte multiple

__device__ __forceinline__ float fcut(float r) { return 0.5f * (__cosf(3.14159265358979f * r / kDescRc) + 1.0f); }

// ---------------------------------------------------------------------------------
// descriptors: warp per (sorted) atom over the EAM neighbour list of the last force call
// ---------------------------------------------------------------------------------
// The three per-atom vectors of the readout: B_m = sum_j phi_m(r_ij) (r_j - r_i) / r_ij,
// phi_m(r) = exp(-(r - nu_m)^2 / (2 * 0.25^2)) fc(r), nu = 2.5, 3.6, 4.4 A (the first three
// FCC shells of the metal workloads).  A model output c (3 numbers per atom) is the
// displacement sum_m c_m B_m: rotating the atom's surroundings rotates it (the invariant
// descriptors alone cannot point anywhere).
__device__ __forceinline__ float phi_shell(int m, float r)
{
    const float nu = m == 0 ? 2.5f : (m == 1 ? 3.6f : 4.4f);
    const float t = r - nu;
    return __expf(-t * t * 8.0f) * fcut(r);
}

// inv[perm[i]] = i: the sorted position of every caller atom
__global__ void invert_perm_kernel(const int* __restrict__ perm, int* __restrict__ inv, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const int o = perm[i];
        if (o >= 0 && o < n) inv[o] = i;
    }
}

// Every atom (rows null; output row = caller atom number) or the atoms rows[0..n_rows)
// (output row = position in rows; inv from invert_perm_kernel).
__global__ void __launch_bounds__(32 * kDescWarps)
descriptor_kernel(BatchDev b, const int* __restrict__ rows, int n_rows, const int* __restrict__ inv,
                  float* __restrict__ desc, float* __restrict__ basis)
{
    __shared__ float4 s_v[kDescWarps][kMaxDescNbr];
    __shared__ float4 s_w[kDescWarps][kMaxDescNbr];
    __shared__ float s_part[kDescWarps][32][33];
    __shared__ int2 s_pq[kDescWarps][64];     // queued pairs inside the cutoff
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wid = blockIdx.x * kDescWarps + warp;
    int i, orow;
    if (rows) {
        if (wid >= n_rows) return;
        orow = wid;
        const int o = rows[wid];
        if (o < 0 || o >= b.n_total) {
            desc[(size_t)orow * kNDesc + lane] = 0.0f;
            desc[(size_t)orow * kNDesc + kNRad + lane] = 0.0f;
            if (basis && lane < 9) basis[(size_t)orow * 9 + lane] = 0.0f;
            return;
        }
        i = inv[o];
    } else {
        i = wid;
        if (i >= b.n_total) return;
        orow = b.perm[i];
    }
    int lo = 0, hi = b.nsys - 1;                 // system of atom i
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (b.geom[mid].atom_begin <= i) lo = mid; else hi = mid - 1;
    }
    const SysGeom& g = b.geom[lo];
    const int a0 = g.atom_begin;
    const double4 hp = b.spos[i];
    const int il = i + list_shift(b, lo);       // its list row
    const int cnt = min(b.nbr_count[il], b.nbr_cap);
    // 1. the neighbours within the descriptor cutoff, compacted in list order
    int m = 0;
    for (int base = 0; base < cnt; base += 32) {
        const int k = base + lane;
        bool keep = false;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (k < cnt) {
            const int j = a0 + (int)b.nbr[(size_t)k * b.n_total + il];
            const double4 pj = b.spos[j];
            double dx = pj.x - hp.x, dy = pj.y - hp.y, dz = pj.z - hp.z;
            dx -= g.L[0] * rint(dx * g.invL[0]);
            dy -= g.L[1] * rint(dy * g.invL[1]);
            dz -= g.L[2] * rint(dz * g.invL[2]);
            const double r2 = dx * dx + dy * dy + dz * dz;
            keep = r2 > 0.0 && r2 < (double)kDescRc * kDescRc;
            v = make_float4((float)dx, (float)dy, (float)dz, (float)sqrt(r2));
        }
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        const int slot = m + __popc(bal & ((1u << lane) - 1u));
        if (keep && slot < kMaxDescNbr) s_v[warp][slot] = v;
        m += __popc(bal);
    }
    m = min(m, kMaxDescNbr);
    __syncwarp();
    // 2. radial: lane = function index
    const float step = 4.5f / (kNRad - 1);
    const float eta_r = 1.0f / (2.0f * step * step);
    float rad = 0.0f;
    const float mu = 0.5f + lane * step;
    for (int e = 0; e < m; e++) {
        const float r = s_v[warp][e].w;
        const float t = r - mu;
        rad += __expf(-eta_r * t * t) * fcut(r);
    }
    // 3. angular.  Per neighbour: fc(r), exp(-eta0 r^2) with eta0 = 0.01, 1/r.  Every eta is
    // a multiple of eta0 (1, 3, 7, 15), so exp(-eta (r_ij^2 + r_ik^2 + r_jk^2)) is a power of
    // E = exp(-eta0 r_ij^2) exp(-eta0 r_ik^2) exp(-eta0 r_jk^2).  The pairs j < k are dealt
    // to the lanes in row-major order, 32 at a time; 32 partial sums per lane.
    for (int e = lane; e < m; e += 32) {
        const float r = s_v[warp][e].w;
        s_w[warp][e] = make_float4(fcut(r), __expf(-0.01f * r * r), 1.0f / r, 0.0f);
    }
    __syncwarp();
    float acc[32];
    #pragma unroll
    for (int t = 0; t < 32; t++) acc[t] = 0.0f;
    const float Lx = (float)g.L[0], Ly = (float)g.L[1], Lz = (float)g.L[2];
    const float iLx = (float)g.invL[0], iLy = (float)g.invL[1], iLz = (float)g.invL[2];
    // the pair terms of queue entry e (pair j < k inside the cutoff, its r_jk^2)
    auto heavy = [&](int2 e) {
        const int j = e.x & 0xffff, k = e.x >> 16;
        const float r2jk = __int_as_float(e.y);
        const float4 vj = s_v[warp][j], wj = s_w[warp][j];
        const float4 vk = s_v[warp][k], wk = s_w[warp][k];
        const float cs = (vj.x * vk.x + vj.y * vk.y + vj.z * vk.z) * (wj.z * wk.z);
        const float base = wj.x * wk.x * fcut(sqrtf(r2jk));
        const float E1 = wj.y * wk.y * __expf(-0.01f * r2jk);
        const float E3 = E1 * E1 * E1, E7 = E3 * E3 * E1, E15 = E7 * E7 * E1;
        const float p1 = 1.0f + cs, q1 = 1.0f - cs;
        const float p2 = p1 * p1, p4 = p2 * p2, p8 = p4 * p4;
        const float q2 = q1 * q1, q4 = q2 * q2, q8 = q4 * q4;
        const float gws[4] = {base * E1, base * E3, base * E7, base * E15};
        #pragma unroll
        for (int ie = 0; ie < 4; ie++) {
            const float gw = gws[ie];
            // zeta 1, 2, 4, 8; the factors 2^(1 - zeta) are applied to the sums
            acc[ie * 8 + 0] = fmaf(gw, p1, acc[ie * 8 + 0]);
            acc[ie * 8 + 1] = fmaf(gw, q1, acc[ie * 8 + 1]);
            acc[ie * 8 + 2] = fmaf(gw, p2, acc[ie * 8 + 2]);
            acc[ie * 8 + 3] = fmaf(gw, q2, acc[ie * 8 + 3]);
            acc[ie * 8 + 4] = fmaf(gw, p4, acc[ie * 8 + 4]);
            acc[ie * 8 + 5] = fmaf(gw, q4, acc[ie * 8 + 5]);
            acc[ie * 8 + 6] = fmaf(gw, p8, acc[ie * 8 + 6]);
            acc[ie * 8 + 7] = fmaf(gw, q8, acc[ie * 8 + 7]);
        }
    };
    // The pairs j < k are dealt to the lanes in row-major order, 32 at a time; the pairs
    // inside the cutoff go to a per-warp queue, and every full 32 of them are taken by the
    // 32 lanes at once, so the pair terms run with every lane busy.
    int2* q = s_pq[warp];
    int nq = 0;
    int j = 0, k = 1 + lane;
    while (j < m - 1 && k >= m) {
        j++;
        k = k - m + j + 1;
    }
    const int npairs = m * (m - 1) / 2;
    for (int base_p = 0; base_p < npairs; base_p += 32) {
        bool in = false;
        float r2jk = 0.0f;
        if (base_p + lane < npairs) {
            const float4 vj = s_v[warp][j], vk = s_v[warp][k];
            float dx = vk.x - vj.x, dy = vk.y - vj.y, dz = vk.z - vj.z;
            dx -= Lx * rintf(dx * iLx);
            dy -= Ly * rintf(dy * iLy);
            dz -= Lz * rintf(dz * iLz);
            r2jk = dx * dx + dy * dy + dz * dz;
            in = r2jk < kDescRc * kDescRc;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, in);
        if (in) q[nq + __popc(bal & ((1u << lane) - 1u))] = make_int2(j | (k << 16), __float_as_int(r2jk));
        nq += __popc(bal);
        __syncwarp();
        if (nq >= 32) {
            heavy(q[lane]);
            __syncwarp();
            if (lane < nq - 32) q[lane] = q[32 + lane];
            nq -= 32;
            __syncwarp();
        }
        k += 32;                                // the pair 32 further on
        while (j < m - 1 && k >= m) {
            j++;
            k = k - m + j + 1;
        }
    }
    if (lane < nq) heavy(q[lane]);
    #pragma unroll
    for (int t = 0; t < 32; t++) s_part[warp][lane][t] = acc[t];
    __syncwarp();
    float ang = 0.0f;
    for (int l = 0; l < 32; l++) ang += s_part[warp][l][lane];     // fixed order
    const int zi = (lane & 7) >> 1;                                  // zeta 1, 2, 4, 8
    ang *= zi == 0 ? 1.0f : (zi == 1 ? 0.5f : (zi == 2 ? 0.125f : 0.0078125f));
    desc[(size_t)orow * kNDesc + lane] = rad;
    desc[(size_t)orow * kNDesc + kNRad + lane] = ang;
    if (basis) {
        // lanes 0..8: component (lane % 3) of B_(lane / 3), summed in list order
        if (lane < 9) {
            const int mm = lane / 3, c = lane % 3;
            float acc = 0.0f;
            for (int e = 0; e < m; e++) {
                const float4 v = s_v[warp][e];
                const float comp = c == 0 ? v.x : (c == 1 ? v.y : v.z);
                acc += phi_shell(mm, v.w) * comp / v.w;
            }
            basis[(size_t)orow * 9 + lane] = acc;
        }
    }
}

// ---------------------------------------------------------------------------------
// MLP shared helpers
// ---------------------------------------------------------------------------------
__device__ __forceinline__ float rbf(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
// SiLU z / (1 + e^-z) with the fast divide; below z = -80 (where 1 + e^-z would leave the
// fast divide's range) the value is below 1e-32 and returned as 0
__device__ __forceinline__ float silu_f(float z) { return z < -80.0f ? 0.0f : __fdividef(z, 1.0f + __expf(-z)); }

// stage the weights (BF16) and biases (FP32) of all four layers
__device__ void stage_params(const float* __restrict__ P, __nv_bfloat16* sW, float* sB)
{
    for (int k = threadIdx.x; k < kNParamsPad; k += blockDim.x) {
        const bool bias = (k >= kOB1 && k < kOW2) || (k >= kOB2 && k < kOW3) || (k >= kOB3 && k < kOW4) ||
                          (k >= kOB4 && k < kNParams);
        sW[k] = __float2bfloat16_rn(k < kNParams && !bias ? P[k] : 0.0f);
    }
    for (int k = threadIdx.x; k < 3 * kH + 3; k += blockDim.x) {
        const int o = k < kH ? kOB1 + k : (k < 2 * kH ? kOB2 + k - kH : (k < 3 * kH ? kOB3 + k - 2 * kH : kOB4 + k - 3 * kH));
        sB[k] = P[o];
    }
}

// out[r][c] = sum_k in[r][k] W[k][c] + bias[c] for R rows x 128 columns, optionally SiLU and
// BF16 rounding; z (if given) keeps the pre-activation.  Thread t owns rows
// (t / 16) * RPT .. + RPT - 1 and columns (t % 16) * 8 .. + 7 (256 threads).
template <int R, int K>
__device__ void dense128(const float* in, int ldi, const __nv_bfloat16* W, const float* bias,
                         float* out, int ldo, float* z, bool act)
{
    constexpr int RPT = R / 16;
    const int rg = threadIdx.x >> 4, cg = threadIdx.x & 15;
    float acc[RPT][8];
    #pragma unroll
    for (int r = 0; r < RPT; r++)
        #pragma unroll
        for (int c = 0; c < 8; c++) acc[r][c] = bias[cg * 8 + c];
    for (int k = 0; k < K; k++) {
        const uint4 wv = *reinterpret_cast<const uint4*>(W + k * kH + cg * 8);
        const __nv_bfloat16* w8 = reinterpret_cast<const __nv_bfloat16*>(&wv);
        float w[8];
        #pragma unroll
        for (int c = 0; c < 8; c++) w[c] = __bfloat162float(w8[c]);
        #pragma unroll
        for (int r = 0; r < RPT; r++) {
            const float a = in[(rg * RPT + r) * ldi + k];
            #pragma unroll
            for (int c = 0; c < 8; c++) acc[r][c] = fmaf(a, w[c], acc[r][c]);
        }
    }
    #pragma unroll
    for (int r = 0; r < RPT; r++)
        #pragma unroll
        for (int c = 0; c < 8; c++) {
            const int row = rg * RPT + r, col = cg * 8 + c;
            if (z) z[row * kH + col] = acc[r][c];
            out[row * ldo + col] = act ? rbf(silu_f(acc[r][c])) : acc[r][c];
        }
}

// ---------------------------------------------------------------------------------
// inference: persistent CTAs over 64-row tiles
// ---------------------------------------------------------------------------------
constexpr int kFwdRows = 64;
constexpr size_t kFwdSmem = sizeof(__nv_bfloat16) * kNParamsPad + sizeof(float) * (3 * kH + 3 + 1) +
                            2 * sizeof(float) * kFwdRows * kH;

__global__ void __launch_bounds__(256)
mlp_forward_kernel(int n, const float* __restrict__ desc, const float* __restrict__ norm,
                   const float* __restrict__ P, const float* __restrict__ basis, float* __restrict__ out)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* sW = reinterpret_cast<__nv_bfloat16*>(smem);
    float* sB = reinterpret_cast<float*>(smem + sizeof(__nv_bfloat16) * kNParamsPad);
    float* A = sB + 3 * kH + 4;
    float* B = A + kFwdRows * kH;
    stage_params(P, sW, sB);
    __syncthreads();
    for (int tile = blockIdx.x; tile * kFwdRows < n; tile += gridDim.x) {
        const int r0 = tile * kFwdRows;
        for (int e = threadIdx.x; e < kFwdRows * kNDesc; e += blockDim.x) {
            const int r = e / kNDesc, c = e % kNDesc;
            const float x = r0 + r < n ? (desc[(size_t)(r0 + r) * kNDesc + c] - norm[c]) * norm[kNDesc + c] : 0.0f;
            A[r * kH + c] = rbf(x);
        }
        __syncthreads();
        dense128<kFwdRows, 64>(A, kH, sW + kOW1, sB, B, kH, nullptr, true);
        __syncthreads();
        dense128<kFwdRows, kH>(B, kH, sW + kOW2, sB + kH, A, kH, nullptr, true);
        __syncthreads();
        dense128<kFwdRows, kH>(A, kH, sW + kOW3, sB + 2 * kH, B, kH, nullptr, true);
        __syncthreads();
        float* Y = A;                                  // the 64 x 3 outputs (A is free)
        for (int e = threadIdx.x; e < kFwdRows * 3; e += blockDim.x) {
            const int r = e / 3, c = e % 3;
            float acc = sB[3 * kH + c];
            for (int k = 0; k < kH; k++) acc = fmaf(B[r * kH + k], __bfloat162float(sW[kOW4 + k * 3 + c]), acc);
            Y[e] = acc;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < kFwdRows * 3; e += blockDim.x) {
            const int r = e / 3, c = e % 3;
            if (r0 + r >= n) continue;
            float v = Y[e];
            if (basis) {                               // displacement = sum_m y_m B_m
                const float* Bm = basis + (size_t)(r0 + r) * 9;
                v = Y[r * 3 + 0] * Bm[c] + Y[r * 3 + 1] * Bm[3 + c] + Y[r * 3 + 2] * Bm[6 + c];
            }
            out[(size_t)(r0 + r) * 3 + c] = v;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------
// inference on the tensor cores (tcgen05): persistent CTAs over 128-row tiles
// ---------------------------------------------------------------------------------
// Per tile, layers 1-3 are D[128 x 128] = A[128 x K] W^T issued by one thread as K/16
// tcgen05.mma (kind::f16, BF16 operands from shared memory, FP32 accumulator in TMEM);
// eight warps read the accumulator back (warp w: TMEM lanes 32 (w % 4).., columns
// 64 (w / 4)..), add the bias, apply SiLU, round to BF16 and write the next layer's A
// operand; layer 4 (128 -> 3) and the readout run on the FP32 pipe from those registers.
// A CTA runs two such groups of eight warps on alternate tiles, each with its own TMEM
// columns, operand buffers and mbarrier, so that one group's epilogue overlaps the other's
// MMAs.  Operands use the canonical K-major layout without swizzle: 8-row x 16-byte core
// matrices, the two core matrices of one 16-wide K step 128 bytes apart (leading byte
// offset), 8-row groups K * 16 bytes apart (stride byte offset).
constexpr int kTcRows = 128;
constexpr int kTcGroups = 2;
constexpr int kTcGroupThreads = 256;
constexpr int kTcThreads = kTcGroups * kTcGroupThreads;
constexpr uint32_t kTcW1 = 0;                            // 128 x 64 BF16, B operand of layer 1
constexpr uint32_t kTcW2 = kTcW1 + 128 * 64 * 2;         // 128 x 128
constexpr uint32_t kTcW3 = kTcW2 + 128 * 128 * 2;
constexpr uint32_t kTcA0 = kTcW3 + 128 * 128 * 2;        // per group: 128 x 64 input rows
constexpr uint32_t kTcH = kTcA0 + kTcGroups * 128 * 64 * 2;   // per group: 128 x 128 hidden rows
constexpr uint32_t kTcW4 = kTcH + kTcGroups * 128 * 128 * 2;  // float [128][3]
constexpr uint32_t kTcBias = kTcW4 + 128 * 3 * 4;        // float [3 * 128 + 3]
constexpr uint32_t kTcPart = kTcBias + (3 * 128 + 4) * 4; // per group float [128][4]: upper-half partials
constexpr uint32_t kTcBar = kTcPart + kTcGroups * 128 * 4 * 4;  // per group mbarrier
constexpr uint32_t kTcSlot = kTcBar + 8 * kTcGroups;     // TMEM address from tcgen05.alloc
constexpr size_t kTcSmem = kTcSlot + 8 + 1024;           // + alignment of the base to 1 KB
constexpr uint32_t kTmemCols = 128 * kTcGroups;
// instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, N = 128, M = 128
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);
constexpr long kTcWaitLimit = 1L << 20;                  // try_wait polls before giving up

__device__ int g_mlp_fault = 0;                          // a tensor-core wait gave up

__device__ __forceinline__ uint32_t core_off(int r, int k, int K)
{
    return (uint32_t)((r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor: start, leading byte offset 128, stride byte offset K * 16,
// descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t saddr, int K)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) |
           ((uint64_t)((K * 16) >> 4) << 32) | (1ull << 46);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
                 :: "r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void tc_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(bar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// bounded wait for phase `parity` of the mbarrier
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity)
{
    for (long i = 0; i < kTcWaitLimit; i++) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, p;\n\t}\n" : "=r"(done) : "r"(bar), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

// 32 consecutive accumulator columns of this thread's TMEM lane
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float* v)
{
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
                 "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
                   "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
                   "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
    #pragma unroll
    for (int k = 0; k < 32; k++) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// B operand of one layer: element (n = output, k = input) = W[k][n] as BF16, core layout
__device__ void tc_stage_weights(const float* __restrict__ P, int off, int K, unsigned char* dst)
{
    for (int e = threadIdx.x; e < K * 128; e += blockDim.x) {
        const int k = e >> 7, n = e & 127;
        *reinterpret_cast<__nv_bfloat16*>(dst + core_off(n, k, K)) = __float2bfloat16_rn(P[off + k * kH + n]);
    }
}

// barrier of one group of kTcGroupThreads threads (named barrier 1 + g); returns the AND
// of `pred` over the group
__device__ __forceinline__ bool group_sync_and(int g, bool pred)
{
    uint32_t r;
    asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\t"
                 "bar.red.and.pred p, %2, %3, q;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
                 : "=r"(r) : "r"((uint32_t)pred), "r"(1 + g), "r"(kTcGroupThreads) : "memory");
    return r != 0;
}

__device__ __forceinline__ void group_sync(int g)
{
    asm volatile("bar.sync %0, %1;" :: "r"(1 + g), "r"(kTcGroupThreads) : "memory");
}

__global__ void __launch_bounds__(kTcThreads, 1)
mlp_forward_tc_kernel(int n, const float* __restrict__ desc, const float* __restrict__ norm,
                      const float* __restrict__ P, const float* __restrict__ basis, float* __restrict__ out)
{
    extern __shared__ unsigned char smem_raw[];
    const uint32_t raw = (uint32_t)__cvta_generic_to_shared(smem_raw);
    const uint32_t pad = ((raw + 1023u) & ~1023u) - raw;
    unsigned char* sm = smem_raw + pad;
    const uint32_t sb = raw + pad;
    const int tid = threadIdx.x, lane = tid & 31;
    const int g = tid / kTcGroupThreads, gt = tid % kTcGroupThreads, gwarp = gt >> 5;
    float* sW4 = reinterpret_cast<float*>(sm + kTcW4);
    float* sBias = reinterpret_cast<float*>(sm + kTcBias);
    float* sPart = reinterpret_cast<float*>(sm + kTcPart) + g * 128 * 4;
    uint32_t* slot = reinterpret_cast<uint32_t*>(sm + kTcSlot);
    const uint32_t bar = sb + kTcBar + 8 * g;
    const uint32_t a0 = kTcA0 + g * 128 * 64 * 2, hb = kTcH + g * 128 * 128 * 2;

    tc_stage_weights(P, kOW1, 64, sm + kTcW1);
    tc_stage_weights(P, kOW2, kH, sm + kTcW2);
    tc_stage_weights(P, kOW3, kH, sm + kTcW3);
    for (int e = tid; e < kH * 3; e += blockDim.x) sW4[e] = rbf(P[kOW4 + e]);
    for (int k = tid; k < 3 * kH + 3; k += blockDim.x) {
        const int o = k < kH ? kOB1 + k : (k < 2 * kH ? kOB2 + k - kH : (k < 3 * kH ? kOB3 + k - 2 * kH : kOB4 + k - 3 * kH));
        sBias[k] = P[o];
    }
    if (gt == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (tid < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(sb + kTcSlot), "r"(kTmemCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot + 128u * g;             // this group's accumulator columns
    const int rq = gwarp & 3, half = gwarp >> 2;
    const int row = 32 * rq + lane;                      // tile row = TMEM lane of this thread
    const uint32_t taddr = tmem + ((uint32_t)(32 * rq) << 16) + 64 * half;
    uint32_t parity = 0;
    bool ok = true;

    for (int tile = kTcGroups * blockIdx.x + g; tile * kTcRows < n && ok; tile += kTcGroups * gridDim.x) {
        const int r0 = tile * kTcRows;
        // input rows: standardise, round to BF16; thread = 8 consecutive features of a row,
        // neighbouring threads on neighbouring rows (conflict-free 16-byte stores)
        for (int e = gt; e < kTcRows * 8; e += kTcGroupThreads) {
            const int r = e & 127, c0 = (e >> 7) * 8;
            __align__(16) __nv_bfloat16 h[8];
            #pragma unroll
            for (int c = 0; c < 8; c++) {
                const float x = r0 + r < n ? (desc[(size_t)(r0 + r) * kNDesc + c0 + c] - norm[c0 + c]) * norm[kNDesc + c0 + c] : 0.0f;
                h[c] = __float2bfloat16_rn(x);
            }
            *reinterpret_cast<uint4*>(sm + a0 + core_off(r, c0, 64)) = *reinterpret_cast<const uint4*>(h);
        }
        for (int layer = 0; layer < 3 && ok; layer++) {
            const int K = layer == 0 ? 64 : kH;
            const uint32_t aoff = layer == 0 ? a0 : hb;
            const uint32_t woff = layer == 0 ? kTcW1 : (layer == 1 ? kTcW2 : kTcW3);
            // this thread's operand stores -> the tensor core; its earlier TMEM reads done
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            tc_fence_before();
            group_sync(g);
            if (gt == 0) {
                tc_fence_after();
                for (int kk = 0; kk < K / 16; kk++)
                    tc_mma(tmem, kmajor_desc(sb + aoff + 256 * kk, K), kmajor_desc(sb + woff + 256 * kk, K), kTcIdesc,
                           kk > 0 ? 1u : 0u);
                tc_commit(bar);
            }
            const bool mine = tc_wait(bar, parity);
            parity ^= 1u;
            ok = group_sync_and(g, mine);
            if (!ok) break;
            tc_fence_after();
            float v[64];
            tc_ld32(taddr, v);
            tc_ld32(taddr + 32, v + 32);
            tc_wait_ld();
            const float* bias = sBias + layer * kH + 64 * half;
            if (layer < 2) {
                // the MMA that read the hidden rows has completed: overwrite them
                #pragma unroll
                for (int c8 = 0; c8 < 8; c8++) {
                    __align__(16) __nv_bfloat16 h[8];
                    #pragma unroll
                    for (int c = 0; c < 8; c++) h[c] = __float2bfloat16_rn(silu_f(v[8 * c8 + c] + bias[8 * c8 + c]));
                    *reinterpret_cast<uint4*>(sm + hb + core_off(row, 64 * half + 8 * c8, kH)) =
                        *reinterpret_cast<const uint4*>(h);
                }
            } else {
                // layer 4 on this thread's 64 hidden values, the halves summed in shared memory
                float y0 = 0.0f, y1 = 0.0f, y2 = 0.0f;
                #pragma unroll
                for (int c = 0; c < 64; c++) {
                    const float h = rbf(silu_f(v[c] + bias[c]));
                    const float* w = sW4 + (64 * half + c) * 3;
                    y0 = fmaf(h, w[0], y0);
                    y1 = fmaf(h, w[1], y1);
                    y2 = fmaf(h, w[2], y2);
                }
                if (half == 1) {
                    sPart[row * 4 + 0] = y0;
                    sPart[row * 4 + 1] = y1;
                    sPart[row * 4 + 2] = y2;
                }
                group_sync(g);
                if (half == 0 && r0 + row < n) {
                    float y[3] = {sBias[3 * kH + 0] + y0 + sPart[row * 4 + 0], sBias[3 * kH + 1] + y1 + sPart[row * 4 + 1],
                                  sBias[3 * kH + 2] + y2 + sPart[row * 4 + 2]};
                    const size_t gr = (size_t)(r0 + row);
                    if (basis) {                         // displacement = sum_m y_m B_m
                        const float* Bm = basis + gr * 9;
                        #pragma unroll
                        for (int c = 0; c < 3; c++)
                            out[gr * 3 + c] = y[0] * Bm[c] + y[1] * Bm[3 + c] + y[2] * Bm[6 + c];
                    } else {
                        #pragma unroll
                        for (int c = 0; c < 3; c++) out[gr * 3 + c] = y[c];
                    }
                }
            }
        }
    }
    if (!ok && gt == 0) {
        // a wait gave up: record it, give the tensor core a bounded time to finish the
        // committed work before the accumulator columns are freed
        atomicExch(&g_mlp_fault, 1);
        tc_wait(bar, parity ^ 1u);
    }
    tc_fence_before();
    __syncthreads();
    if (tid < 32) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(*slot), "r"(kTmemCols) : "memory");
    }
}

// ---------------------------------------------------------------------------------
// training: per 32-row tile forward with caches, backward, partial gradients per tile
// ---------------------------------------------------------------------------------
constexpr int kTrRows = 32;
constexpr size_t kTrSmem = sizeof(__nv_bfloat16) * kNParamsPad + sizeof(float) * (3 * kH + 4) +
                           sizeof(float) * (kTrRows * kH            // X (stride kH)
                                            + 3 * kTrRows * kH      // H1..H3
                                            + 3 * kTrRows * kH      // Z1..Z3, then dZ
                                            + kTrRows * kH          // dH scratch
                                            + kTrRows * 4);         // dZ4

// g[k][c] (+)= sum_r H[r][k] dZ[r][c] for a K x 128 block, written to gout (K*128 floats)
template <int K>
__device__ void wgrad128(const float* H, const float* dZ, float* gout)
{
    // thread t: k rows (t / 16) * (K / 16) .. , cols (t % 16) * 8 ..
    constexpr int KPT = K / 16;
    const int kg = threadIdx.x >> 4, cg = threadIdx.x & 15;
    float acc[KPT][8];
    #pragma unroll
    for (int a = 0; a < KPT; a++)
        #pragma unroll
        for (int c = 0; c < 8; c++) acc[a][c] = 0.0f;
    for (int r = 0; r < kTrRows; r++) {
        float d[8];
        #pragma unroll
        for (int c = 0; c < 8; c++) d[c] = dZ[r * kH + cg * 8 + c];
        #pragma unroll
        for (int a = 0; a < KPT; a++) {
            const float h = H[r * kH + kg * KPT + a];
            #pragma unroll
            for (int c = 0; c < 8; c++) acc[a][c] = fmaf(h, d[c], acc[a][c]);
        }
    }
    #pragma unroll
    for (int a = 0; a < KPT; a++)
        #pragma unroll
        for (int c = 0; c < 8; c++) gout[(kg * KPT + a) * kH + cg * 8 + c] = acc[a][c];
}

// dH[r][k] = sum_c dZ[r][c] W[k][c] (W is K x 128), then dZ_prev = dH * silu'(Z) in place
// of Z; when Z is null dH is returned as is.
__device__ void back128(const float* dZ, const __nv_bfloat16* W, int K, float* Z)
{
    for (int e = threadIdx.x; e < kTrRows * K; e += blockDim.x) {
        const int r = e / K, k = e % K;
        float acc = 0.0f;
        for (int c = 0; c < kH; c++) acc = fmaf(dZ[r * kH + c], __bfloat162float(W[k * kH + c]), acc);
        const float z = Z[r * kH + k];
        const float s = 1.0f / (1.0f + __expf(-z));
        Z[r * kH + k] = acc * (s * (1.0f + z * (1.0f - s)));
    }
}

__global__ void __launch_bounds__(256)
mlp_train_tile_kernel(int n, const float* __restrict__ desc, const float* __restrict__ target,
                      const float* __restrict__ norm, const float* __restrict__ P,
                      const float* __restrict__ basis, float* __restrict__ gpart,
                      float* __restrict__ lpart, float scale)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* sW = reinterpret_cast<__nv_bfloat16*>(smem);
    float* sB = reinterpret_cast<float*>(smem + sizeof(__nv_bfloat16) * kNParamsPad);
    float* X = sB + 3 * kH + 4;
    float* H1 = X + kTrRows * kH;
    float* H2 = H1 + kTrRows * kH;
    float* H3 = H2 + kTrRows * kH;
    float* Z1 = H3 + kTrRows * kH;
    float* Z2 = Z1 + kTrRows * kH;
    float* Z3 = Z2 + kTrRows * kH;
    float* T = Z3 + kTrRows * kH;          // scratch (kTrRows x kH)
    float* D4 = T + kTrRows * kH;          // dZ4 (kTrRows x 4)
    stage_params(P, sW, sB);
    const int r0 = blockIdx.x * kTrRows;
    for (int e = threadIdx.x; e < kTrRows * kH; e += blockDim.x) {
        const int r = e / kH, c = e % kH;
        float x = 0.0f;
        if (c < kNDesc && r0 + r < n) x = (desc[(size_t)(r0 + r) * kNDesc + c] - norm[c]) * norm[kNDesc + c];
        X[e] = c < kNDesc ? rbf(x) : 0.0f;
    }
    __syncthreads();
    dense128<kTrRows, 64>(X, kH, sW + kOW1, sB, H1, kH, Z1, true);
    __syncthreads();
    dense128<kTrRows, kH>(H1, kH, sW + kOW2, sB + kH, H2, kH, Z2, true);
    __syncthreads();
    dense128<kTrRows, kH>(H2, kH, sW + kOW3, sB + 2 * kH, H3, kH, Z3, true);
    __syncthreads();
    // output layer (outputs into T's first columns), the prediction p = y or sum_m y_m B_m,
    // its error; dZ4 = scale * (dp/dy)^T (p - t) for real rows, 0 for padding
    for (int e = threadIdx.x; e < kTrRows * 3; e += blockDim.x) {
        const int r = e / 3, c = e % 3;
        float acc = sB[3 * kH + c];
        for (int k = 0; k < kH; k++) acc = fmaf(H3[r * kH + k], __bfloat162float(sW[kOW4 + k * 3 + c]), acc);
        T[r * 4 + c] = acc;
    }
    __syncthreads();
    float lsum = 0.0f;
    for (int r = threadIdx.x; r < kTrRows; r += blockDim.x) {
        float d[3] = {0.0f, 0.0f, 0.0f};
        if (r0 + r < n) {
            const float* y = T + r * 4;
            const float* t = target + (size_t)(r0 + r) * 3;
            if (basis) {
                const float* Bm = basis + (size_t)(r0 + r) * 9;
                for (int c = 0; c < 3; c++) {
                    d[c] = y[0] * Bm[c] + y[1] * Bm[3 + c] + y[2] * Bm[6 + c] - t[c];
                    lsum += d[c] * d[c];
                }
                float g[3];
                for (int mm = 0; mm < 3; mm++) g[mm] = Bm[3 * mm] * d[0] + Bm[3 * mm + 1] * d[1] + Bm[3 * mm + 2] * d[2];
                d[0] = g[0];
                d[1] = g[1];
                d[2] = g[2];
            } else {
                for (int c = 0; c < 3; c++) {
                    d[c] = y[c] - t[c];
                    lsum += d[c] * d[c];
                }
            }
        }
        for (int c = 0; c < 3; c++) D4[r * 4 + c] = scale * d[c];
    }
    // loss partial of this tile (block reduction in fixed order)
    __shared__ float s_red[256];
    s_red[threadIdx.x] = lsum;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int k = 0; k < (int)blockDim.x; k++) t += s_red[k];
        lpart[blockIdx.x] = t;
    }
    float* G = gpart + (size_t)blockIdx.x * kNParams;
    // W4 (128 x 3), b4
    for (int e = threadIdx.x; e < kH * 3 + 3; e += blockDim.x) {
        float acc = 0.0f;
        if (e < kH * 3) {
            const int k = e / 3, c = e % 3;
            for (int r = 0; r < kTrRows; r++) acc = fmaf(H3[r * kH + k], D4[r * 4 + c], acc);
            G[kOW4 + e] = acc;
        } else {
            const int c = e - kH * 3;
            for (int r = 0; r < kTrRows; r++) acc += D4[r * 4 + c];
            G[kOB4 + c] = acc;
        }
    }
    // dZ3 = (dZ4 W4^T) * silu'(Z3), in Z3
    for (int e = threadIdx.x; e < kTrRows * kH; e += blockDim.x) {
        const int r = e / kH, k = e % kH;
        float acc = 0.0f;
        for (int c = 0; c < 3; c++) acc = fmaf(D4[r * 4 + c], __bfloat162float(sW[kOW4 + k * 3 + c]), acc);
        const float z = Z3[e];
        const float s = 1.0f / (1.0f + __expf(-z));
        Z3[e] = acc * (s * (1.0f + z * (1.0f - s)));
    }
    __syncthreads();
    wgrad128<kH>(H2, Z3, G + kOW3);
    for (int c = threadIdx.x; c < kH; c += blockDim.x) {
        float acc = 0.0f;
        for (int r = 0; r < kTrRows; r++) acc += Z3[r * kH + c];
        G[kOB3 + c] = acc;
    }
    back128(Z3, sW + kOW3, kH, Z2);                  // dZ2 in Z2
    __syncthreads();
    wgrad128<kH>(H1, Z2, G + kOW2);
    for (int c = threadIdx.x; c < kH; c += blockDim.x) {
        float acc = 0.0f;
        for (int r = 0; r < kTrRows; r++) acc += Z2[r * kH + c];
        G[kOB2 + c] = acc;
    }
    back128(Z2, sW + kOW2, kH, Z1);                  // dZ1 in Z1
    __syncthreads();
    wgrad128<64>(X, Z1, G + kOW1);
    for (int c = threadIdx.x; c < kH; c += blockDim.x) {
        float acc = 0.0f;
        for (int r = 0; r < kTrRows; r++) acc += Z1[r * kH + c];
        G[kOB1 + c] = acc;
    }
}

// gradient = sum over tiles in tile order; then one Adam step on the FP32 parameters
__global__ void adam_kernel(int ntiles, const float* __restrict__ gpart, float* __restrict__ P,
                            float* __restrict__ m, float* __restrict__ v, float lr, float b1,
                            float b2, float eps, float c1, float c2, float* __restrict__ grad_out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= kNParams) return;
    float g = 0.0f;
    for (int t = 0; t < ntiles; t++) g += gpart[(size_t)t * kNParams + k];
    if (grad_out) grad_out[k] = g;
    if (lr == 0.0f) return;
    const float mk = b1 * m[k] + (1.0f - b1) * g;
    const float vk = b2 * v[k] + (1.0f - b2) * g * g;
    m[k] = mk;
    v[k] = vk;
    P[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
}

// ---------------------------------------------------------------------------------
// training on the tensor cores (tcgen05): one CTA per 128-row tile
// ---------------------------------------------------------------------------------
// Forward as in inference, the pre-activations Z1..Z3 left in TMEM (columns 0, 128, 256) and
// the activations X, H1, H2 kept in shared memory.  Backward: dZ4 and the layer-4 gradients
// on the FP32 pipe; for l = 3, 2, 1: dZ_l = dH_l * SiLU'(Z_l) rounded to BF16 (the tensor
// core's operand; the bias gradient sums these values), dW_l = H_{l-1}^T dZ_l and
// dH_{l-1} = dZ_l W_l^T on the tensor core (TMEM columns 384..511).  The transposed operands
// are the same shared-memory buffers read MN-major: a buffer written K-major for rows r and
// features k (core matrices of 8 r x 8 k, k contiguous) is, seen with k as the M or N index
// and r as the K index, an MN-major operand with 8-column groups 128 bytes apart (stride byte
// offset) and 8-row groups K * 16 bytes apart (leading byte offset).  dW1 is formed
// transposed (dZ1^T X: M = 128 outputs, N = 64 inputs) since M must be 128.
constexpr uint32_t kTtW1 = 0;                            // B operands of the forward
constexpr uint32_t kTtW2 = kTtW1 + 128 * 64 * 2;
constexpr uint32_t kTtW3 = kTtW2 + 128 * 128 * 2;
constexpr uint32_t kTtX = kTtW3 + 128 * 128 * 2;         // 128 x 64 input rows
constexpr uint32_t kTtH1 = kTtX + 128 * 64 * 2;          // 128 x 128
constexpr uint32_t kTtH2 = kTtH1 + 128 * 128 * 2;
constexpr uint32_t kTtDZ = kTtH2 + 128 * 128 * 2;        // H3, then dZ3, dZ2, dZ1 (BF16)
constexpr uint32_t kTtW4 = kTtDZ + 128 * 128 * 2;        // float [128][3]
constexpr uint32_t kTtBias = kTtW4 + 128 * 3 * 4;        // float [3 * 128 + 3]
constexpr uint32_t kTtD4 = kTtBias + (3 * 128 + 4) * 4;  // float [128][4]: dZ4 (and half sums)
constexpr uint32_t kTtRed = kTtD4 + 128 * 4 * 4;         // float [8]: loss partials per warp
constexpr uint32_t kTtBar = kTtRed + 8 * 4;
constexpr uint32_t kTtSlot = kTtBar + 8;
constexpr size_t kTtSmem = kTtSlot + 8 + 1024;
constexpr int kTtThreads = 256;
constexpr uint32_t kTtCols = 512;
// instruction descriptors (FP32 accumulator, BF16 operands, M = 128): forward (A, B K-major),
// weight gradient (A, B MN-major), input gradient (A K-major, B MN-major); N = 128 or 64
__host__ __device__ constexpr uint32_t tt_idesc(uint32_t a_mn, uint32_t b_mn, uint32_t N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (a_mn << 15) | (b_mn << 16) | ((N >> 3) << 17) | ((128u >> 4) << 24);
}

// MN-major view of a K-major buffer with Kb features per row: leading byte offset Kb * 16
// (8-row groups), stride byte offset 128 (8-feature groups)
__device__ __forceinline__ uint64_t mn_desc(uint32_t saddr, int Kb)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((Kb * 16) >> 4) << 16) |
           ((uint64_t)(128 >> 4) << 32) | (1ull << 46);
}

// `steps` MMAs by thread 0 (descriptor start advanced by a_step / b_step bytes per step),
// commit, bounded wait; false (on every thread) when the wait gave up
__device__ __forceinline__ bool tt_gemm(uint32_t d, uint64_t a, uint32_t a_step, uint64_t b, uint32_t b_step,
                                        int steps, uint32_t idesc, uint32_t bar, uint32_t& parity)
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0) {
        tc_fence_after();
        for (int kk = 0; kk < steps; kk++)
            tc_mma(d, a + (uint64_t)((a_step * kk) >> 4), b + (uint64_t)((b_step * kk) >> 4), idesc, kk > 0 ? 1u : 0u);
        tc_commit(bar);
    }
    const bool mine = tc_wait(bar, parity);
    parity ^= 1u;
    const bool ok = __syncthreads_and(mine) != 0;
    tc_fence_after();
    return ok;
}

__device__ __forceinline__ float silu_grad(float z)
{
    const float sg = z < -80.0f ? 0.0f : __fdividef(1.0f, 1.0f + __expf(-z));
    return sg * (1.0f + z * (1.0f - sg));
}

__device__ __forceinline__ float bf16_at(const unsigned char* buf, int r, int k, int K)
{
    return __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(buf + core_off(r, k, K)));
}

__global__ void __launch_bounds__(kTtThreads, 1)
mlp_train_tc_kernel(int n, const float* __restrict__ desc, const float* __restrict__ target,
                    const float* __restrict__ norm, const float* __restrict__ P,
                    const float* __restrict__ basis, float* __restrict__ gpart,
                    float* __restrict__ lpart, float scale)
{
    extern __shared__ unsigned char smem_raw[];
    const uint32_t raw = (uint32_t)__cvta_generic_to_shared(smem_raw);
    const uint32_t pad = ((raw + 1023u) & ~1023u) - raw;
    unsigned char* sm = smem_raw + pad;
    const uint32_t sb = raw + pad;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    float* sW4 = reinterpret_cast<float*>(sm + kTtW4);
    float* sBias = reinterpret_cast<float*>(sm + kTtBias);
    float* sD4 = reinterpret_cast<float*>(sm + kTtD4);
    float* sRed = reinterpret_cast<float*>(sm + kTtRed);
    uint32_t* slot = reinterpret_cast<uint32_t*>(sm + kTtSlot);
    const uint32_t bar = sb + kTtBar;
    const int r0 = blockIdx.x * kTcRows;
    float* G = gpart + (size_t)blockIdx.x * kNParams;

    tc_stage_weights(P, kOW1, 64, sm + kTtW1);
    tc_stage_weights(P, kOW2, kH, sm + kTtW2);
    tc_stage_weights(P, kOW3, kH, sm + kTtW3);
    for (int e = tid; e < kH * 3; e += blockDim.x) sW4[e] = rbf(P[kOW4 + e]);
    for (int k = tid; k < 3 * kH + 3; k += blockDim.x) {
        const int o = k < kH ? kOB1 + k : (k < 2 * kH ? kOB2 + k - kH : (k < 3 * kH ? kOB3 + k - 2 * kH : kOB4 + k - 3 * kH));
        sBias[k] = P[o];
    }
    for (int e = tid; e < kTcRows * 8; e += blockDim.x) {
        const int r = e & 127, c0 = (e >> 7) * 8;
        __align__(16) __nv_bfloat16 h[8];
        #pragma unroll
        for (int c = 0; c < 8; c++) {
            const float x = r0 + r < n ? (desc[(size_t)(r0 + r) * kNDesc + c0 + c] - norm[c0 + c]) * norm[kNDesc + c0 + c] : 0.0f;
            h[c] = __float2bfloat16_rn(x);
        }
        *reinterpret_cast<uint4*>(sm + kTtX + core_off(r, c0, 64)) = *reinterpret_cast<const uint4*>(h);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(sb + kTtSlot), "r"(kTtCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot;
    const int rq = warp & 3, half = warp >> 2;
    const int row = 32 * rq + lane;                      // TMEM lane of this thread
    const uint32_t lane_base = tmem + ((uint32_t)(32 * rq) << 16);
    uint32_t parity = 0;
    bool ok = true;
    const uint32_t kFwd = tt_idesc(0, 0, 128), kWgt = tt_idesc(1, 1, 128), kInp = tt_idesc(0, 1, 128),
                   kWgt64 = tt_idesc(1, 1, 64);

    // ---- forward: Z_l in TMEM columns 128 (l - 1); H1, H2 and then H3 (in the dZ buffer)
    for (int layer = 0; layer < 3 && ok; layer++) {
        const int K = layer == 0 ? 64 : kH;
        const uint32_t aoff = layer == 0 ? kTtX : (layer == 1 ? kTtH1 : kTtH2);
        const uint32_t woff = layer == 0 ? kTtW1 : (layer == 1 ? kTtW2 : kTtW3);
        const uint32_t outb = layer == 0 ? kTtH1 : (layer == 1 ? kTtH2 : kTtDZ);
        ok = tt_gemm(tmem + 128 * layer, kmajor_desc(sb + aoff, K), 256, kmajor_desc(sb + woff, K), 256, K / 16, kFwd,
                     bar, parity);
        if (!ok) break;
        float y0 = 0.0f, y1 = 0.0f, y2 = 0.0f;
        for (int ch = 0; ch < 2; ch++) {
            const int c0 = 64 * half + 32 * ch;
            float v[32];
            tc_ld32(lane_base + 128 * layer + c0, v);
            tc_wait_ld();
            #pragma unroll
            for (int c8 = 0; c8 < 4; c8++) {
                __align__(16) __nv_bfloat16 h[8];
                #pragma unroll
                for (int c = 0; c < 8; c++) {
                    const int k = c0 + 8 * c8 + c;
                    h[c] = __float2bfloat16_rn(silu_f(v[8 * c8 + c] + sBias[layer * kH + k]));
                    if (layer == 2) {
                        const float hv = __bfloat162float(h[c]);
                        y0 = fmaf(hv, sW4[k * 3 + 0], y0);
                        y1 = fmaf(hv, sW4[k * 3 + 1], y1);
                        y2 = fmaf(hv, sW4[k * 3 + 2], y2);
                    }
                }
                *reinterpret_cast<uint4*>(sm + outb + core_off(row, c0 + 8 * c8, kH)) = *reinterpret_cast<const uint4*>(h);
            }
        }
        if (layer == 2) {
            // outputs, loss and dZ4 (upper column half's sums through shared memory)
            if (half == 1) {
                sD4[row * 4 + 0] = y0;
                sD4[row * 4 + 1] = y1;
                sD4[row * 4 + 2] = y2;
            }
            __syncthreads();
            float l2 = 0.0f;
            if (half == 0) {
                float y[3] = {sBias[3 * kH + 0] + y0 + sD4[row * 4 + 0], sBias[3 * kH + 1] + y1 + sD4[row * 4 + 1],
                              sBias[3 * kH + 2] + y2 + sD4[row * 4 + 2]};
                float d[3] = {0.0f, 0.0f, 0.0f};
                if (r0 + row < n) {
                    const size_t gr = (size_t)(r0 + row);
                    const float* t = target + gr * 3;
                    if (basis) {
                        const float* Bm = basis + gr * 9;
                        float e[3];
                        for (int c = 0; c < 3; c++) {
                            e[c] = y[0] * Bm[c] + y[1] * Bm[3 + c] + y[2] * Bm[6 + c] - t[c];
                            l2 += e[c] * e[c];
                        }
                        for (int m = 0; m < 3; m++) d[m] = Bm[3 * m] * e[0] + Bm[3 * m + 1] * e[1] + Bm[3 * m + 2] * e[2];
                    } else {
                        for (int c = 0; c < 3; c++) {
                            d[c] = y[c] - t[c];
                            l2 += d[c] * d[c];
                        }
                    }
                }
                __syncwarp();
                for (int c = 0; c < 3; c++) sD4[row * 4 + c] = scale * d[c];
                // loss partial of this warp in lane order, then warps in order
                for (int o = 16; o > 0; o >>= 1) l2 += __shfl_down_sync(0xffffffffu, l2, o);
                if (lane == 0) sRed[rq] = l2;
            }
            __syncthreads();
            if (tid == 0) lpart[blockIdx.x] = (sRed[0] + sRed[1]) + (sRed[2] + sRed[3]);
        }
    }
    if (ok) {
        // ---- layer 4: dW4 = H3^T dZ4, db4 (rows in order), from the H3 copy in the dZ buffer
        for (int e = tid; e < kH * 3 + 3; e += blockDim.x) {
            float acc = 0.0f;
            if (e < kH * 3) {
                const int k = e / 3, c = e % 3;
                for (int r = 0; r < kTcRows; r++) acc = fmaf(bf16_at(sm + kTtDZ, r, k, kH), sD4[r * 4 + c], acc);
                G[kOW4 + e] = acc;
            } else {
                for (int r = 0; r < kTcRows; r++) acc += sD4[r * 4 + e - kH * 3];
                G[kOB4 + e - kH * 3] = acc;
            }
        }
        __syncthreads();
        // dZ3 = (dZ4 W4^T) SiLU'(Z3), BF16, over the H3 copy
        for (int ch = 0; ch < 2; ch++) {
            const int c0 = 64 * half + 32 * ch;
            float z[32];
            tc_ld32(lane_base + 256 + c0, z);
            tc_wait_ld();
            const float d0 = sD4[row * 4 + 0], d1 = sD4[row * 4 + 1], d2 = sD4[row * 4 + 2];
            #pragma unroll
            for (int c8 = 0; c8 < 4; c8++) {
                __align__(16) __nv_bfloat16 h[8];
                #pragma unroll
                for (int c = 0; c < 8; c++) {
                    const int k = c0 + 8 * c8 + c;
                    const float dh = fmaf(d2, sW4[k * 3 + 2], fmaf(d1, sW4[k * 3 + 1], d0 * sW4[k * 3 + 0]));
                    h[c] = __float2bfloat16_rn(dh * silu_grad(z[8 * c8 + c] + sBias[2 * kH + k]));
                }
                *reinterpret_cast<uint4*>(sm + kTtDZ + core_off(row, c0 + 8 * c8, kH)) = *reinterpret_cast<const uint4*>(h);
            }
        }
    }
    // ---- layers 3, 2, 1
    for (int layer = 2; layer >= 0 && ok; layer--) {
        const int K = layer == 0 ? 64 : kH;                  // inputs of this layer
        const uint32_t hin = layer == 0 ? kTtX : (layer == 1 ? kTtH1 : kTtH2);
        const uint32_t w = layer == 0 ? kTtW1 : (layer == 1 ? kTtW2 : kTtW3);
        const int ow = layer == 0 ? kOW1 : (layer == 1 ? kOW2 : kOW3);
        const int ob = layer == 0 ? kOB1 : (layer == 1 ? kOB2 : kOB3);
        __syncthreads();
        // bias gradient: column sums of the BF16 dZ, rows in order
        for (int k = tid; k < kH; k += blockDim.x) {
            float acc = 0.0f;
            for (int r = 0; r < kTcRows; r++) acc += bf16_at(sm + kTtDZ, r, k, kH);
            G[ob + k] = acc;
        }
        if (layer > 0) {
            // dW = H^T dZ: M = inputs, N = outputs, K = rows
            ok = tt_gemm(tmem + 384, mn_desc(sb + hin, K), 2 * K * 16, mn_desc(sb + kTtDZ, kH), 2 * kH * 16,
                         kTcRows / 16, kWgt, bar, parity);
            if (!ok) break;
            for (int ch = 0; ch < 2; ch++) {
                const int c0 = 64 * half + 32 * ch;
                float v[32];
                tc_ld32(lane_base + 384 + c0, v);
                tc_wait_ld();
                float* dst = G + ow + row * kH + c0;           // input `row`, outputs c0 ..
                #pragma unroll
                for (int c = 0; c < 32; c++) dst[c] = v[c];
            }
            // dH = dZ W^T: M = rows, N = inputs, K = outputs; then dZ of the layer below
            ok = tt_gemm(tmem + 384, kmajor_desc(sb + kTtDZ, kH), 256, mn_desc(sb + w, K), 2 * K * 16, kH / 16, kInp,
                         bar, parity);
            if (!ok) break;
            for (int ch = 0; ch < 2; ch++) {
                const int c0 = 64 * half + 32 * ch;
                float dh[32], z[32];
                tc_ld32(lane_base + 384 + c0, dh);
                tc_ld32(lane_base + 128 * (layer - 1) + c0, z);
                tc_wait_ld();
                #pragma unroll
                for (int c8 = 0; c8 < 4; c8++) {
                    __align__(16) __nv_bfloat16 h[8];
                    #pragma unroll
                    for (int c = 0; c < 8; c++) {
                        const int k = c0 + 8 * c8 + c;
                        h[c] = __float2bfloat16_rn(dh[8 * c8 + c] * silu_grad(z[8 * c8 + c] + sBias[(layer - 1) * kH + k]));
                    }
                    *reinterpret_cast<uint4*>(sm + kTtDZ + core_off(row, c0 + 8 * c8, kH)) = *reinterpret_cast<const uint4*>(h);
                }
            }
        } else {
            // dW1^T = dZ1^T X: M = outputs (128), N = inputs (64), K = rows
            ok = tt_gemm(tmem + 384, mn_desc(sb + kTtDZ, kH), 2 * kH * 16, mn_desc(sb + kTtX, 64), 2 * 64 * 16,
                         kTcRows / 16, kWgt64, bar, parity);
            if (!ok) break;
            float v[32];
            tc_ld32(lane_base + 384 + 32 * half, v);         // output `row`, inputs 32 half ..
            tc_wait_ld();
            #pragma unroll
            for (int c = 0; c < 32; c++) G[kOW1 + (32 * half + c) * kH + row] = v[c];
        }
    }
    if (!ok && tid == 0) {
        atomicExch(&g_mlp_fault, 1);
        tc_wait(bar, parity ^ 1u);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(kTtCols) : "memory");
    }
}

// ---------------------------------------------------------------------------------
// starting displacements of the walkers from the model's predictions: CTA per walker
// ---------------------------------------------------------------------------------
constexpr int kSeedThreads = 256;

// Walker s (atoms begin[s] .. begin[s+1]-1): its eligible atoms are those whose predicted
// displacement is at least min_disp long; the candidates are the eligible atoms whose score
// is at least threshold * (the largest score of an eligible atom); with uniforms u_q of the Philox stream of
// key (seed, s) and counter (counter, 0), the chosen atom c is candidate floor(u_0 * count)
// in atom order.  disp = scale * pred[c] on c, plus noise * (z_x, z_y, z_z) on every atom
// within `radius` of c (minimum image), z = sqrt(-2 ln(1 - u_a)) cos(2 pi u_b) from the
// uniforms (a, b) = (1 + 6j, 2 + 6j), (3 + 6j, 4 + 6j), (5 + 6j, 6 + 6j) of atom j (index
// within the walker); mode = pred[c] on c, zero elsewhere.  A walker without an eligible atom
// or whose largest eligible score is below min_score gets c = -1 and zero displacement and
// mode.
__global__ void __launch_bounds__(kSeedThreads)
proposal_seeds_kernel(const long long* __restrict__ begin, const double* __restrict__ pos,
                      const double* __restrict__ box, const double* __restrict__ center,
                      const float* __restrict__ pred,
                      const float* __restrict__ score, int score_stride, akmc_proposal_params p,
                      uint64_t seed, uint64_t counter, double* __restrict__ disp,
                      double* __restrict__ mode, int* __restrict__ chosen)
{
    __shared__ float s_red[kSeedThreads / 32];
    __shared__ int s_cnt[kSeedThreads / 32];
    __shared__ int s_pick, s_total;
    __shared__ float s_max;
    const int w = blockIdx.x;
    const long long a = begin[w];
    const int n = (int)(begin[w + 1] - a);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // 1. the largest score
    // eligible atoms: predicted displacement at least min_disp long
    const float md2 = (float)(p.min_disp * p.min_disp);
    // ... and, with a centre for this walker, within `region` of it (minimum image)
    const bool local = center != nullptr && p.region > 0.0;
    const double cx0 = local ? center[3 * w] : 0.0, cy0 = local ? center[3 * w + 1] : 0.0,
                 cz0 = local ? center[3 * w + 2] : 0.0;
    const double bl0 = box[3 * w], bl1 = box[3 * w + 1], bl2 = box[3 * w + 2];
    auto eligible = [&](int j) {
        const float* q = pred + (size_t)(a + j) * 3;
        if (!(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] >= md2)) return false;
        if (!local) return true;
        double dx = pos[3 * (a + j)] - cx0, dy = pos[3 * (a + j) + 1] - cy0, dz = pos[3 * (a + j) + 2] - cz0;
        dx -= bl0 * rint(dx / bl0);
        dy -= bl1 * rint(dy / bl1);
        dz -= bl2 * rint(dz / bl2);
        return dx * dx + dy * dy + dz * dz < p.region * p.region;
    };
    float mx = -INFINITY;
    for (int j = threadIdx.x; j < n; j += blockDim.x)
        if (eligible(j)) mx = fmaxf(mx, score[(size_t)(a + j) * score_stride]);
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) s_red[warp] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        float m = -INFINITY;
        for (int k = 0; k < kSeedThreads / 32; k++) m = fmaxf(m, s_red[k]);
        s_max = m;
        s_pick = -1;
        s_total = 0;
    }
    __syncthreads();
    const float thr = (float)p.threshold * s_max;
    const bool any = n > 0 && s_max >= (float)p.min_score;
    if (any) {
        // 2. count the candidates
        int cnt = 0;
        for (int j = threadIdx.x; j < n; j += blockDim.x) cnt += eligible(j) && score[(size_t)(a + j) * score_stride] >= thr;
        for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        if (lane == 0) s_cnt[warp] = cnt;
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int k = 0; k < kSeedThreads / 32; k++) t += s_cnt[k];
            s_total = t;
        }
        __syncthreads();
        const double u0 = philox_uniform(seed, (uint64_t)w, counter, 0, 0);
        // stratified over a group of walkers on one system: walker g of the group draws from
        // the g-th of `group` equal slices of the candidate list
        const double frac = p.group > 1 ? ((double)(w % p.group) + u0) / (double)p.group : u0;
        const int want = min((int)(frac * s_total), s_total - 1);
        // 3. the want-th candidate in atom order: tiles of blockDim atoms, rank by ballots
        int seen = 0;
        for (int base = 0; base < n; base += blockDim.x) {
            const int j = base + threadIdx.x;
            const bool c = j < n && eligible(j) && score[(size_t)(a + j) * score_stride] >= thr;
            const unsigned bal = __ballot_sync(0xffffffffu, c);
            if (lane == 0) s_cnt[warp] = __popc(bal);
            __syncthreads();
            int before = seen;
            for (int k = 0; k < warp; k++) before += s_cnt[k];
            int tile = 0;
            for (int k = 0; k < kSeedThreads / 32; k++) tile += s_cnt[k];
            if (c && before + __popc(bal & ((1u << lane) - 1u)) == want) s_pick = j;
            seen += tile;
            __syncthreads();
            if (s_pick >= 0) break;
        }
    }
    __syncthreads();
    const int c = s_pick;
    if (threadIdx.x == 0) chosen[w] = c;
    double cx = 0.0, cy = 0.0, cz = 0.0;
    if (c >= 0) {
        cx = pos[3 * (a + c)];
        cy = pos[3 * (a + c) + 1];
        cz = pos[3 * (a + c) + 2];
    }
    const double L0 = box[3 * w], L1 = box[3 * w + 1], L2 = box[3 * w + 2];
    const double r2max = p.radius * p.radius;
    const double two_pi = 6.283185307179586;
    // 4. the displacement and the mode
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        double d[3] = {0.0, 0.0, 0.0}, m[3] = {0.0, 0.0, 0.0};
        if (c >= 0) {
            double dx = pos[3 * (a + j)] - cx, dy = pos[3 * (a + j) + 1] - cy, dz = pos[3 * (a + j) + 2] - cz;
            dx -= L0 * rint(dx / L0);
            dy -= L1 * rint(dy / L1);
            dz -= L2 * rint(dz / L2);
            if (p.noise > 0.0 && dx * dx + dy * dy + dz * dz < r2max) {
                for (int k = 0; k < 3; k++) {
                    const uint64_t q = 1 + 6 * (uint64_t)j + 2 * k;
                    const double ua = philox_uniform(seed, (uint64_t)w, counter, 0, q);
                    const double ub = philox_uniform(seed, (uint64_t)w, counter, 0, q + 1);
                    d[k] = p.noise * (sqrt(-2.0 * log(1.0 - ua)) * cos(two_pi * ub));
                }
            }
            if (j == c) {
                for (int k = 0; k < 3; k++) {
                    m[k] = (double)pred[(size_t)(a + j) * 3 + k];
                    d[k] += p.scale * m[k];
                }
            }
        }
        for (int k = 0; k < 3; k++) {
            disp[3 * (a + j) + k] = d[k];
            if (mode) mode[3 * (a + j) + k] = m[k];
        }
    }
}

}  // namespace

cudaError_t configure_mlp_kernels()
{
    cudaError_t e = cudaFuncSetAttribute(mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFwdSmem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(mlp_forward_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(mlp_train_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTtSmem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(mlp_train_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrSmem);
}

}  // namespace akmc

using namespace akmc;

extern "C" {

int akmc_mlp_num_params(void) { return kNParams; }

akmc_status akmc_batch_descriptors(akmc_batch* b, float* desc_dev, float* basis_dev, void* stream)
{
    if (!b || !desc_dev) return fail(AKMC_ERR_ARG, "null argument");
    if (b->field->pot.family != AKMC_FAMILY_EAM || !b->view.nbr)
        return fail(AKMC_ERR_UNSUPPORTED, "descriptors need an EAM batch with a neighbour list");
    if (b->field->pot.cutoff + b->view.skin < (double)kDescRc)
        return fail(AKMC_ERR_UNSUPPORTED, "the neighbour lists do not reach the descriptor cutoff");
    const int blocks = (b->n_total + kDescWarps - 1) / kDescWarps;
    descriptor_kernel<<<blocks, 32 * kDescWarps, 0, (cudaStream_t)stream>>>(b->view, nullptr, 0, nullptr,
                                                                           desc_dev, basis_dev);
    AKMC_CUDA(cudaGetLastError());
    return AKMC_OK;
}

akmc_status akmc_batch_descriptors_rows(akmc_batch* b, const int* rows_dev, int n_rows, float* desc_dev,
                                        float* basis_dev, void* stream)
{
    if (!b || n_rows < 0 || (n_rows > 0 && (!rows_dev || !desc_dev))) return fail(AKMC_ERR_ARG, "bad arguments");
    if (b->field->pot.family != AKMC_FAMILY_EAM || !b->view.nbr)
        return fail(AKMC_ERR_UNSUPPORTED, "descriptors need an EAM batch with a neighbour list");
    if (b->field->pot.cutoff + b->view.skin < (double)kDescRc)
        return fail(AKMC_ERR_UNSUPPORTED, "the neighbour lists do not reach the descriptor cutoff");
    if (n_rows == 0) return AKMC_OK;
    if (!b->inv_perm.p) AKMC_CUDA(b->inv_perm.alloc((size_t)b->n_total));
    cudaStream_t s = (cudaStream_t)stream;
    invert_perm_kernel<<<(b->n_total + 255) / 256, 256, 0, s>>>(b->view.perm, b->inv_perm.p, b->n_total);
    const int blocks = (n_rows + kDescWarps - 1) / kDescWarps;
    descriptor_kernel<<<blocks, 32 * kDescWarps, 0, s>>>(b->view, rows_dev, n_rows, b->inv_perm.p, desc_dev,
                                                        basis_dev);
    AKMC_CUDA(cudaGetLastError());
    return AKMC_OK;
}

akmc_status akmc_mlp_forward(int n, const float* desc_dev, const float* norm_dev,
                             const float* params_dev, const float* basis_dev, float* out_dev,
                             void* stream)
{
    if (n < 0 || (n > 0 && (!desc_dev || !norm_dev || !params_dev || !out_dev)))
        return fail(AKMC_ERR_ARG, "bad mlp arguments");
    if (n == 0) return AKMC_OK;
    static bool configured = false;
    if (!configured) {
        AKMC_CUDA(configure_mlp_kernels());
        configured = true;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int tiles = (n + kTcRows - 1) / kTcRows;
    mlp_forward_tc_kernel<<<std::max(1, std::min((tiles + kTcGroups - 1) / kTcGroups, sms)), kTcThreads, kTcSmem,
                            (cudaStream_t)stream>>>(
        n, desc_dev, norm_dev, params_dev, basis_dev, out_dev);
    AKMC_CUDA(cudaGetLastError());
    return AKMC_OK;
}

akmc_status akmc_mlp_forward_fp32pipe(int n, const float* desc_dev, const float* norm_dev,
                                      const float* params_dev, const float* basis_dev, float* out_dev,
                                      void* stream)
{
    if (n < 0 || (n > 0 && (!desc_dev || !norm_dev || !params_dev || !out_dev)))
        return fail(AKMC_ERR_ARG, "bad mlp arguments");
    if (n == 0) return AKMC_OK;
    static bool configured = false;
    if (!configured) {
        AKMC_CUDA(configure_mlp_kernels());
        configured = true;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int tiles = (n + kFwdRows - 1) / kFwdRows;
    mlp_forward_kernel<<<std::min(tiles, sms), 256, kFwdSmem, (cudaStream_t)stream>>>(n, desc_dev, norm_dev,
                                                                                      params_dev, basis_dev, out_dev);
    AKMC_CUDA(cudaGetLastError());
    return AKMC_OK;
}

akmc_status akmc_mlp_check(void)
{
    int fault = 0;
    AKMC_CUDA(cudaMemcpyFromSymbol(&fault, g_mlp_fault, sizeof(int)));
    if (fault) return fail(AKMC_ERR_CUDA, "a tensor-core wait of the MLP kernel gave up");
    return AKMC_OK;
}

akmc_status akmc_mlp_train_step(int n, const float* desc_dev, const float* target_dev,
                                const float* norm_dev, const float* basis_dev, float* params_dev,
                                float* adam_m_dev, float* adam_v_dev, float* scratch_dev, int step,
                                float lr, float* loss_dev, float* grad_dev, void* stream)
{
    if (n < 1 || !desc_dev || !target_dev || !norm_dev || !params_dev || !scratch_dev || !loss_dev ||
        (lr != 0.0f && (!adam_m_dev || !adam_v_dev || step < 1)))
        return fail(AKMC_ERR_ARG, "bad training arguments");
    static bool configured = false;
    if (!configured) {
        AKMC_CUDA(configure_mlp_kernels());
        configured = true;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int tiles = (n + kTcRows - 1) / kTcRows;
    mlp_train_tc_kernel<<<tiles, kTtThreads, kTtSmem, s>>>(n, desc_dev, target_dev, norm_dev, params_dev, basis_dev,
                                                            scratch_dev, loss_dev, 2.0f / n);
    AKMC_CUDA(cudaGetLastError());
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, (float)std::max(step, 1)), c2 = 1.0f - powf(b2, (float)std::max(step, 1));
    adam_kernel<<<(kNParams + 255) / 256, 256, 0, s>>>(tiles, scratch_dev, params_dev, adam_m_dev, adam_v_dev, lr, b1,
                                                       b2, 1e-8f, c1, c2, grad_dev);
    AKMC_CUDA(cudaGetLastError());
    return AKMC_OK;
}

akmc_status akmc_mlp_train_step_fp32pipe(int n, const float* desc_dev, const float* target_dev,
                                         const float* norm_dev, const float* basis_dev, float* params_dev,
                                         float* adam_m_dev, float* adam_v_dev, float* scratch_dev, int step,
                                         float lr, float* loss_dev, float* grad_dev, void* stream)
{
    if (n < 1 || !desc_dev || !target_dev || !norm_dev || !params_dev || !scratch_dev || !loss_dev ||
        (lr != 0.0f && (!adam_m_dev || !adam_v_dev || step < 1)))
        return fail(AKMC_ERR_ARG, "bad training arguments");
    static bool configured = false;
    if (!configured) {
        AKMC_CUDA(configure_mlp_kernels());
        configured = true;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int tiles = (n + kTrRows - 1) / kTrRows;
    mlp_train_tile_kernel<<<tiles, 256, kTrSmem, s>>>(n, desc_dev, target_dev, norm_dev, params_dev, basis_dev,
                                                      scratch_dev, loss_dev, 2.0f / n);
    AKMC_CUDA(cudaGetLastError());
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, (float)std::max(step, 1)), c2 = 1.0f - powf(b2, (float)std::max(step, 1));
    adam_kernel<<<(kNParams + 255) / 256, 256, 0, s>>>(tiles, scratch_dev, params_dev, adam_m_dev, adam_v_dev, lr, b1,
                                                       b2, 1e-8f, c1, c2, grad_dev);
    AKMC_CUDA(cudaGetLastError());
    return AKMC_OK;
}

akmc_status akmc_proposal_seeds(int n_walkers, const long long* begin_dev, const double* pos_dev,
                                const double* box_dev, const double* center_dev, const float* pred_dev,
                                const float* score_dev, int score_stride, const akmc_proposal_params* params,
                                uint64_t seed, uint64_t counter, double* disp_dev, double* mode_dev,
                                int* chosen_dev, void* stream)
{
    if (n_walkers < 0 || !params || score_stride < 1)
        return fail(AKMC_ERR_ARG, "bad proposal arguments");
    if (n_walkers == 0) return AKMC_OK;
    if (!begin_dev || !pos_dev || !box_dev || !pred_dev || !score_dev || !disp_dev || !chosen_dev)
        return fail(AKMC_ERR_ARG, "null argument");
    if (!(params->threshold >= 0.0 && params->threshold <= 1.0) || !(params->radius >= 0.0) ||
        !(params->noise >= 0.0) || !(params->min_disp >= 0.0) || !(params->region >= 0.0))
        return fail(AKMC_ERR_ARG, "bad proposal parameters");
    proposal_seeds_kernel<<<n_walkers, kSeedThreads, 0, (cudaStream_t)stream>>>(
        begin_dev, pos_dev, box_dev, center_dev, pred_dev, score_dev, score_stride, *params, seed, counter, disp_dev,
        mode_dev, chosen_dev);
    AKMC_CUDA(cudaGetLastError());
    return AKMC_OK;
}

}  // extern "C"
