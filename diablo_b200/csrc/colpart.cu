// colpart.cu -- the column work of one RK_CHAN_1 substage, one pass over
// HBM: Fourier RHS assembly (channel.f:77-293), the Crank-Nicolson y solves
// of every field (channel.f:581-626, 737-1029), the REM_DIV_CHAN projection
// (channel.f:1103-1214) and the pressure update CP += phi/h
// (channel.f:1059-1065), for one pair of adjacent (kx,kz) columns per block.
//
// A block stages everything it reads -- CU, CF, the nonlinear term and CP
// of both columns, all rows -- into shared memory with asynchronous copies
// issued at once, assembles the right-hand sides row-parallel, solves the
// 2*nf CN systems one warp each, the two phi systems one warp each, and
// writes the new CU, CF and CP row-parallel: the state is read once and
// written once.
//
// Each tridiagonal system is solved with the partition method: its padded
// rows are cut into 32 consecutive blocks of R rows, one per lane.  A lane
// eliminates the interior rows of its block, which expresses every interior
// unknown as  x_i = y_i + p_i x_s + q_i x_e  in terms of the block's first
// and last unknowns; the first rows are eliminated into a 32-unknown
// tridiagonal system in the last unknowns t_k, solved by parallel cyclic
// reduction over the lanes (shuffles), and every row is reconstructed.
//
// The CN operator depends on y only (no LES), so its partition factors --
// interior multipliers and reciprocal pivots, p and q, the reduced system and
// its PCR multipliers -- are the same for every column and are built once per
// substage by k_cn_part; a column only carries its right-hand side through
// them.  The phi operator carries KX^2+KZ^2, so the phi system is factored
// per column on the fly.  Both systems are non-singular and diagonally
// dominant; the result equals the reference's sequential elimination
// (mpi.f:630-865) to round-off.
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.cuh"
#include "launch.h"

namespace dgpu {

namespace {

constexpr int NPART = 32;         // blocks (lanes) per tridiagonal system
constexpr int NPCR = 5;           // PCR steps: strides 1, 2, 4, 8, 16

__device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 operator*(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
__device__ __forceinline__ double2 ik(double K, double2 a) { return make_double2(-K * a.y, K * a.x); }
template <typename TN>
__device__ __forceinline__ double2 as_d2(const TN& v) { return make_double2((double)v.x, (double)v.y); }

__device__ __forceinline__ double2 shfl_up2(double2 v, int d) {
    return make_double2(__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d));
}
__device__ __forceinline__ double2 shfl_dn2(double2 v, int d) {
    return make_double2(__shfl_down_sync(0xffffffffu, v.x, d), __shfl_down_sync(0xffffffffu, v.y, d));
}
__host__ __device__ __forceinline__ double rcp_guard(double v) { return v != 0.0 ? 1.0 / v : 0.0; }

// 1/b by Newton-Raphson refinement (r <- r (2 - b r), quadratic convergence)
// of the single-precision reciprocal: 24 -> 48 -> 96 correct bits, i.e. within
// an ulp or so of the FP64 quotient; 0 for b = 0 (the guarded eliminations
// of mpi.f:700-865 skip a zero pivot).  Outside the float range the FP64
// division is used.
__device__ __forceinline__ double rcp_nr(double b) {
    const double ab = fabs(b);
    if (!(ab > 1e-30 && ab < 1e30)) return b != 0.0 ? 1.0 / b : 0.0;
    double r = (double)__frcp_rn((float)b);
    r = r * fma(-b, r, 2.0);
    r = r * fma(-b, r, 2.0);
    return r;
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

}  // namespace

// ---------------------------------------------------------------------------
// Partition tables of the CN systems, per field (PartTab offsets, doubles):
//   rows (NPR = 32*RC):  A, C (row coefficients), M (interior multipliers
//   a_i/beta_{i-1}), RB (interior 1/beta_i), P, Q (interior unknowns in
//   terms of the block's first / last unknown); row r of block k (system
//   row k*RC + r) is stored at r*32 + k, so a warp reads 32 consecutive
//   entries;
//   blocks (32 each):    rBs = 1/B_s, aS = a_s/B_s, cS = C_s/B_s,
//   W1 = A_e/B_s, W2 = c_e/B_s' (next block), RBT (1/pivot of the reduced
//   system after PCR), PA[5], PG[5] (PCR multipliers of strides 1..16).
// ---------------------------------------------------------------------------
struct PartTab {
    int npr;
    __host__ __device__ int A() const { return 0; }
    __host__ __device__ int C() const { return npr; }
    __host__ __device__ int M() const { return 2 * npr; }
    __host__ __device__ int RB() const { return 3 * npr; }
    __host__ __device__ int P() const { return 4 * npr; }
    __host__ __device__ int Q() const { return 5 * npr; }
    __host__ __device__ int blk(int which) const { return 6 * npr + NPART * which; }
    __host__ __device__ int size() const { return 6 * npr + NPART * 16; }
    __host__ __device__ static int at(int r, int k) { return r * NPART + k; }
};
enum { PB_RBS = 0, PB_AS, PB_CS, PB_W1, PB_W2, PB_RBT, PB_PA0, PB_PG0 = PB_PA0 + NPCR };

int part_rows(int nyp) {
    for (int r : {3, 5, 9, 17})
        if (NPART * r >= nyp) return r;
    return 0;
}

size_t part_table_doubles(int nyp) {
    PartTab t{NPART * part_rows(nyp)};
    return (size_t)t.size();
}

// Rows of every CN system (the order of the reference's set-up: interior
// rows, then the lower and upper BC routines APPLY_BC_TH_*, APPLY_BC_2_*,
// APPLY_BC_1_*, APPLY_BC_3_*, channel.f:1660-2282 via mpi.f:1083-1237), then
// the partition factors.  One block; dynamic shared memory holds the rows.
__global__ void __launch_bounds__(256) k_cn_part(CoefParams c, int RC, double* __restrict__ tabs,
                                                 double* __restrict__ bcv, signed char* __restrict__ kind) {
    extern __shared__ double sh[];
    const int ny = c.d.ny, nyp = c.d.nyp, nf = c.d.nf;
    const int npr = NPART * RC;
    const PartTab T{npr};
    double* sL = sh;
    double* sD = sL + nf * npr;
    double* sU = sD + nf * npr;
    double* sV = sU + nf * npr;
    double* sB = sV + nf * npr;                    // [nf][NPART][6]: a_s, B_s, C_s, A_e, B_e, c_e
    signed char* sK = reinterpret_cast<signed char*>(sB + nf * NPART * 6);
    const double* DY = c.dy;
    const double* DYF = c.dyf;
    for (int e = threadIdx.x; e < nf * npr; e += blockDim.x) {
        const int f = e / npr, j = e % npr;
        double l = 0.0, dd = 1.0, u = 0.0;
        signed char k = 1;
        if (j < nyp) {
            if (f >= 3) {
                const int n = f - 3;
                const double cc = c.temp1 / c.pr[n] * c.nu_v_scale;
                if (j >= c.jstart_th[n] && j <= ny) {
                    l = -cc / (DY[j] * DYF[j]);
                    dd = 1. + cc / (DY[j + 1] * DYF[j]) + cc / (DY[j] * DYF[j]);
                    u = -cc / (DY[j + 1] * DYF[j]);
                    k = 0;
                }
            } else if (f == 1) {
                const double t = c.temp1 * c.nu_v_scale;
                if (j >= 2 && j <= ny) {
                    l = -t / (DYF[j - 1] * DY[j]);
                    dd = 1. + t / (DYF[j] * DY[j]) + t / (DYF[j - 1] * DY[j]);
                    u = -t / (DYF[j] * DY[j]);
                    k = 0;
                }
            } else {
                const double t = c.temp1 * c.nu_v_scale;
                if (j >= 2 && j <= ny) {
                    l = -t / (DY[j] * DYF[j]);
                    dd = 1. - t * (-1. / (DY[j + 1] * DYF[j]) - 1. / (DY[j] * DYF[j]));
                    u = -t / (DY[j + 1] * DYF[j]);
                    k = 0;
                }
            }
        }
        sL[e] = l; sD[e] = dd; sU[e] = u; sV[e] = 0.0; sK[e] = k;
    }
    __syncthreads();
    if ((int)threadIdx.x < nf) {
        const int f = threadIdx.x;
        double* L = sL + f * npr;
        double* D = sD + f * npr;
        double* U = sU + f * npr;
        double* V = sV + f * npr;
        signed char* K = sK + f * npr;
        auto setrow = [&](int j, double l, double dd, double u, double v) {
            L[j] = l; D[j] = dd; U[j] = u; V[j] = v; K[j] = 1;
        };
        const int lo = c.bc_type[f][0], hi = c.bc_type[f][1];
        const double clo = c.bc_c1[f][0], chi = c.bc_c1[f][1];
        if (f >= 3) {
            if (lo == 0) { setrow(0, 0., 1., 0., 0.); setrow(1, 0., 1., 0., clo); }
            else { setrow(1, 0., -1., 1., DY[2] * clo); setrow(0, 0., 1., 0., 0.); }
            if (hi == 0) { setrow(ny + 1, 0., 1., 0., 0.); setrow(ny, 0., 1., 0., chi); }
            else { setrow(ny, -1., 1., 0., DY[ny] * chi); setrow(ny + 1, 0., 1., 0., 0.); }
        } else if (f == 1) {
            if (lo == 0) { setrow(1, 0., 1., 0., clo); setrow(2, 0., 1., 0., clo); }
            else { setrow(1, 0., -1., 1., DYF[1] * clo); }
            setrow(0, 0., 1., 0., 0.);
            if (hi == 0) { setrow(ny + 1, 0., 1., 0., chi); setrow(ny, 0., 1., 0., chi); }
            else { setrow(ny + 1, -1., 1., 0., DYF[ny] * chi); }
        } else {
            if (lo == 0) { setrow(0, 0., 1., 0., 0.); setrow(1, 0., 1., 0., clo); }
            else { setrow(0, 0., 1., 0., 0.); setrow(1, 0., -1., 1., DY[2] * clo); }
            if (hi == 0) { setrow(ny + 1, 0., 1., 0., 0.); setrow(ny, 0., 1., 0., chi); }
            else { setrow(ny, -1., 1., 0., DY[ny] * chi); setrow(ny + 1, 0., 1., 0., 0.); }
        }
        L[0] = 0.0;            // no row -1
        U[nyp - 1] = 0.0;      // no row NY+2
    }
    __syncthreads();
    // interior elimination of every block (one thread per field and block)
    for (int t = threadIdx.x; t < nf * NPART; t += blockDim.x) {
        const int f = t / NPART, k = t % NPART;
        const double* L = sL + f * npr;
        const double* D = sD + f * npr;
        const double* U = sU + f * npr;
        double* tb = tabs + (size_t)f * T.size();
        const int s = k * RC, e = s + RC - 1;
        double beta = D[s + 1], pp = -L[s + 1];
        tb[T.M() + PartTab::at(1, k)] = 0.0;
        tb[T.RB() + PartTab::at(1, k)] = rcp_guard(beta);
        tb[T.P() + PartTab::at(1, k)] = pp;                   // forward-eliminated p' for now
        for (int i = s + 2; i <= e - 1; ++i) {
            const double m = L[i] * rcp_guard(beta);
            beta = D[i] - m * U[i - 1];
            pp = -m * pp;
            tb[T.M() + PartTab::at(i - s, k)] = m;
            tb[T.RB() + PartTab::at(i - s, k)] = rcp_guard(beta);
            tb[T.P() + PartTab::at(i - s, k)] = pp;
        }
        double pn = 0.0, qn = 0.0;
        for (int i = e - 1; i >= s + 1; --i) {
            const double rb = tb[T.RB() + PartTab::at(i - s, k)];
            const double pi = (i == e - 1) ? tb[T.P() + PartTab::at(i - s, k)] * rb : (tb[T.P() + PartTab::at(i - s, k)] - U[i] * pn) * rb;
            const double qi = (i == e - 1) ? -U[i] * rb : -U[i] * qn * rb;
            tb[T.P() + PartTab::at(i - s, k)] = pi;
            tb[T.Q() + PartTab::at(i - s, k)] = qi;
            pn = pi;
            qn = qi;
        }
        for (int i = s; i <= e; ++i) {
            tb[T.A() + PartTab::at(i - s, k)] = L[i];
            tb[T.C() + PartTab::at(i - s, k)] = U[i];
        }
        tb[T.M() + PartTab::at(0, k)] = tb[T.RB() + PartTab::at(0, k)] = tb[T.P() + PartTab::at(0, k)] = tb[T.Q() + PartTab::at(0, k)] = 0.0;
        tb[T.M() + PartTab::at(RC - 1, k)] = tb[T.RB() + PartTab::at(RC - 1, k)] = tb[T.P() + PartTab::at(RC - 1, k)] = tb[T.Q() + PartTab::at(RC - 1, k)] = 0.0;
        double* b6 = sB + (f * NPART + k) * 6;
        b6[0] = L[s];
        b6[1] = D[s] + U[s] * tb[T.P() + PartTab::at(1, k)];
        b6[2] = U[s] * tb[T.Q() + PartTab::at(1, k)];
        b6[3] = L[e] * tb[T.P() + PartTab::at(RC - 2, k)];
        b6[4] = D[e] + L[e] * tb[T.Q() + PartTab::at(RC - 2, k)];
        b6[5] = U[e];
    }
    __syncthreads();
    // reduced system of the blocks' last unknowns and its PCR multipliers
    if ((int)threadIdx.x < nf) {
        const int f = threadIdx.x;
        double* tb = tabs + (size_t)f * T.size();
        const double* b6 = sB + f * NPART * 6;
        double al[NPART], be[NPART], ga[NPART], rbs[NPART];
        for (int k = 0; k < NPART; ++k) rbs[k] = rcp_guard(b6[k * 6 + 1]);
        for (int k = 0; k < NPART; ++k) {
            const double as = b6[k * 6 + 0], Cs = b6[k * 6 + 2], Ae = b6[k * 6 + 3], Be = b6[k * 6 + 4],
                         ce = b6[k * 6 + 5];
            const bool nx = k < NPART - 1;
            const double asn = nx ? b6[(k + 1) * 6 + 0] : 0.0, Csn = nx ? b6[(k + 1) * 6 + 2] : 0.0;
            const double rbn = nx ? rbs[k + 1] : 0.0;
            tb[T.blk(PB_RBS) + k] = rbs[k];
            tb[T.blk(PB_AS) + k] = as * rbs[k];
            tb[T.blk(PB_CS) + k] = Cs * rbs[k];
            tb[T.blk(PB_W1) + k] = Ae * rbs[k];
            tb[T.blk(PB_W2) + k] = ce * rbn;
            al[k] = -Ae * as * rbs[k];
            be[k] = Be - Ae * Cs * rbs[k] - ce * asn * rbn;
            ga[k] = -ce * Csn * rbn;
        }
        for (int st = 0; st < NPCR; ++st) {
            const int sg = 1 << st;
            double al2[NPART], be2[NPART], ga2[NPART];
            for (int k = 0; k < NPART; ++k) {
                const int lo = k - sg, hi = k + sg;
                const double a = lo >= 0 ? al[k] * rcp_guard(be[lo]) : 0.0;
                const double g = hi < NPART ? ga[k] * rcp_guard(be[hi]) : 0.0;
                al2[k] = lo >= 0 ? -a * al[lo] : 0.0;
                ga2[k] = hi < NPART ? -g * ga[hi] : 0.0;
                be2[k] = be[k] - (lo >= 0 ? a * ga[lo] : 0.0) - (hi < NPART ? g * al[hi] : 0.0);
                tb[T.blk(PB_PA0 + st) + k] = a;
                tb[T.blk(PB_PG0 + st) + k] = g;
            }
            for (int k = 0; k < NPART; ++k) { al[k] = al2[k]; be[k] = be2[k]; ga[k] = ga2[k]; }
        }
        for (int k = 0; k < NPART; ++k) tb[T.blk(PB_RBT) + k] = rcp_guard(be[k]);
    }
    for (int e = threadIdx.x; e < nf * nyp; e += blockDim.x) {
        const int f = e / nyp, j = e % nyp;
        bcv[e] = sV[f * npr + j];
        kind[e] = sK[f * npr + j];
    }
}

CoefParams make_coef(const Dims& d, const CnArgs& a, const int* bc_type, const double* bc_c1);

cudaError_t launch_cn_part(const Dims& d, const CnArgs& a, double* tabs, double* bcv, signed char* kind,
                           const int* bc_type, const double* bc_c1, cudaStream_t st) {
    const int RC = part_rows(d.nyp);
    if (RC == 0) return cudaErrorInvalidValue;
    const CoefParams c = make_coef(d, a, bc_type, bc_c1);
    const int npr = NPART * RC;
    const size_t smem =
        sizeof(double) * ((size_t)4 * d.nf * npr + (size_t)d.nf * NPART * 6) + (size_t)d.nf * npr;
    cudaFuncSetAttribute(k_cn_part, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_cn_part<<<1, 256, smem, st>>>(c, RC, tabs, bcv, kind);
    return cudaGetLastError();
}

CoefParams make_coef(const Dims& d, const CnArgs& a, const int* bc_type, const double* bc_c1) {
    CoefParams c;
    c.d = d;
    c.dy = a.dy;
    c.dyf = a.dyf;
    c.temp1 = a.temp1;
    c.nu_v_scale = a.nu_v_scale;
    for (int n = 0; n < 4; ++n) {
        c.pr[n] = a.pr[n];
        c.jstart_th[n] = a.cf_lo[3 + n < MAXF ? 3 + n : 0];
    }
    for (int f = 0; f < MAXF; ++f) {
        c.bc_type[f][0] = bc_type[2 * f];
        c.bc_type[f][1] = bc_type[2 * f + 1];
        c.bc_c1[f][0] = bc_c1[2 * f];
        c.bc_c1[f][1] = bc_c1[2 * f + 1];
    }
    return c;
}

// ---------------------------------------------------------------------------
// The column kernel: NW warps (2*nf <= NW), RC rows per lane and system.
// Shared memory, [slot][row][column] with NROW = 32*RC rows:
//   sU  nf slots   old CU (A1-A2), then RHS G -> solution x (B-D)
//   sP  1 slot     old CP                          (A1-D)
//   sPh 1 slot     phi                             (C-D)
//   sF  1 slot     phi factors of the pair         (A1-C)
//   sK  [nf][NROW] row kinds, sC per-field coefficients
// The nonlinear term and the old CF are read straight from global memory,
// each thread issuing the loads of all its rows before it uses any.
// ---------------------------------------------------------------------------
template <int NW, int RC, typename TN, bool PB>
__device__ __forceinline__ void colpart_body(const ColArgs& A, const TN* __restrict__ nl,
                                             const double* __restrict__ tabs, int tstride, unsigned bx) {
    constexpr int NROW = NPART * RC;
    constexpr int NT = 32 * NW;
    constexpr int NTHMAX = NW / 2 - 3 < 4 ? NW / 2 - 3 : 4;
    constexpr int NIT = (NW / 2) * NROW * 2 / NT;   // RHS items per thread at most (= RC)
    constexpr int NF2 = NROW * 2 > NPART * 16 ? NROW * 2 : NPART * 16;   // sF, double2
    const CnArgs& a = A.cn;
    const Dims& d = a.d;
    const int nf = d.nf, ny = d.ny, nyp = d.nyp;
    extern __shared__ __align__(16) unsigned char smem[];
    double2* sU = reinterpret_cast<double2*>(smem);
    double2* sW = sU;                               // RHS G -> solution x, over the old CU (B-D)
    double2* sP = sU + (size_t)nf * NROW * 2;
    double2* sPh = sP + NROW * 2;                   // phi (C-D)
    double2* sF = sPh + NROW * 2;                   // phi factors of the pair (A1-C)
    signed char* sK = reinterpret_cast<signed char*>(sF + NF2);
    double* sC = reinterpret_cast<double*>(sF + NF2) + (nf * NROW + 7) / 8;   // [MAXF][10]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const size_t ps = d.splane();
    const size_t fs = ps * nyp;
    const size_t g0 = (size_t)bx * 2;
    const bool proj = A.project != 0;
    const bool rk1 = a.rk_step > 1;
    auto slot = [](int f, int j, int c) { return ((size_t)f * NROW + j) * 2 + c; };
    const double2 zero = make_double2(0.0, 0.0);

    // ---- A1: stage CU, CF, CP of both columns (all rows), row tables -------
    {
        auto stream = [&](const double2* src, double2* dst) {      // 32 bytes per row
            for (int e = tid; e < nyp * 2; e += NT) {
                const int j = e >> 1, q = e & 1;
                cp_async16(dst + 2 * j + q, src + (size_t)j * ps + q);
            }
        };
        for (int f = 0; f < nf; ++f) {
            stream(a.cu + (size_t)f * fs + g0, sU + slot(f, 0, 0));
        }
        stream(a.cp + g0, sP);
        if (proj) {   // the pair's phi factors, 2 x 4 KB, contiguous per column pair
            const double2* src = reinterpret_cast<const double2*>(A.phitab + g0 * (NPART * 16));
            for (int e = tid; e < NPART * 16; e += NT) cp_async16(sF + e, src + e);
        }
        for (int e = tid; e < nf * NROW; e += NT) {
            const int f = e / NROW, j = e % NROW;
            sK[e] = j < nyp ? a.kind[f * nyp + j] : (signed char)1;
        }
        // per-field coefficients of the explicit terms (channel.f:77-293):
        // nu_f, U1 and U3 couplings, CN factor, horizontal gravity, is-U2,
        // KX / KZ selectors of the pressure gradient, first and last CF row
        if (tid < nf) {
            const int f = tid;
            double* q = sC + f * 10;
            double nuf = a.nu, cU1 = 0.0, cU3 = 0.0, cn_c = a.temp1 * a.nu_v_scale, cthv = 0.0, kxs = 0.0, kzs = 0.0;
            if (f == 0) { cU3 = a.i_ro; kxs = 1.0; cthv = a.grav_x; }
            else if (f == 2) { cU1 = -a.i_ro; kzs = 1.0; cthv = a.grav_z; }
            else if (f >= 3) {
                const int n = f - 3;
                nuf = a.nu / a.pr[n];
                cU1 = -a.drhodx[n];
                cU3 = -a.drhodz[n];
                cn_c = (a.temp1 / a.pr[n]) * a.nu_v_scale;
            }
            q[0] = nuf; q[1] = cU1; q[2] = cU3; q[3] = cn_c; q[4] = cthv; q[5] = f == 1 ? 1.0 : 0.0;
            q[6] = kxs; q[7] = kzs; q[8] = (double)a.cf_lo[f]; q[9] = (double)a.cf_hi[f];
        }
        cp_async_wait_all();
    }
    __syncthreads();

    // per-column constants of the pair
    const int kx0 = (int)(g0 % d.ldx), m0 = (int)(g0 / d.ldx);   // g0 even, ldx even: same kz row
    const double KX0 = a.kx[kx0], KX1 = a.kx[kx0 + 1], KZm = a.kz[m0];
    const double k20 = A.k2[g0], k21 = A.k2[g0 + 1];
    const bool zm0 = (kx0 == 0 && m0 == 0);
    // grid-metric row tables (small, shared by all blocks: read through L1)
    const double* RDY = A.rows + RT_RDY * nyp;
    const double* RDYF = A.rows + RT_RDYF * nyp;
    const double* E1P = A.rows + RT_E1P * nyp;
    const double* E1M = A.rows + RT_E1M * nyp;
    const double* E2P = A.rows + RT_E2P * nyp;
    const double* E2M = A.rows + RT_E2M * nyp;
    const double* BY0 = A.rows + RT_BY0 * nyp;
    const double* BY1 = A.rows + RT_BY1 * nyp;

    // ---- A2: right-hand sides, row-parallel; new CF out -------------------
    {
        const int nitem = nf * nyp * 2;
        // item e = tid + it*NT: column c = e&1, row j and field f of e>>1
        int jj[NIT], ff[NIT];
        {
            int r = tid >> 1, f = 0;
            while (r >= nyp) { r -= nyp; ++f; }
#pragma unroll
            for (int it = 0; it < NIT; ++it) {
                jj[it] = r;
                ff[it] = f;
                r += NT / 2;
                while (r >= nyp) { r -= nyp; ++f; }
            }
        }
        const int c = tid & 1;
        TN nlv[NIT];
        double2 cfv[NIT];
#pragma unroll
        for (int it = 0; it < NIT; ++it) {
            const bool v = tid + it * NT < nitem;
            const size_t o = (size_t)ff[it] * fs + spec_at(d, PB, jj[it], g0 + c);    // CF
            const size_t on = (size_t)ff[it] * fs + spec_at(d, false, jj[it], g0 + c); // NL: S layout
            if (v) nlv[it] = nl[on];
            cfv[it] = (v && rk1) ? a.cf[o] : zero;
        }
        const bool zero_mode = zm0 && c == 0;
        const double KX = c ? KX1 : KX0;
        const double k2 = c ? k21 : k20;
        const double fzm = zero_mode ? 1.0 : 0.0;
        const double t3 = rk1 ? a.temp3 : 0.0;
        double2 Gv[NIT];
        // all right-hand sides first, then the stores; straight-line items
        // (selects, predicated stores) so that they interleave
#pragma unroll
        for (int it = 0; it < NIT; ++it) {
            const bool valid = tid + it * NT < nitem;
            const int j = valid ? jj[it] : 0, f = valid ? ff[it] : 0;
            const double* cq = sC + f * 10;
            const double nuf = cq[0], cU1 = cq[1], cU3 = cq[2], cn_c = cq[3], cthv = cq[4], fu2 = cq[5];
            const double Kf = cq[6] * KX + cq[7] * KZm;
            const bool inr = j >= (int)cq[8] && j <= (int)cq[9];
            const bool isu2 = fu2 != 0.0;
            const int jm = j >= 1 ? j - 1 : 0, jp = j + 1 < nyp ? j + 1 : nyp - 1;
            const double wm = j >= 1 ? 1.0 : 0.0, wp = j + 1 < nyp ? 1.0 : 0.0;
            const double2 w1 = sU[slot(f, j, c)];
            const double2 w0 = wm * sU[slot(f, jm, c)];
            const double2 w2 = wp * sU[slot(f, jp, c)];          // row NY+2 is zero
            double2 cpl = cU1 * sU[slot(0, j, c)] + cU3 * sU[slot(2, j, c)];
#pragma unroll
            for (int n = 0; n < NTHMAX; ++n) {
                if (n < d.nth) {
                    const double2 thj = sU[slot(3 + n, j, c)];
                    const double2 thm = wm * sU[slot(3 + n, jm, c)];
                    cpl = cpl + (a.ri[n] * cthv) * thj +
                          (fu2 * (1.0 - fzm) * a.ri[n] * a.grav_y) * (BY0[j] * thj + BY1[j] * thm);
                }
            }
            double2 CF = (-nuf * k2) * w1 + cpl + as_d2(nlv[it]);
            if (A.mean_split && zero_mode && j >= A.jlo_prod && j <= ny) {
                // the mean x mean part of the y-flux product, -d/dy of (Q V) with
                // Q this field's plane mean and V = U2's (channel.f:514-516,
                // 535-537, 557-558): the only products that reach the (0,0) mode
                const double v0 = sU[slot(1, j, 0)].x, vp = sU[slot(1, jp, 0)].x, vm = sU[slot(1, jm, 0)].x;
                double mm;
                if (isu2) {
                    mm = 0.25 * ((v0 + vp) * (v0 + vp) - (v0 + vm) * (v0 + vm)) * RDY[j];
                } else {
                    const double q0 = sU[slot(f, j, 0)].x, qp = sU[slot(f, jp, 0)].x, qm = sU[slot(f, jm, 0)].x;
                    mm = ((qp + q0) * vp - (q0 + qm) * v0) * (0.5 * RDYF[j]);
                }
                CF.x -= mm;
            }
            const double2 cpj = sP[j * 2 + c];
            const double2 cpm = wm * sP[jm * 2 + c];
            const double2 cfo = cfv[it];
            double2 R = w1 + t3 * cfo - a.temp4 * ik(Kf, cpj) - (fu2 * a.temp4 * RDY[j]) * (cpj - cpm);
            R.x -= (f == 0 ? fzm : 0.0) * a.forcing;
            R = R + a.temp5 * CF;
            const double ep = isu2 ? E2P[j] : E1P[j], em = isu2 ? E2M[j] : E1M[j];
            const double2 Gi = R + cn_c * (ep * (w2 - w1) - em * (w1 - w0));
            const int knd = sK[f * NROW + j];
            double2 G = inr ? Gi : zero;
            if (knd != 0) G = zero_mode ? make_double2(a.bcv[f * nyp + j], 0.0) : zero;
            if (valid && inr && a.store_cf) a.cf[(size_t)f * fs + spec_at(d, PB, j, g0 + c)] = CF;
            Gv[it] = G;
        }
        __syncthreads();             // every old CU has been read
#pragma unroll
        for (int it = 0; it < NIT; ++it)
            if (tid + it * NT < nitem) sW[slot(ff[it], jj[it], c)] = Gv[it];
    }
    __syncthreads();

    // ---- B: CN solves, warp = (column, field) ------------------------------
    {
        const int c = warp & 1, f = warp >> 1, k = lane;
        if (f < nf) {
            const double* tb = tabs + (size_t)f * tstride;
            const PartTab T{NROW};
            double2 x[RC];
            const int i0 = k * RC;
#pragma unroll
            for (int r = 0; r < RC; ++r) {
                const int j = i0 + r;
                x[r] = j < nyp ? sW[slot(f, j, c)] : zero;
            }
            double tm[RC], trb[RC], tc[RC], tpp[RC], tq[RC], tpa[NPCR], tpg[NPCR];
#pragma unroll
            for (int r = 0; r < RC; ++r) {
                tm[r] = tb[T.M() + PartTab::at(r, k)];
                trb[r] = tb[T.RB() + PartTab::at(r, k)];
                tc[r] = tb[T.C() + PartTab::at(r, k)];
            }
            const double taE = tb[T.A() + PartTab::at(RC - 1, k)];
            const double tw1 = tb[T.blk(PB_W1) + k], tw2 = tb[T.blk(PB_W2) + k];
#pragma unroll
            for (int st = 0; st < NPCR; ++st) {
                tpa[st] = tb[T.blk(PB_PA0 + st) + k];
                tpg[st] = tb[T.blk(PB_PG0 + st) + k];
            }
            const double trbt = tb[T.blk(PB_RBT) + k], trbs = tb[T.blk(PB_RBS) + k];
            const double tas = tb[T.blk(PB_AS) + k], tcs = tb[T.blk(PB_CS) + k];
#pragma unroll
            for (int r = 0; r < RC; ++r) {
                tpp[r] = tb[T.P() + PartTab::at(r, k)];
                tq[r] = tb[T.Q() + PartTab::at(r, k)];
            }
#pragma unroll
            for (int r = 2; r <= RC - 2; ++r) x[r] = x[r] - tm[r] * x[r - 1];
            x[RC - 2] = trb[RC - 2] * x[RC - 2];
#pragma unroll
            for (int r = RC - 3; r >= 1; --r) x[r] = trb[r] * (x[r] - tc[r] * x[r + 1]);
            const double2 Ds = x[0] - tc[0] * x[1];
            const double2 De = x[RC - 1] - taE * x[RC - 2];
            const double2 Dsn = shfl_dn2(Ds, 1);
            double2 rk = De - tw1 * Ds - tw2 * Dsn;
#pragma unroll
            for (int st = 0; st < NPCR; ++st) {
                const int sg = 1 << st;
                const double2 rl = shfl_up2(rk, sg);
                const double2 rh = shfl_dn2(rk, sg);
                rk = rk - tpa[st] * rl - tpg[st] * rh;
            }
            const double2 t = trbt * rk;
            double2 tp = shfl_up2(t, 1);
            if (k == 0) tp = zero;
            const double2 u = trbs * Ds - tas * tp - tcs * t;
#pragma unroll
            for (int r = 1; r <= RC - 2; ++r) x[r] = x[r] + tpp[r] * u + tq[r] * t;
            x[0] = u;
            x[RC - 1] = t;
#pragma unroll
            for (int r = 0; r < RC; ++r) {
                const int j = i0 + r;
                if (j < nyp) sW[slot(f, j, c)] = x[r];
            }
        }
    }
    __syncthreads();

    // ---- C: phi of each column, warp c = column ----------------------------
    if (proj) {
        if (warp < 2) {
            const int c = warp, k = lane;
            const bool zero_mode = zm0 && c == 0;
            const double KX = c ? KX1 : KX0, KZ = KZm;
            const double K2 = KX * KX + KZ * KZ;
            // rows of APPLY_BC_REM_DIV_MPI (row 1, row NY) and REM_DIV_CHAN
            auto coef = [&](int j, double& A_, double& B_, double& C_) {
                A_ = 0.0; B_ = 1.0; C_ = 0.0;
                if (j == ny) { A_ = 1.0; B_ = -1.0; }
                else if (j == 1) { C_ = zero_mode ? 0.0 : -1.0; }
                else if (j >= 2 && j < ny) { A_ = E1M[j]; B_ = -K2 - E1P[j] - E1M[j]; C_ = E1P[j]; }
            };
            const int jb = k * RC;
            double2 y[RC];
#pragma unroll
            for (int r = 0; r < RC; ++r) {
                const int j = jb + r;
                double2 G = zero;
                if (j >= 2 && j < ny)
                    G = ik(KX, sW[slot(0, j, c)]) + RDYF[j] * (sW[slot(1, j + 1, c)] - sW[slot(1, j, c)]) +
                        ik(KZ, sW[slot(2, j, c)]);
                y[r] = G;
            }
            double rb[RC], pp[RC], qq[RC];
            {
                double A_, B_, C_, Cp;
                coef(jb + 1, A_, B_, C_);
                double beta = B_;
                rb[1] = rcp_nr(beta);
                pp[1] = -A_;
                Cp = C_;
#pragma unroll
                for (int r = 2; r <= RC - 2; ++r) {
                    coef(jb + r, A_, B_, C_);
                    const double mlt = A_ * rb[r - 1];
                    beta = B_ - mlt * Cp;
                    rb[r] = rcp_nr(beta);
                    y[r] = y[r] - mlt * y[r - 1];
                    pp[r] = -mlt * pp[r - 1];
                    Cp = C_;
                }
                y[RC - 2] = rb[RC - 2] * y[RC - 2];
                pp[RC - 2] = rb[RC - 2] * pp[RC - 2];
                qq[RC - 2] = -Cp * rb[RC - 2];
#pragma unroll
                for (int r = RC - 3; r >= 1; --r) {
                    coef(jb + r, A_, B_, C_);
                    y[r] = rb[r] * (y[r] - C_ * y[r + 1]);
                    pp[r] = rb[r] * (pp[r] - C_ * pp[r + 1]);
                    qq[r] = -C_ * qq[r + 1] * rb[r];
                }
            }
            // reduced system: the column's precomputed factors (k_phi_part)
            double2 Ds, De;
            {
                double A_, B_, C_;
                coef(jb, A_, B_, C_);
                Ds = y[0] - C_ * y[1];
                coef(jb + RC - 1, A_, B_, C_);
                De = y[RC - 1] - A_ * y[RC - 2];
            }
            const double* pt = reinterpret_cast<const double*>(sF) + (size_t)c * (NPART * 16);
            const double2 Dsn = shfl_dn2(Ds, 1);
            double2 rk = De - pt[PB_W1 * NPART + k] * Ds - pt[PB_W2 * NPART + k] * Dsn;
#pragma unroll
            for (int st = 0; st < NPCR; ++st) {
                const int sg = 1 << st;
                const double2 rl = shfl_up2(rk, sg);
                const double2 rh = shfl_dn2(rk, sg);
                rk = rk - pt[(PB_PA0 + st) * NPART + k] * rl - pt[(PB_PG0 + st) * NPART + k] * rh;
            }
            const double2 t = pt[PB_RBT * NPART + k] * rk;
            double2 tp = shfl_up2(t, 1);
            if (k == 0) tp = zero;
            const double2 u = pt[PB_RBS * NPART + k] * Ds - pt[PB_AS * NPART + k] * tp - pt[PB_CS * NPART + k] * t;
#pragma unroll
            for (int r = 0; r < RC; ++r) {
                const int j = jb + r;
                double2 phi = (r == 0) ? u : (r == RC - 1) ? t : y[r] + pp[r] * u + qq[r] * t;
                if (j < 1 || j > ny) phi = zero;
                sPh[j * 2 + c] = phi;
            }
        }
        __syncthreads();
    }

    // ---- D: new CU (projected), CP update, phi out; row-parallel ----------
    bool bad = false;                // a non-finite new CU value (DIABLO_ENAN)
    for (int e = tid; e < (nf + 1) * nyp * 2; e += NT) {
        const int c = e & 1, r = e >> 1;
        const int j = r % nyp, q = r / nyp;
        const size_t g = g0 + c;
        if (q < nf) {
            if (j < a.cb_lo[q]) continue;
            double2 v = sW[slot(q, j, c)];
            if (proj && q < 3 && j >= 1 && j <= ny) {
                const double2 phi = sPh[j * 2 + c];
                if (q == 0) v = v - ik(c ? KX1 : KX0, phi);
                else if (q == 2) v = v - ik(KZm, phi);
                else if (j >= 2) v = v - RDY[j] * (phi - sPh[(j - 1) * 2 + c]);
            }
            a.cu[(size_t)q * fs + (size_t)j * ps + g] = v;
            bad = bad || !(isfinite(v.x) && isfinite(v.y));
        } else if (proj && j >= 1 && j <= ny) {
            const double2 phi = sPh[j * 2 + c];
            if (A.update_cp && j >= 2) {
                double2* cpo = const_cast<double2*>(a.cp);
                cpo[(size_t)j * ps + g] = sP[j * 2 + c] + A.inv_h * phi;
            }
            if (A.store_phi) A.phi[(size_t)j * ps + g] = phi;
        }
    }
    if (bad && A.nan_flag) atomicOr(A.nan_flag, 1);
}

// Blocks per SM: three at up to 5 rows per lane (80 registers; the few rows
// of a small NY leave the phases short, so more pairs in flight pay), two
// at 9 and 17 rows, whose solve holds more values.
template <int NW, int RC, typename TN, bool PB>
__global__ void __launch_bounds__(32 * NW, NW == 8 ? (RC <= 5 ? 3 : 2) : 1)
k_colpart(ColArgs A, const TN* __restrict__ nl, const double* __restrict__ tabs, int tstride) {
    colpart_body<NW, RC, TN, PB>(A, nl, tabs, tstride, blockIdx.x);
}

// Batched form: instance blockIdx.y of a group of equal shape.
template <int NW, int RC, typename TN, bool PB>
__global__ void __launch_bounds__(32 * NW, NW == 8 ? (RC <= 5 ? 3 : 2) : 1)
k_colpart_b(const ColJob* __restrict__ jobs, int tstride) {
    const ColJob& j = jobs[blockIdx.y];
    const ColArgs& A = j.A;     // read in place: a copy would sit in every thread's stack
    colpart_body<NW, RC, TN, PB>(A, reinterpret_cast<const TN*>(j.nl), j.tabs, tstride, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Partition factors of every column's phi system (the REM_DIV_CHAN rows,
// which depend on the grid and on KX^2+KZ^2 only): the reduced system of
// the blocks' last unknowns and its PCR multipliers, in the PB_* layout of
// the CN tables ([which][block]).  Built once per instance; one warp per
// column.
// ---------------------------------------------------------------------------
template <int RC>
__global__ void __launch_bounds__(128) k_phi_part(Dims d, const double* __restrict__ rows,
                                                  const double* __restrict__ kxw, const double* __restrict__ kzw,
                                                  double* __restrict__ tab) {
    const int k = threadIdx.x & 31;
    const size_t g = (size_t)blockIdx.x * 4 + (threadIdx.x >> 5);
    if (g >= d.splane()) return;
    const int ny = d.ny, nyp = d.nyp;
    const int kx = (int)(g % d.ldx), m = (int)(g / d.ldx);
    const bool zero_mode = (kx == 0 && m == 0);
    const double K2 = kxw[kx] * kxw[kx] + kzw[m] * kzw[m];
    const double* E1P = rows + RT_E1P * nyp;
    const double* E1M = rows + RT_E1M * nyp;
    auto coef = [&](int j, double& A_, double& B_, double& C_) {
        A_ = 0.0; B_ = 1.0; C_ = 0.0;
        if (j == ny) { A_ = 1.0; B_ = -1.0; }
        else if (j == 1) { C_ = zero_mode ? 0.0 : -1.0; }
        else if (j >= 2 && j < ny) { A_ = E1M[j]; B_ = -K2 - E1P[j] - E1M[j]; C_ = E1P[j]; }
    };
    const int jb = k * RC;
    double rb[RC], pp[RC], qq[RC];
    {
        double A_, B_, C_, Cp;
        coef(jb + 1, A_, B_, C_);
        double beta = B_;
        rb[1] = rcp_guard(beta);
        pp[1] = -A_;
        Cp = C_;
        for (int r = 2; r <= RC - 2; ++r) {
            coef(jb + r, A_, B_, C_);
            const double mlt = A_ * rb[r - 1];
            beta = B_ - mlt * Cp;
            rb[r] = rcp_guard(beta);
            pp[r] = -mlt * pp[r - 1];
            Cp = C_;
        }
        pp[RC - 2] = rb[RC - 2] * pp[RC - 2];
        qq[RC - 2] = -Cp * rb[RC - 2];
        for (int r = RC - 3; r >= 1; --r) {
            coef(jb + r, A_, B_, C_);
            pp[r] = rb[r] * (pp[r] - C_ * pp[r + 1]);
            qq[r] = -C_ * qq[r + 1] * rb[r];
        }
    }
    double as, Bs, Cs, Ae, Be, ce;
    {
        double A_, B_, C_;
        coef(jb, A_, B_, C_);
        as = A_; Bs = B_ + C_ * pp[1]; Cs = C_ * qq[1];
        coef(jb + RC - 1, A_, B_, C_);
        Ae = A_ * pp[RC - 2]; Be = B_ + A_ * qq[RC - 2]; ce = C_;
    }
    const double rBs = rcp_guard(Bs);
    const double asn = __shfl_down_sync(0xffffffffu, as, 1);
    const double Csn = __shfl_down_sync(0xffffffffu, Cs, 1);
    const double rBn = __shfl_down_sync(0xffffffffu, rBs, 1);
    const bool nxt = k < NPART - 1;
    double* pt = tab + g * (NPART * 16);
    pt[PB_RBS * NPART + k] = rBs;
    pt[PB_AS * NPART + k] = as * rBs;
    pt[PB_CS * NPART + k] = Cs * rBs;
    pt[PB_W1 * NPART + k] = Ae * rBs;
    pt[PB_W2 * NPART + k] = nxt ? ce * rBn : 0.0;
    double al = -Ae * as * rBs;
    double be = Be - Ae * Cs * rBs - (nxt ? ce * asn * rBn : 0.0);
    double ga = nxt ? -ce * Csn * rBn : 0.0;
    for (int st = 0; st < NPCR; ++st) {
        const int sg = 1 << st;
        const double all = __shfl_up_sync(0xffffffffu, al, sg), bel = __shfl_up_sync(0xffffffffu, be, sg),
                     gal = __shfl_up_sync(0xffffffffu, ga, sg);
        const double alh = __shfl_down_sync(0xffffffffu, al, sg), beh = __shfl_down_sync(0xffffffffu, be, sg),
                     gah = __shfl_down_sync(0xffffffffu, ga, sg);
        const bool hl = k >= sg, hh = k + sg < NPART;
        const double fa = hl ? al * rcp_guard(bel) : 0.0;
        const double fg = hh ? ga * rcp_guard(beh) : 0.0;
        const double al2 = hl ? -fa * all : 0.0;
        const double ga2 = hh ? -fg * gah : 0.0;
        be = be - (hl ? fa * gal : 0.0) - (hh ? fg * alh : 0.0);
        al = al2;
        ga = ga2;
        pt[(PB_PA0 + st) * NPART + k] = fa;
        pt[(PB_PG0 + st) * NPART + k] = fg;
    }
    pt[PB_RBT * NPART + k] = rcp_guard(be);
}

// ---------------------------------------------------------------------------
// REM_DIV_CHAN on its own (channel.f:1103-1214, with the rows of
// APPLY_BC_REM_DIV_MPI, mpi.f:1239-1278) and the pressure update
// CP += phi/h (channel.f:1059-1065): the projection step of k_colpart
// without the CN solves.  Four adjacent columns per block; CU1..CU3 of the
// four are staged row by row (64-byte runs), warp c solves column c's phi
// system by the partition method with the column's factors from
// k_phi_part, and the corrections are written back row-parallel.
// Shared memory: [3][NROW][4] velocity (staged with cp.async, all rows in
// flight at once), [NROW][4] phi.
// ---------------------------------------------------------------------------
template <int RC>
__global__ void __launch_bounds__(128) k_proj(RemDivArgs a) {
    constexpr int NROW = NPART * RC;
    extern __shared__ __align__(16) unsigned char smem[];
    double2* sV = reinterpret_cast<double2*>(smem);   // [3][NROW][4]
    double2* sPh = sV + 3 * NROW * 4;                 // [NROW][4]
    const Dims& d = a.d;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ny = d.ny, nyp = d.nyp;
    const size_t ps = d.splane(), fs = ps * d.nyp;
    const size_t g0 = (size_t)blockIdx.x * 4;
    const double2 zero = make_double2(0.0, 0.0);
    const double* RDY = a.rows + RT_RDY * nyp;
    const double* RDYF = a.rows + RT_RDYF * nyp;
    const double* E1P = a.rows + RT_E1P * nyp;
    const double* E1M = a.rows + RT_E1M * nyp;
    auto live = [&](int c) {
        const size_t g = g0 + c;
        return (int)(g % d.ldx) < d.nkxp && (int)(g / d.ldx) < d.nkzt;
    };
    for (int e = tid; e < 3 * nyp * 4; e += 128) {
        const int c = e & 3, r = e >> 2;
        const int j = r % nyp, f = r / nyp;
        cp_async16(sV + ((size_t)f * NROW + j) * 4 + c, a.cu + (size_t)f * fs + (size_t)j * ps + g0 + c);
    }
    cp_async_wait_all();
    __syncthreads();
    {
        const int c = warp, k = lane;
        const size_t g = g0 + c;
        const int kx = (int)(g % d.ldx), m = (int)(g / d.ldx);
        if (live(c)) {
            const bool zero_mode = (kx == 0 && m == 0);
            const double KX = a.kx[kx], KZ = a.kz[m];
            const double K2 = KX * KX + KZ * KZ;
            auto coef = [&](int j, double& A_, double& B_, double& C_) {
                A_ = 0.0; B_ = 1.0; C_ = 0.0;
                if (j == ny) { A_ = 1.0; B_ = -1.0; }
                else if (j == 1) { C_ = zero_mode ? 0.0 : -1.0; }
                else if (j >= 2 && j < ny) { A_ = E1M[j]; B_ = -K2 - E1P[j] - E1M[j]; C_ = E1P[j]; }
            };
            auto V = [&](int f, int j) { return sV[((size_t)f * NROW + j) * 4 + c]; };
            const int jb = k * RC;
            double2 y[RC];
#pragma unroll
            for (int r = 0; r < RC; ++r) {
                const int j = jb + r;
                double2 G = zero;
                if (j >= 2 && j < ny) G = ik(KX, V(0, j)) + RDYF[j] * (V(1, j + 1) - V(1, j)) + ik(KZ, V(2, j));
                y[r] = G;
            }
            double rb[RC], pp[RC], qq[RC];
            {
                double A_, B_, C_, Cp;
                coef(jb + 1, A_, B_, C_);
                double beta = B_;
                rb[1] = rcp_nr(beta);
                pp[1] = -A_;
                Cp = C_;
#pragma unroll
                for (int r = 2; r <= RC - 2; ++r) {
                    coef(jb + r, A_, B_, C_);
                    const double mlt = A_ * rb[r - 1];
                    beta = B_ - mlt * Cp;
                    rb[r] = rcp_nr(beta);
                    y[r] = y[r] - mlt * y[r - 1];
                    pp[r] = -mlt * pp[r - 1];
                    Cp = C_;
                }
                y[RC - 2] = rb[RC - 2] * y[RC - 2];
                pp[RC - 2] = rb[RC - 2] * pp[RC - 2];
                qq[RC - 2] = -Cp * rb[RC - 2];
#pragma unroll
                for (int r = RC - 3; r >= 1; --r) {
                    coef(jb + r, A_, B_, C_);
                    y[r] = rb[r] * (y[r] - C_ * y[r + 1]);
                    pp[r] = rb[r] * (pp[r] - C_ * pp[r + 1]);
                    qq[r] = -C_ * qq[r + 1] * rb[r];
                }
            }
            double2 Ds, De;
            {
                double A_, B_, C_;
                coef(jb, A_, B_, C_);
                Ds = y[0] - C_ * y[1];
                coef(jb + RC - 1, A_, B_, C_);
                De = y[RC - 1] - A_ * y[RC - 2];
            }
            const double* pt = a.phitab + g * (NPART * 16);
            const double2 Dsn = shfl_dn2(Ds, 1);
            double2 rk = De - pt[PB_W1 * NPART + k] * Ds - pt[PB_W2 * NPART + k] * Dsn;
#pragma unroll
            for (int st = 0; st < NPCR; ++st) {
                const int sg = 1 << st;
                const double2 rl = shfl_up2(rk, sg);
                const double2 rh = shfl_dn2(rk, sg);
                rk = rk - pt[(PB_PA0 + st) * NPART + k] * rl - pt[(PB_PG0 + st) * NPART + k] * rh;
            }
            const double2 t = pt[PB_RBT * NPART + k] * rk;
            double2 tp = shfl_up2(t, 1);
            if (k == 0) tp = zero;
            const double2 u = pt[PB_RBS * NPART + k] * Ds - pt[PB_AS * NPART + k] * tp - pt[PB_CS * NPART + k] * t;
#pragma unroll
            for (int r = 0; r < RC; ++r) {
                const int j = jb + r;
                double2 phi = (r == 0) ? u : (r == RC - 1) ? t : y[r] + pp[r] * u + qq[r] * t;
                if (j < 1 || j > ny) phi = zero;
                sPh[j * 4 + c] = phi;
            }
        }
    }
    __syncthreads();
    // corrected velocity (rows 1..NY; CU2 rows 2..NY), CP += phi/h (rows
    // 2..NY) and phi (rows 1..NY), row-parallel
    bool bad = false;                // a non-finite new velocity value (DIABLO_ENAN)
    auto put = [&](double2* dst, const double2 v) {
        *dst = v;
        bad = bad || !(isfinite(v.x) && isfinite(v.y));
    };
    for (int e = tid; e < 5 * ny * 4; e += 128) {
        const int c = e & 3, r = e >> 2;
        const int j = 1 + r % ny, q = r / ny;
        if (!live(c)) continue;
        const size_t g = g0 + c;
        const size_t o = (size_t)j * ps + g;
        const double2 phi = sPh[j * 4 + c];
        if (q == 0) {
            put(a.cu + o, sV[((size_t)0 * NROW + j) * 4 + c] - ik(a.kx[g % d.ldx], phi));
        } else if (q == 2) {
            put(a.cu + 2 * fs + o, sV[((size_t)2 * NROW + j) * 4 + c] - ik(a.kz[g / d.ldx], phi));
        } else if (q == 1) {
            if (j >= 2) put(a.cu + fs + o, sV[((size_t)1 * NROW + j) * 4 + c] - RDY[j] * (phi - sPh[(j - 1) * 4 + c]));
        } else if (q == 3) {
            if (a.update_cp && j >= 2) a.cp[o] = a.cp[o] + a.inv_h * phi;
        } else {
            a.phi[o] = phi;
        }
    }
    if (bad && a.nan_flag) atomicOr(a.nan_flag, 1);
}

size_t phi_table_doubles(const Dims& d) { return d.splane() * (size_t)(NPART * 16); }

cudaError_t launch_remdiv(const RemDivArgs& a, cudaStream_t st) {
    const Dims& d = a.d;
    const int RC = part_rows(d.nyp);
    const size_t smem = sizeof(double2) * 4 * (size_t)NPART * RC * 4;
    const unsigned nblk = (unsigned)(d.splane() / 4);
    auto go = [&](auto kern) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<nblk, 128, smem, st>>>(a);
    };
    switch (RC) {
        case 3: go(k_proj<3>); break;
        case 5: go(k_proj<5>); break;
        case 9: go(k_proj<9>); break;
        case 17: go(k_proj<17>); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_phi_part(const Dims& d, const double* rows, const double* kx, const double* kz, double* tab,
                            cudaStream_t st) {
    const unsigned nblk = (unsigned)((d.splane() + 3) / 4);
    switch (part_rows(d.nyp)) {
        case 3: k_phi_part<3><<<nblk, 128, 0, st>>>(d, rows, kx, kz, tab); break;
        case 5: k_phi_part<5><<<nblk, 128, 0, st>>>(d, rows, kx, kz, tab); break;
        case 9: k_phi_part<9><<<nblk, 128, 0, st>>>(d, rows, kx, kz, tab); break;
        case 17: k_phi_part<17><<<nblk, 128, 0, st>>>(d, rows, kx, kz, tab); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <typename TN>
size_t colpart_smem(const Dims& d) {
    const int RC = part_rows(d.nyp);
    const size_t NROW = (size_t)NPART * RC;
    const size_t NF2 = NROW * 2 > NPART * 16 ? NROW * 2 : NPART * 16;
    return (NROW * 2 * ((size_t)d.nf + 2) + NF2) * sizeof(double2) + (NROW * (size_t)d.nf + 7) / 8 * 8 +
           MAXF * 10 * sizeof(double);
}

template <typename TN>
cudaError_t launch_colpart(const ColArgs& a, const TN* nl, const double* tabs, cudaStream_t st) {
    const Dims& d = a.cn.d;
    const int RC = part_rows(d.nyp);
    const size_t smem = colpart_smem<TN>(d);
    const int tstride = (int)part_table_doubles(d.nyp);
    const unsigned nblk = (unsigned)(d.splane() / 2);
    auto go = [&](auto kern, int nw) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<nblk, 32 * nw, smem, st>>>(a, nl, tabs, tstride);
    };
#define DGPU_RC_PB(NW, R)                                                       \
    if (a.pair_blocked) go(k_colpart<NW, R, TN, true>, NW);                     \
    else go(k_colpart<NW, R, TN, false>, NW);
#define DGPU_RC_CASES(NW)                                        \
    switch (RC) {                                                \
        case 3: DGPU_RC_PB(NW, 3) break;                         \
        case 5: DGPU_RC_PB(NW, 5) break;                         \
        case 9: DGPU_RC_PB(NW, 9) break;                         \
        case 17: DGPU_RC_PB(NW, 17) break;                       \
        default: return cudaErrorInvalidValue;                   \
    }
    if (d.nf <= 4) { DGPU_RC_CASES(8) }
    else if (d.nf <= 8) { DGPU_RC_CASES(16) }
    else return cudaErrorInvalidValue;
#undef DGPU_RC_CASES
#undef DGPU_RC_PB
    return cudaGetLastError();
}

template <typename TN>
cudaError_t launch_colpart_b(const Dims& d, const ColJob* jobs, int ninst, bool pair_blocked, cudaStream_t st) {
    const int RC = part_rows(d.nyp);
    const size_t smem = colpart_smem<TN>(d);
    const int tstride = (int)part_table_doubles(d.nyp);
    dim3 grid((unsigned)(d.splane() / 2), (unsigned)ninst);
    auto go = [&](auto kern, int nw) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<grid, 32 * nw, smem, st>>>(jobs, tstride);
    };
#define DGPU_RC_PB(NW, R)                                                       \
    if (pair_blocked) go(k_colpart_b<NW, R, TN, true>, NW);                     \
    else go(k_colpart_b<NW, R, TN, false>, NW);
#define DGPU_RC_CASES(NW)                                        \
    switch (RC) {                                                \
        case 3: DGPU_RC_PB(NW, 3) break;                         \
        case 5: DGPU_RC_PB(NW, 5) break;                         \
        case 9: DGPU_RC_PB(NW, 9) break;                         \
        case 17: DGPU_RC_PB(NW, 17) break;                       \
        default: return cudaErrorInvalidValue;                   \
    }
    if (d.nf <= 4) { DGPU_RC_CASES(8) }
    else if (d.nf <= 8) { DGPU_RC_CASES(16) }
    else return cudaErrorInvalidValue;
#undef DGPU_RC_CASES
#undef DGPU_RC_PB
    return cudaGetLastError();
}

template cudaError_t launch_colpart_b<cpx<float>>(const Dims&, const ColJob*, int, bool, cudaStream_t);
template cudaError_t launch_colpart_b<cpx<double>>(const Dims&, const ColJob*, int, bool, cudaStream_t);
template cudaError_t launch_colpart<cpx<float>>(const ColArgs&, const cpx<float>*, const double*, cudaStream_t);
template cudaError_t launch_colpart<cpx<double>>(const ColArgs&, const cpx<double>*, const double*, cudaStream_t);
template size_t colpart_smem<cpx<float>>(const Dims&);
template size_t colpart_smem<cpx<double>>(const Dims&);

}  // namespace dgpu
