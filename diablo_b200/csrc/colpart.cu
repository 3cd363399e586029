// colpart.cu -- the column work of one RK_CHAN_1 substage, one pass over
// HBM: Fourier RHS assembly (channel.f:77-293), the Crank-Nicolson y solves
// of every field (channel.f:581-626, 737-1029), the REM_DIV_CHAN projection
// (channel.f:1103-1214) and the pressure update CP += phi/h
// (channel.f:1059-1065), for one pair of adjacent (kx,kz) columns per block.
//
// Each tridiagonal system is solved with the partition method: its padded
// rows are cut into P consecutive blocks of R rows, one per lane.  A lane
// eliminates the interior rows of its block, which expresses every interior
// unknown as  x_i = y_i + p_i x_s + q_i x_e  in terms of the block's first
// and last unknowns; the first rows are then eliminated into a P-unknown
// tridiagonal system in the last unknowns t_k, solved by parallel cyclic
// reduction over the lanes (shuffles), and every row is reconstructed.  All
// of a column stays in registers and shared memory, so the state is read
// once and written once.
//
// The CN operator depends on y only (no LES), so its partition factors --
// interior multipliers and reciprocal pivots, p and q, the reduced system and
// its PCR multipliers -- are the same for every column and are built once per
// substage by k_cn_part; a column only carries its right-hand side through
// them.  The phi operator carries KX^2+KZ^2, so the phi system is factored
// per column on the fly.  Both systems are non-singular and diagonally
// dominant; the result equals the reference's sequential elimination
// (mpi.f:630-865) to round-off.
//
// Lanes.  CN phase: warp f = field f; lane = c*16 + k, column c of the pair,
// block k of 16 (R = RC rows each).  Phi phase: warp c = column c; lane k of
// 32 blocks (R = RP rows each).
#include <cuda_runtime.h>

#include "kernels.cuh"
#include "launch.h"

namespace dgpu {

namespace {

__device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 operator*(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
__device__ __forceinline__ double2 ik(double K, double2 a) { return make_double2(-K * a.y, K * a.x); }
template <typename TN>
__device__ __forceinline__ double2 as_d2(const TN& v) { return make_double2((double)v.x, (double)v.y); }

__device__ __forceinline__ double2 shfl_up2(double2 v, int d, int w) {
    return make_double2(__shfl_up_sync(0xffffffffu, v.x, d, w), __shfl_up_sync(0xffffffffu, v.y, d, w));
}
__device__ __forceinline__ double2 shfl_dn2(double2 v, int d, int w) {
    return make_double2(__shfl_down_sync(0xffffffffu, v.x, d, w), __shfl_down_sync(0xffffffffu, v.y, d, w));
}
__host__ __device__ __forceinline__ double rcp_guard(double v) { return v != 0.0 ? 1.0 / v : 0.0; }

}  // namespace

// ---------------------------------------------------------------------------
// Partition tables of the CN systems, per field (PartTab offsets, doubles):
//   rows (NPR = 16*RC):  A, C (row coefficients), M (interior multipliers
//   a_i/beta_{i-1}), RB (interior 1/beta_i), P, Q (interior unknowns in
//   terms of the block's first / last unknown);
//   blocks (16 each):    rBs = 1/B_s, aS = a_s/B_s, cS = C_s/B_s,
//   W1 = A_e/B_s, W2 = c_e/B_s' (next block), RBT (1/pivot of the reduced
//   system after PCR), PA[4], PG[4] (PCR multipliers of the steps 1,2,4,8).
// ---------------------------------------------------------------------------
struct PartTab {
    int npr;
    __host__ __device__ int A() const { return 0; }
    __host__ __device__ int C() const { return npr; }
    __host__ __device__ int M() const { return 2 * npr; }
    __host__ __device__ int RB() const { return 3 * npr; }
    __host__ __device__ int P() const { return 4 * npr; }
    __host__ __device__ int Q() const { return 5 * npr; }
    __host__ __device__ int blk(int which) const { return 6 * npr + 16 * which; }
    __host__ __device__ int size() const { return 6 * npr + 16 * 14; }
};
enum { PB_RBS = 0, PB_AS, PB_CS, PB_W1, PB_W2, PB_RBT, PB_PA0, PB_PG0 = PB_PA0 + 4 };

int part_rows(int nyp) {
    for (int r : {5, 9, 17, 33})
        if (16 * r >= nyp) return r;
    return 0;
}

size_t part_table_doubles(int nyp) {
    PartTab t{16 * part_rows(nyp)};
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
    const int npr = 16 * RC;
    const PartTab T{npr};
    double* sL = sh;
    double* sD = sL + nf * npr;
    double* sU = sD + nf * npr;
    double* sV = sU + nf * npr;
    double* sB = sV + nf * npr;                    // [nf][16][6]: a_s, B_s, C_s, A_e, B_e, c_e
    signed char* sK = reinterpret_cast<signed char*>(sB + nf * 16 * 6);
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
    for (int t = threadIdx.x; t < nf * 16; t += blockDim.x) {
        const int f = t / 16, k = t % 16;
        const double* L = sL + f * npr;
        const double* D = sD + f * npr;
        const double* U = sU + f * npr;
        double* tb = tabs + (size_t)f * T.size();
        const int s = k * RC, e = s + RC - 1;
        double beta = D[s + 1], pp = -L[s + 1];
        tb[T.M() + s + 1] = 0.0;
        tb[T.RB() + s + 1] = rcp_guard(beta);
        tb[T.P() + s + 1] = pp;                   // forward-eliminated p' for now
        for (int i = s + 2; i <= e - 1; ++i) {
            const double m = L[i] * rcp_guard(beta);
            beta = D[i] - m * U[i - 1];
            pp = -m * pp;
            tb[T.M() + i] = m;
            tb[T.RB() + i] = rcp_guard(beta);
            tb[T.P() + i] = pp;
        }
        double pn = 0.0, qn = 0.0;
        for (int i = e - 1; i >= s + 1; --i) {
            const double rb = tb[T.RB() + i];
            const double pi = (i == e - 1) ? tb[T.P() + i] * rb : (tb[T.P() + i] - U[i] * pn) * rb;
            const double qi = (i == e - 1) ? -U[i] * rb : -U[i] * qn * rb;
            tb[T.P() + i] = pi;
            tb[T.Q() + i] = qi;
            pn = pi;
            qn = qi;
        }
        for (int i = s; i <= e; ++i) {
            tb[T.A() + i] = L[i];
            tb[T.C() + i] = U[i];
        }
        tb[T.M() + s] = tb[T.RB() + s] = tb[T.P() + s] = tb[T.Q() + s] = 0.0;
        tb[T.M() + e] = tb[T.RB() + e] = tb[T.P() + e] = tb[T.Q() + e] = 0.0;
        double* b6 = sB + (f * 16 + k) * 6;
        b6[0] = L[s];
        b6[1] = D[s] + U[s] * tb[T.P() + s + 1];
        b6[2] = U[s] * tb[T.Q() + s + 1];
        b6[3] = L[e] * tb[T.P() + e - 1];
        b6[4] = D[e] + L[e] * tb[T.Q() + e - 1];
        b6[5] = U[e];
    }
    __syncthreads();
    // reduced system of the blocks' last unknowns and its PCR multipliers
    if ((int)threadIdx.x < nf) {
        const int f = threadIdx.x;
        double* tb = tabs + (size_t)f * T.size();
        const double* b6 = sB + f * 16 * 6;
        double al[16], be[16], ga[16], rbs[16];
        for (int k = 0; k < 16; ++k) rbs[k] = rcp_guard(b6[k * 6 + 1]);
        for (int k = 0; k < 16; ++k) {
            const double as = b6[k * 6 + 0], Cs = b6[k * 6 + 2], Ae = b6[k * 6 + 3], Be = b6[k * 6 + 4],
                         ce = b6[k * 6 + 5];
            const bool nx = k < 15;
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
        for (int st = 0; st < 4; ++st) {
            const int sg = 1 << st;
            double al2[16], be2[16], ga2[16];
            for (int k = 0; k < 16; ++k) {
                const int lo = k - sg, hi = k + sg;
                const double a = lo >= 0 ? al[k] * rcp_guard(be[lo]) : 0.0;
                const double g = hi < 16 ? ga[k] * rcp_guard(be[hi]) : 0.0;
                al2[k] = lo >= 0 ? -a * al[lo] : 0.0;
                ga2[k] = hi < 16 ? -g * ga[hi] : 0.0;
                be2[k] = be[k] - (lo >= 0 ? a * ga[lo] : 0.0) - (hi < 16 ? g * al[hi] : 0.0);
                tb[T.blk(PB_PA0 + st) + k] = a;
                tb[T.blk(PB_PG0 + st) + k] = g;
            }
            for (int k = 0; k < 16; ++k) { al[k] = al2[k]; be[k] = be2[k]; ga[k] = ga2[k]; }
        }
        for (int k = 0; k < 16; ++k) tb[T.blk(PB_RBT) + k] = rcp_guard(be[k]);
    }
    for (int e = threadIdx.x; e < nf * nyp; e += blockDim.x) {
        const int f = e / nyp, j = e % nyp;
        bcv[e] = sV[f * npr + j];
        kind[e] = sK[f * npr + j];
    }
}

cudaError_t launch_cn_part(const Dims& d, const CnArgs& a, double* tabs, double* bcv, signed char* kind,
                           const int* bc_type, const double* bc_c1, cudaStream_t st) {
    const int RC = part_rows(d.nyp);
    if (RC == 0) return cudaErrorInvalidValue;
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
    const int npr = 16 * RC;
    const size_t smem = sizeof(double) * ((size_t)4 * d.nf * npr + (size_t)d.nf * 16 * 6) + (size_t)d.nf * npr;
    cudaFuncSetAttribute(k_cn_part, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_cn_part<<<1, 256, smem, st>>>(c, RC, tabs, bcv, kind);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// The column kernel.  NW warps (NW >= nf, NW >= 2); RC rows per CN block,
// RP = (RC+1)/2 rows per phi block; NROW = 32*RP padded rows in shared memory.
// ---------------------------------------------------------------------------
template <int NW, int RC, typename TN>
__global__ void __launch_bounds__(32 * NW, (NW == 4 ? 4 : 2))
k_colpart(ColArgs A, const TN* __restrict__ nl, const double* __restrict__ tabs, int tstride) {
    constexpr int RP = (RC + 1) / 2;
    constexpr int NROW = 32 * RP;
    constexpr int NTHMAX = NW - 3 < 4 ? NW - 3 : 4;
    const CnArgs& a = A.cn;
    const Dims& d = a.d;
    const int nf = d.nf, ny = d.ny, nyp = d.nyp;
    extern __shared__ __align__(16) unsigned char smem[];
    double2* sU = reinterpret_cast<double2*>(smem);            // [nf][NROW][2]
    double2* sP = sU + (size_t)nf * NROW * 2;                   // [NROW][2]
    double2* sPhi = sP + NROW * 2;                              // [NROW][2]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const size_t ps = d.splane();
    const size_t fs = ps * nyp;
    const size_t g0 = (size_t)blockIdx.x * 2;
    const bool proj = A.project != 0;

    // ---- phase 0: old CU (all fields) and CP of both columns to shared -----
    for (int e = tid; e < (nf + 1) * NROW * 2; e += 32 * NW) {
        const int c = e & 1, rest = e >> 1;
        const int j = rest % NROW, f = rest / NROW;
        double2 v = make_double2(0.0, 0.0);
        if (j < nyp) {
            const double2* src = (f < nf ? a.cu + (size_t)f * fs : a.cp) + (size_t)j * ps + g0 + c;
            v = *src;
        }
        if (f < nf) sU[((size_t)f * NROW + j) * 2 + c] = v;
        else sP[j * 2 + c] = v;
    }
    __syncthreads();
    auto SU = [&](int f, int j, int c) -> double2 { return sU[((size_t)f * NROW + j) * 2 + c]; };

    // ---- phases 1-2: RHS and CN solve, warp = field ------------------------
    const int f = warp;
    const bool fw = f < nf;
    double2 x[RC];
    {
        const int c = lane >> 4, k = lane & 15;
        const size_t g = g0 + c;
        const int kx = (int)(g % d.ldx), m = (int)(g / d.ldx);
        const bool zero_mode = (kx == 0 && m == 0);
        const double KX = a.kx[kx], KZ = a.kz[m];
        const double k2 = A.k2[g];
        const bool rk1 = a.rk_step > 1;
        const int fe = fw ? f : 0;
        double nuf = a.nu, cU1 = 0.0, cU3 = 0.0, cn_c = a.temp1 * a.nu_v_scale, Kf = 0.0;
        double cth[NTHMAX > 0 ? NTHMAX : 1];
#pragma unroll
        for (int n = 0; n < NTHMAX; ++n) cth[n] = 0.0;
        if (f == 0) {
            cU3 = a.i_ro; Kf = KX;
#pragma unroll
            for (int n = 0; n < NTHMAX; ++n) cth[n] = n < d.nth ? a.ri[n] * a.grav_x : 0.0;
        } else if (f == 2) {
            cU1 = -a.i_ro; Kf = KZ;
#pragma unroll
            for (int n = 0; n < NTHMAX; ++n) cth[n] = n < d.nth ? a.ri[n] * a.grav_z : 0.0;
        } else if (f >= 3 && fw) {
            const int n = f - 3;
            nuf = a.nu / a.pr[n];
            cU1 = -a.drhodx[n];
            cU3 = -a.drhodz[n];
            cn_c = (a.temp1 / a.pr[n]) * a.nu_v_scale;
        }
        const bool isu2 = (f == 1);
        const bool buoy_y = isu2 && !zero_mode;
        const double force = (f == 0 && zero_mode) ? a.forcing : 0.0;
        const int cf_lo = a.cf_lo[fe], cf_hi = a.cf_hi[fe];
        const double* RDY = A.rows + RT_RDY * nyp;
        const double* E1P = A.rows + RT_E1P * nyp;
        const double* E1M = A.rows + RT_E1M * nyp;
        const double* E2P = A.rows + RT_E2P * nyp;
        const double* E2M = A.rows + RT_E2M * nyp;
        const double* BY0 = A.rows + RT_BY0 * nyp;
        const double* BY1 = A.rows + RT_BY1 * nyp;
        const TN* nlf = nl + (size_t)fe * fs + g;
        const double2* cff = a.cf + (size_t)fe * fs + g;
        double2* cfo = a.cf + (size_t)fe * fs + g;
        const double2 zero = make_double2(0.0, 0.0);
        if (fw) {
#pragma unroll
            for (int r = 0; r < RC; ++r) {
                const int j = k * RC + r;
                double2 G = zero;
                if (j < nyp) {
                    const double2 w1 = SU(f, j, c);
                    const double2 w0 = j >= 1 ? SU(f, j - 1, c) : zero;
                    const double2 w2 = SU(f, j + 1, c);
                    const double2 nlj = as_d2(nlf[(size_t)j * ps]);
                    const double2 cfj = rk1 ? cff[(size_t)j * ps] : zero;
                    const double2 cpj = sP[j * 2 + c];
                    const double2 cpm = j >= 1 ? sP[(j - 1) * 2 + c] : zero;
                    double2 cpl = cU1 * SU(0, j, c) + cU3 * SU(2, j, c);
#pragma unroll
                    for (int n = 0; n < NTHMAX; ++n) {
                        if (n < d.nth) {
                            const double2 thj = SU(3 + n, j, c);
                            const double2 thm = j >= 1 ? SU(3 + n, j - 1, c) : zero;
                            cpl = cpl + cth[n] * thj;
                            if (buoy_y) cpl = cpl + (a.ri[n] * a.grav_y) * (BY0[j] * thj + BY1[j] * thm);
                        }
                    }
                    const int row = f * nyp + j;
                    const int knd = a.kind[row];
                    if (j >= cf_lo && j <= cf_hi) {
                        const double2 CF = (-nuf * k2) * w1 + cpl + nlj;
                        if (a.store_cf) cfo[(size_t)j * ps] = CF;
                        if (knd == 0) {
                            double2 R = w1;
                            if (rk1) R = R + a.temp3 * cfj;
                            R = R - a.temp4 * ik(Kf, cpj);
                            if (isu2) R = R - (a.temp4 * RDY[j]) * (cpj - cpm);
                            R.x -= force;
                            R = R + a.temp5 * CF;
                            const double ep = isu2 ? E2P[j] : E1P[j], em = isu2 ? E2M[j] : E1M[j];
                            const double2 ex = ep * (w2 - w1) - em * (w1 - w0);
                            G = R + cn_c * ex;
                        }
                    }
                    if (knd != 0) G = zero_mode ? make_double2(a.bcv[row], 0.0) : zero;
                }
                x[r] = G;
            }
            // partition solve with the precomputed factors of field f
            const double* tb = tabs + (size_t)fe * tstride;
            const PartTab T{16 * RC};
            const int i0 = k * RC;
#pragma unroll
            for (int r = 2; r <= RC - 2; ++r) x[r] = x[r] - tb[T.M() + i0 + r] * x[r - 1];
            x[RC - 2] = tb[T.RB() + i0 + RC - 2] * x[RC - 2];
#pragma unroll
            for (int r = RC - 3; r >= 1; --r) x[r] = tb[T.RB() + i0 + r] * (x[r] - tb[T.C() + i0 + r] * x[r + 1]);
            const double2 Ds = x[0] - tb[T.C() + i0] * x[1];
            const double2 De = x[RC - 1] - tb[T.A() + i0 + RC - 1] * x[RC - 2];
            const double2 Dsn = shfl_dn2(Ds, 1, 16);
            double2 rk = De - tb[T.blk(PB_W1) + k] * Ds - (k < 15 ? tb[T.blk(PB_W2) + k] : 0.0) * Dsn;
#pragma unroll
            for (int st = 0; st < 4; ++st) {
                const int sg = 1 << st;
                const double2 rl = shfl_up2(rk, sg, 16);
                const double2 rh = shfl_dn2(rk, sg, 16);
                const double pa = tb[T.blk(PB_PA0 + st) + k], pg = tb[T.blk(PB_PG0 + st) + k];
                rk = rk - (k >= sg ? pa : 0.0) * rl - (k + sg < 16 ? pg : 0.0) * rh;
            }
            const double2 t = tb[T.blk(PB_RBT) + k] * rk;
            double2 tp = shfl_up2(t, 1, 16);
            if (k == 0) tp = zero;
            const double2 u = tb[T.blk(PB_RBS) + k] * Ds - tb[T.blk(PB_AS) + k] * tp - tb[T.blk(PB_CS) + k] * t;
#pragma unroll
            for (int r = 1; r <= RC - 2; ++r) x[r] = x[r] + tb[T.P() + i0 + r] * u + tb[T.Q() + i0 + r] * t;
            x[0] = u;
            x[RC - 1] = t;
        }
    }
    __syncthreads();                 // every warp is done reading the old state
    if (fw) {
        const int c = lane >> 4, k = lane & 15;
        const int cb_lo = a.cb_lo[f];
        double2* cuo = a.cu + (size_t)f * fs + g0 + c;
#pragma unroll
        for (int r = 0; r < RC; ++r) {
            const int j = k * RC + r;
            if (j < nyp) {
                if (proj && f < 3) sU[((size_t)f * NROW + j) * 2 + c] = x[r];
                else if (j >= cb_lo) cuo[(size_t)j * ps] = x[r];
            }
        }
    }
    if (!proj) return;
    __syncthreads();

    // ---- phase 4: phi of each column, warp c = column ----------------------
    if (warp < 2) {
        const int c = warp, k = lane;
        const size_t g = g0 + c;
        const int kx = (int)(g % d.ldx), m = (int)(g / d.ldx);
        const bool zero_mode = (kx == 0 && m == 0);
        const double KX = a.kx[kx], KZ = a.kz[m];
        const double K2 = KX * KX + KZ * KZ;
        const double* RDYF = A.rows + RT_RDYF * nyp;
        const double* E1P = A.rows + RT_E1P * nyp;
        const double* E1M = A.rows + RT_E1M * nyp;
        // row coefficients of the phi system (APPLY_BC_REM_DIV_MPI rows 1, NY)
        auto coef = [&](int j, double& A_, double& B_, double& C_) {
            A_ = 0.0; B_ = 1.0; C_ = 0.0;
            if (j == ny) { A_ = 1.0; B_ = -1.0; }
            else if (j == 1) { C_ = zero_mode ? 0.0 : -1.0; }
            else if (j >= 2 && j < ny) { A_ = E1M[j]; B_ = -K2 - E1P[j] - E1M[j]; C_ = E1P[j]; }
        };
        const int jb = k * RP;
        double2 y[RP];
#pragma unroll
        for (int r = 0; r < RP; ++r) {
            const int j = jb + r;
            double2 G = make_double2(0.0, 0.0);
            if (j >= 2 && j < ny)
                G = ik(KX, SU(0, j, c)) + RDYF[j] * (SU(1, j + 1, c) - SU(1, j, c)) + ik(KZ, SU(2, j, c));
            y[r] = G;
        }
        // interior elimination: y -> local solution, pp -> p, qq -> q
        double rb[RP], pp[RP], qq[RP];
        {
            double A_, B_, C_, Cp;
            coef(jb + 1, A_, B_, C_);
            double beta = B_;
            rb[1] = rcp_guard(beta);
            pp[1] = -A_;
            Cp = C_;
#pragma unroll
            for (int r = 2; r <= RP - 2; ++r) {
                coef(jb + r, A_, B_, C_);
                const double mlt = A_ * rb[r - 1];
                beta = B_ - mlt * Cp;
                rb[r] = rcp_guard(beta);
                y[r] = y[r] - mlt * y[r - 1];
                pp[r] = -mlt * pp[r - 1];
                Cp = C_;
            }
            y[RP - 2] = rb[RP - 2] * y[RP - 2];
            pp[RP - 2] = rb[RP - 2] * pp[RP - 2];
            qq[RP - 2] = -Cp * rb[RP - 2];
#pragma unroll
            for (int r = RP - 3; r >= 1; --r) {
                coef(jb + r, A_, B_, C_);
                y[r] = rb[r] * (y[r] - C_ * y[r + 1]);
                pp[r] = rb[r] * (pp[r] - C_ * pp[r + 1]);
                qq[r] = -C_ * qq[r + 1] * rb[r];
            }
        }
        double as, Bs, Cs, Ae, Be, ce;
        {
            double A_, B_, C_;
            coef(jb, A_, B_, C_);
            as = A_; Bs = B_ + C_ * pp[1]; Cs = C_ * qq[1];
            y[0] = y[0] - C_ * y[1];                    // D_s
            coef(jb + RP - 1, A_, B_, C_);
            Ae = A_ * pp[RP - 2]; Be = B_ + A_ * qq[RP - 2]; ce = C_;
            y[RP - 1] = y[RP - 1] - A_ * y[RP - 2];     // D_e
        }
        const double2 Ds = y[0], De = y[RP - 1];
        const double rBs = rcp_guard(Bs);
        // next block's first-row quantities
        const double asn = __shfl_down_sync(0xffffffffu, as, 1);
        const double Csn = __shfl_down_sync(0xffffffffu, Cs, 1);
        const double rBn = __shfl_down_sync(0xffffffffu, rBs, 1);
        const double2 Dsn = shfl_dn2(Ds, 1, 32);
        const bool nxt = k < 31;
        double al = -Ae * as * rBs;
        double be = Be - Ae * Cs * rBs - (nxt ? ce * asn * rBn : 0.0);
        double ga = nxt ? -ce * Csn * rBn : 0.0;
        double2 rr = De - (Ae * rBs) * Ds - (nxt ? ce * rBn : 0.0) * Dsn;
#pragma unroll
        for (int st = 0; st < 5; ++st) {
            const int sg = 1 << st;
            const double all = __shfl_up_sync(0xffffffffu, al, sg), bel = __shfl_up_sync(0xffffffffu, be, sg),
                         gal = __shfl_up_sync(0xffffffffu, ga, sg);
            const double alh = __shfl_down_sync(0xffffffffu, al, sg), beh = __shfl_down_sync(0xffffffffu, be, sg),
                         gah = __shfl_down_sync(0xffffffffu, ga, sg);
            const double2 rl = shfl_up2(rr, sg, 32), rh = shfl_dn2(rr, sg, 32);
            const bool hl = k >= sg, hh = k + sg < 32;
            const double fa = hl ? al * rcp_guard(bel) : 0.0;
            const double fg = hh ? ga * rcp_guard(beh) : 0.0;
            const double al2 = hl ? -fa * all : 0.0;
            const double ga2 = hh ? -fg * gah : 0.0;
            be = be - (hl ? fa * gal : 0.0) - (hh ? fg * alh : 0.0);
            rr = rr - fa * rl - fg * rh;
            al = al2;
            ga = ga2;
        }
        const double2 t = rcp_guard(be) * rr;
        double2 tp = shfl_up2(t, 1, 32);
        if (k == 0) tp = make_double2(0.0, 0.0);
        const double2 u = rBs * (Ds - as * tp - Cs * t);
#pragma unroll
        for (int r = 0; r < RP; ++r) {
            const int j = k * RP + r;
            double2 phi = (r == 0) ? u : (r == RP - 1) ? t : y[r] + pp[r] * u + qq[r] * t;
            if (j < 1 || j > ny) phi = make_double2(0.0, 0.0);
            sPhi[j * 2 + c] = phi;
        }
    }
    __syncthreads();

    // ---- phase 5: velocity correction, CP update, phi out ------------------
    const double* RDY = A.rows + RT_RDY * nyp;
    for (int e = tid; e < 4 * nyp * 2; e += 32 * NW) {
        const int c = e & 1, rest = e >> 1;
        const int j = rest % nyp, q = rest / nyp;
        const size_t g = g0 + c;
        if (q < 3) {
            if (j < a.cb_lo[q]) continue;
            double2 v = SU(q, j, c);
            if (j >= 1 && j <= ny) {
                const double2 phi = sPhi[j * 2 + c];
                if (q == 0) v = v - ik(a.kx[g % d.ldx], phi);
                else if (q == 2) v = v - ik(a.kz[g / d.ldx], phi);
                else if (j >= 2) v = v - RDY[j] * (phi - sPhi[(j - 1) * 2 + c]);
            }
            a.cu[(size_t)q * fs + (size_t)j * ps + g] = v;
        } else if (j >= 1 && j <= ny) {
            const double2 phi = sPhi[j * 2 + c];
            if (A.update_cp && j >= 2) {
                double2* cpo = const_cast<double2*>(a.cp);
                cpo[(size_t)j * ps + g] = sP[j * 2 + c] + A.inv_h * phi;
            }
            if (A.store_phi) A.phi[(size_t)j * ps + g] = phi;
        }
    }
}

template <typename TN>
size_t colpart_smem(const Dims& d) {
    const int RC = part_rows(d.nyp);
    const int NROW = 32 * ((RC + 1) / 2);
    return sizeof(double2) * (size_t)NROW * 2 * (d.nf + 2);
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
#define DGPU_RC_CASES(NW)                                        \
    switch (RC) {                                                \
        case 5: go(k_colpart<NW, 5, TN>, NW); break;             \
        case 9: go(k_colpart<NW, 9, TN>, NW); break;             \
        case 17: go(k_colpart<NW, 17, TN>, NW); break;           \
        case 33: go(k_colpart<NW, 33, TN>, NW); break;           \
        default: return cudaErrorInvalidValue;                   \
    }
    if (d.nf <= 4) { DGPU_RC_CASES(4) }
    else if (d.nf <= 8) { DGPU_RC_CASES(8) }
    else return cudaErrorInvalidValue;
#undef DGPU_RC_CASES
    return cudaGetLastError();
}

template cudaError_t launch_colpart<cpx<float>>(const ColArgs&, const cpx<float>*, const double*, cudaStream_t);
template cudaError_t launch_colpart<cpx<double>>(const ColArgs&, const cpx<double>*, const double*, cudaStream_t);
template size_t colpart_smem<cpx<float>>(const Dims&);
template size_t colpart_smem<cpx<double>>(const Dims&);

}  // namespace dgpu
