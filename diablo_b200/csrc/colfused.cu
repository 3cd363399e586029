// colfused.cu -- the column work of one RK_CHAN_1 substage in one kernel:
// Fourier RHS assembly, Crank-Nicolson y solves of every field
// (channel.f:77-293, 581-626, 737-1029), the REM_DIV_CHAN projection
// (channel.f:1103-1214) and the pressure update CP += phi/h
// (channel.f:1059-1065), for CB consecutive (kx,kz) columns per block.
//
// Data movement: the columns of a block are one contiguous 16-byte-aligned
// run in every plane of the S layout, so each (row, field, array) slice is a
// single 1-D bulk copy.  A ring of D shared-memory stages, refilled by one
// thread with cp.async.bulk and tracked by one mbarrier per stage, keeps up
// to D rows of every operand in flight while the lanes sweep the rows.
//
// Lanes: one lane per (column, field); a warp holds CW = 32/FS columns and
// FS field slots (lane = field*CW + column).  Couplings between fields are
// warp shuffles.  Three sweeps:
//   1 ascending:  RHS, new CF, forward elimination (G' to global)
//   2 descending: back substitution (CU to global); divergence of the new
//                 velocity and the reverse elimination of the phi system
//   3 ascending:  phi, velocity correction, CP update, phi to global.
// The CN factors are shared by all columns (built by k_cn_coef).  The phi
// system is eliminated bottom-up here (the reference sweeps top-down,
// mpi.f:700-865); both are exact for these diagonally dominant systems and
// agree to round-off.
#include <cuda_runtime.h>

#include "kernels.cuh"
#include "launch.h"
#include "tma.cuh"

namespace dgpu {

namespace {

__device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 operator*(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
__device__ __forceinline__ double2 ik(double K, double2 a) { return make_double2(-K * a.y, K * a.x); }
__device__ __forceinline__ double2 shfl2(double2 v, int src) {
    return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}
template <typename TN>
__device__ __forceinline__ double2 as_d2(const TN& v) { return make_double2((double)v.x, (double)v.y); }

struct StageGeom {
    uint32_t szC, szN, bytes;
    uint32_t oCF, oNL, oCP;      // sweep 1
    uint32_t oB, oG, oCP3;       // sweep 3
};

template <int CB, typename TN>
__host__ __device__ inline StageGeom stage_geom(int nf) {
    StageGeom s;
    s.szC = CB * 16;
    s.szN = CB * (uint32_t)sizeof(TN);
    s.oCF = nf * s.szC;
    s.oNL = 2 * nf * s.szC;
    s.oCP = s.oNL + nf * s.szN;
    const uint32_t b1 = s.oCP + s.szC;
    s.oB = 3 * s.szC;
    s.oG = s.oB + CB * 8;
    s.oCP3 = s.oG + s.szC;
    const uint32_t b3 = s.oCP3 + s.szC;
    s.bytes = ((b1 > b3 ? b1 : b3) + 15) / 16 * 16;
    return s;
}

}  // namespace

template <int FS, typename TN, int D>
__global__ void __launch_bounds__(128, 4) k_column(ColArgs A, const TN* __restrict__ nl) {
    constexpr int CW = 32 / FS;
    constexpr int CB = 4 * CW;
    constexpr int NTHMAX = FS - 3 < 4 ? FS - 3 : 4;
    const CnArgs& a = A.cn;
    const Dims& d = a.d;
    const int nf = d.nf, ny = d.ny, nyp = d.nyp;
    extern __shared__ __align__(128) unsigned char smem[];
    const StageGeom sg = stage_geom<CB, TN>(nf);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + (size_t)D * sg.bytes);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int c = lane % CW, f = lane / CW;
    const int cl = warp * CW + c;                       // column within the block
    const size_t gblk = (size_t)blockIdx.x * CB;        // first column of the block
    const size_t g = gblk + cl;
    const int kx = (int)(g % d.ldx), m = (int)(g / d.ldx);
    const bool fvalid = f < nf;
    const int fe = fvalid ? f : nf - 1;
    const size_t ps = d.splane();
    const size_t fs = ps * nyp;
    const bool zero_mode = (kx == 0 && m == 0);
    const double KX = a.kx[kx], KZ = a.kz[m];
    const double k2 = A.k2[g];                          // (KX^2+KZ^2)**BETA
    const double K2 = KX * KX + KZ * KZ;
    const bool rk1 = a.rk_step > 1;
    int* err = A.err;

    if (tid == 0) {
        for (int s = 0; s < D; ++s) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    __syncthreads();

    // ---- producer (warp 0): one stage = one row of every operand -----------
    // lane 0 posts the byte count, then lane i issues the i-th bulk copy.
    auto issue = [&](int q, int sweep, int j) {
        uint64_t* bar = &bars[q % D];
        unsigned char* base = smem + (size_t)(q % D) * sg.bytes;
        const size_t off = (size_t)j * ps + gblk;
        uint32_t bytes;
        int ncopy;
        if (sweep == 1) { bytes = nf * sg.szC * (rk1 ? 2 : 1) + nf * sg.szN + sg.szC; ncopy = 3 * nf + 1; }
        else if (sweep == 2) { bytes = nf * sg.szC; ncopy = nf; }
        else { bytes = 5 * sg.szC + CB * 8; ncopy = 6; }
        if (lane == 0) mbar_arrive_expect_tx(bar, bytes);
        __syncwarp();
        const int l = lane;
        if (l < ncopy) {
            if (sweep == 1) {
                if (l < nf) bulk_g2s(base + l * sg.szC, a.cu + l * fs + off, sg.szC, bar);
                else if (l < 2 * nf) {
                    if (rk1) bulk_g2s(base + sg.oCF + (l - nf) * sg.szC, a.cf + (l - nf) * fs + off, sg.szC, bar);
                } else if (l < 3 * nf) {
                    bulk_g2s(base + sg.oNL + (l - 2 * nf) * sg.szN, nl + (l - 2 * nf) * fs + off, sg.szN, bar);
                } else {
                    bulk_g2s(base + sg.oCP, a.cp + off, sg.szC, bar);
                }
            } else if (sweep == 2) {
                bulk_g2s(base + l * sg.szC, a.cu + l * fs + off, sg.szC, bar);
            } else {
                if (l < 3) bulk_g2s(base + l * sg.szC, a.cu + l * fs + off, sg.szC, bar);
                else if (l == 3) bulk_g2s(base + sg.oB, A.bsc + off, CB * 8, bar);
                else if (l == 4) bulk_g2s(base + sg.oG, A.gsc + off, sg.szC, bar);
                else bulk_g2s(base + sg.oCP3, a.cp + off, sg.szC, bar);
            }
        }
    };
    auto stage = [&](int q) -> unsigned char* { return smem + (size_t)(q % D) * sg.bytes; };
    auto wait = [&](int q) { mbar_wait_bounded(&bars[q % D], (uint32_t)((q / D) & 1), err); };
    auto ldC = [&](int q, uint32_t off, int fld) -> double2 {
        return reinterpret_cast<const double2*>(stage(q) + off + fld * sg.szC)[cl];
    };

    // ---- per-lane coefficients of the explicit terms ------------------------
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
    } else if (f >= 3 && fvalid) {
        const int n = f - 3;
        nuf = a.nu / a.pr[n];
        cU1 = -a.drhodx[n];
        cU3 = -a.drhodz[n];
        cn_c = (a.temp1 / a.pr[n]) * a.nu_v_scale;
    }
    const bool isu2 = (f == 1);
    const bool buoy_y = isu2 && !zero_mode;
    const double force = (f == 0 && zero_mode) ? a.forcing : 0.0;
    const int cf_lo = a.cf_lo[fe], cf_hi = a.cf_hi[fe], cb_lo = a.cb_lo[fe];
    double2* cuo = a.cu + (size_t)fe * fs + g;
    double2* cfo = a.cf + (size_t)fe * fs + g;
    const double2 zero = make_double2(0.0, 0.0);
    const double* RDY = A.rows + RT_RDY * nyp;
    const double* RDYF = A.rows + RT_RDYF * nyp;
    const double* E1P = A.rows + RT_E1P * nyp;
    const double* E1M = A.rows + RT_E1M * nyp;
    const double* E2P = A.rows + RT_E2P * nyp;
    const double* E2M = A.rows + RT_E2M * nyp;
    const double* BY0 = A.rows + RT_BY0 * nyp;
    const double* BY1 = A.rows + RT_BY1 * nyp;

    // ======================= sweep 1 (ascending) ==============================
    const int n1 = ny + 2;
    if (warp == 0)
        for (int q = 0; q < D && q < n1; ++q) issue(q, 1, q);
    wait(0);
    wait(1);
    double2 w0 = zero, w1 = ldC(0, 0, fe), w2 = ldC(1, 0, fe);
    double2 cpm = zero, cpj = ldC(0, sg.oCP, 0), cpn = ldC(1, sg.oCP, 0);
    double2 gprev = zero, g0 = zero;
    for (int j = 0; j <= ny + 1; ++j) {
        const TN nlr = reinterpret_cast<const TN*>(stage(j) + sg.oNL + fe * sg.szN)[cl];
        const double2 nlj = as_d2(nlr);
        const double2 cfj = rk1 ? ldC(j, sg.oCF, fe) : zero;
        const double2 u1j = shfl2(w1, 0 * CW + c);
        const double2 u3j = shfl2(w1, 2 * CW + c);
        double2 cpl = cU1 * u1j + cU3 * u3j;
#pragma unroll
        for (int n = 0; n < NTHMAX; ++n) {
            const double2 thj = shfl2(w1, (3 + n) * CW + c);
            const double2 thm = shfl2(w0, (3 + n) * CW + c);
            cpl = cpl + cth[n] * thj;
            if (buoy_y && n < d.nth)
                cpl = cpl + (a.ri[n] * a.grav_y) * (BY0[j] * thj + BY1[j] * thm);
        }
        const int row = fe * nyp + j;
        const int knd = a.kind[row];
        double2 G = zero;
        if (j >= cf_lo && j <= cf_hi) {
            const double2 CF = (-nuf * k2) * w1 + cpl + nlj;
            if (fvalid && a.store_cf) cfo[(size_t)j * ps] = CF;
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
        if (j == 0) {
            g0 = G;
            gprev = G;
        } else {
            G = G + a.mult[row] * gprev;
            gprev = G;
            if (fvalid) cuo[(size_t)j * ps] = G;
        }
        __syncthreads();                         // stage j consumed by all lanes
        if (warp == 0 && j + D < n1) issue(j + D, 1, j + D);
        w0 = w1;
        w1 = w2;
        cpm = cpj;
        cpj = cpn;
        if (j + 2 <= ny + 1) {
            wait(j + 2);
            w2 = ldC(j + 2, 0, fe);
            cpn = ldC(j + 2, sg.oCP, 0);
        } else {
            w2 = zero;
            cpn = zero;
        }
    }

    // ======================= sweep 2 (descending) =============================
    fence_proxy_async_global();
    __syncthreads();
    const int q2base = n1;                       // rows ny+1 .. 1
    const int n2 = ny + 1;
    if (warp == 0)
        for (int i = 0; i < D && i < n2; ++i) issue(q2base + i, 2, ny + 1 - i);
    double2 xn = zero;                           // own field's x(j+1)
    double rbt_n = 0.0, a_n = 0.0;               // phi system: reverse-eliminated row j+1
    double2 gt_n = zero;
    const bool proj = A.project != 0;
    const bool phi_lane = (f == FS - 1);
    for (int j = ny + 1; j >= 0; --j) {
        const int i = ny + 1 - j;
        double2 gj;
        if (j >= 1) {
            wait(q2base + i);
            gj = ldC(q2base + i, 0, fe);
        } else {
            gj = g0;
        }
        const int row = fe * nyp + j;
        const double ipv = a.piv[row];
        double2 x;
        if (j == ny + 1) x = ipv * gj;
        else x = ipv * (gj - a.cup[row] * xn);
        if (fvalid && j >= cb_lo) cuo[(size_t)j * ps] = x;
        if (proj && j >= 1 && j <= ny) {
            const double2 x1 = shfl2(x, 0 * CW + c);
            const double2 x2 = shfl2(x, 1 * CW + c);
            const double2 x3 = shfl2(x, 2 * CW + c);
            const double2 x2p = shfl2(xn, 1 * CW + c);
            double Aj, Bj, Cj;
            double2 Gj;
            if (j == ny) { Aj = 1.0; Bj = -1.0; Cj = 0.0; Gj = zero; }
            else if (j == 1) { Aj = 0.0; Bj = 1.0; Cj = zero_mode ? 0.0 : -1.0; Gj = zero; }
            else {
                Aj = E1M[j];
                Bj = -K2 - E1P[j] - E1M[j];
                Cj = E1P[j];
                Gj = ik(KX, x1) + RDYF[j] * (x2p - x2) + ik(KZ, x3);
            }
            double bt;
            double2 gt;
            if (j == ny) { bt = Bj; gt = Gj; }
            else {
                const double fac = Cj * rbt_n;
                bt = Bj - fac * a_n;
                gt = Gj - fac * gt_n;
            }
            const double rbt = bt != 0.0 ? 1.0 / bt : 0.0;   // the one division per row
            if (phi_lane) {
                A.bsc[(size_t)j * ps + g] = rbt;
                A.gsc[(size_t)j * ps + g] = gt;
            }
            rbt_n = rbt;
            gt_n = gt;
            a_n = Aj;
        }
        xn = x;
        __syncthreads();
        if (warp == 0 && j >= 1 && i + D < n2) issue(q2base + i + D, 2, ny + 1 - (i + D));
    }
    if (!proj) return;

    // ======================= sweep 3 (ascending) ==============================
    fence_proxy_async_global();
    __syncthreads();
    const int q3base = q2base + n2;              // rows 1 .. ny
    const int n3 = ny;
    if (warp == 0)
        for (int i = 0; i < D && i < n3; ++i) issue(q3base + i, 3, 1 + i);
    const int f3 = f < 3 ? f : 0;
    double2 phip = zero;                          // phi(j-1)
    for (int j = 1; j <= ny; ++j) {
        const int q = q3base + j - 1;
        wait(q);
        const unsigned char* st = stage(q);
        const double rbt = reinterpret_cast<const double*>(st + sg.oB)[cl];
        const double2 gt = reinterpret_cast<const double2*>(st + sg.oG)[cl];
        const double Aj = (j == 1) ? 0.0 : (j == ny ? 1.0 : E1M[j]);
        const double2 phi = rbt * (gt - Aj * phip);
        const double2 u = ldC(q, 0, f3);
        if (f == 0) cuo[(size_t)j * ps] = u - ik(KX, phi);
        else if (f == 2) cuo[(size_t)j * ps] = u - ik(KZ, phi);
        else if (f == 1 && j >= 2) cuo[(size_t)j * ps] = u - RDY[j] * (phi - phip);
        if (phi_lane) {
            if (A.update_cp && j >= 2) {
                const double2 cpv = reinterpret_cast<const double2*>(st + sg.oCP3)[cl];
                double2* cpo = const_cast<double2*>(a.cp) + g;
                cpo[(size_t)j * ps] = cpv + A.inv_h * phi;
            }
            if (A.store_phi) A.phi[(size_t)j * ps + g] = phi;
        }
        phip = phi;
        __syncthreads();
        if (warp == 0 && j - 1 + D < n3) issue(q + D, 3, j + D);
    }
}

template <typename TN>
size_t column_smem(const Dims& d) {
    constexpr int D = COL_STAGES;
    if (d.nf <= 4) return (size_t)D * stage_geom<32, TN>(d.nf).bytes + D * sizeof(uint64_t);
    return (size_t)D * stage_geom<16, TN>(d.nf).bytes + D * sizeof(uint64_t);
}

template <typename TN>
cudaError_t launch_column(const ColArgs& a, const TN* nl, cudaStream_t st) {
    constexpr int D = COL_STAGES;
    const Dims& d = a.cn.d;
    const size_t ncol = d.splane();
    const size_t smem = column_smem<TN>(d);
    auto go = [&](auto kern, int cb) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<(unsigned)(ncol / cb), 128, smem, st>>>(a, nl);
    };
    if (d.nf <= 4) go(k_column<4, TN, D>, 32);
    else if (d.nf <= 8) go(k_column<8, TN, D>, 16);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

template cudaError_t launch_column<cpx<float>>(const ColArgs&, const cpx<float>*, cudaStream_t);
template cudaError_t launch_column<cpx<double>>(const ColArgs&, const cpx<double>*, cudaStream_t);
template size_t column_smem<cpx<float>>(const Dims&);
template size_t column_smem<cpx<double>>(const Dims&);

}  // namespace dgpu
