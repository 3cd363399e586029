// column.cu -- FP64 column kernels: the Crank-Nicolson y solves of RK_CHAN_1
// and the REM_DIV_CHAN projection, one thread per Fourier column (kx, kz).
//
// The reference solves the implicit y systems in physical space, one (x,z)
// column at a time (channel.f:762-1029 with THOMAS_*_REAL_MPI,
// mpi.f:630-809).  Without LES the y operator does not depend on x or z and
// every field is band-limited, so the same solves are done here in Fourier
// space, one column per retained (kx,kz) mode; the boundary rows carry the
// wall values only in the (0,0) mode, which is the Fourier image of a value
// that is constant over the wall.  The tridiagonal factors are then shared
// by all columns and are built once per substage by k_cn_coef.
#include <cuda_runtime.h>

#include "kernels.cuh"
#include "launch.h"

namespace dgpu {

__device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 operator*(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
__device__ __forceinline__ double2 operator/(double2 a, double s) { return make_double2(a.x / s, a.y / s); }
// (i K) * a
__device__ __forceinline__ double2 ik(double K, double2 a) { return make_double2(-K * a.y, K * a.x); }

template <typename TN>
__device__ __forceinline__ double2 ldn(const TN* p);
template <>
__device__ __forceinline__ double2 ldn<cpx<float>>(const cpx<float>* p) {
    const float2 v = *reinterpret_cast<const float2*>(p);
    return make_double2((double)v.x, (double)v.y);
}
template <>
__device__ __forceinline__ double2 ldn<cpx<double>>(const cpx<double>* p) {
    return *reinterpret_cast<const double2*>(p);
}

// ---------------------------------------------------------------------------
// Tridiagonal rows of each CN system and their forward elimination.
// bc_type/bc_c1 per field: [lower, upper].  Row set-up replays the order of
// the reference: interior rows, then the lower and upper BC routines
// (APPLY_BC_TH_*, APPLY_BC_2_*, APPLY_BC_1_*, APPLY_BC_3_*).
// ---------------------------------------------------------------------------
struct CoefParams {
    Dims d;
    const double* dy;
    const double* dyf;
    double temp1, nu_v_scale;
    double pr[4];
    int jstart_th[4];
    int bc_type[MAXF][2];
    double bc_c1[MAXF][2];
};

__global__ void k_cn_coef(CoefParams c, double* mult, double* piv, double* cup, double* bcv,
                          signed char* kind) {
    const int f = threadIdx.x;
    if (f >= c.d.nf) return;
    const int ny = c.d.ny, nyp = c.d.nyp;
    double* L = mult + (size_t)f * nyp;
    double* D = piv + (size_t)f * nyp;
    double* U = cup + (size_t)f * nyp;
    double* V = bcv + (size_t)f * nyp;
    signed char* K = kind + (size_t)f * nyp;
    const double* DY = c.dy;
    const double* DYF = c.dyf;
    auto setrow = [&](int j, double l, double dd, double u, double v) {
        L[j] = l; D[j] = dd; U[j] = u; V[j] = v; K[j] = 1;
    };
    for (int j = 0; j < nyp; ++j) setrow(j, 0.0, 1.0, 0.0, 0.0);
    const int lo = c.bc_type[f][0], hi = c.bc_type[f][1];
    const double clo = c.bc_c1[f][0], chi = c.bc_c1[f][1];
    if (f >= 3) {
        const int n = f - 3;
        const double cc = c.temp1 / c.pr[n] * c.nu_v_scale;
        for (int j = c.jstart_th[n]; j <= ny; ++j) {
            L[j] = -cc / (DY[j] * DYF[j]);
            D[j] = 1. + cc / (DY[j + 1] * DYF[j]) + cc / (DY[j] * DYF[j]);
            U[j] = -cc / (DY[j + 1] * DYF[j]);
            K[j] = 0;
        }
        if (lo == 0) { setrow(0, 0., 1., 0., 0.); setrow(1, 0., 1., 0., clo); }
        else { setrow(1, 0., -1., 1., DY[2] * clo); setrow(0, 0., 1., 0., 0.); }
        if (hi == 0) { setrow(ny + 1, 0., 1., 0., 0.); setrow(ny, 0., 1., 0., chi); }
        else { setrow(ny, -1., 1., 0., DY[ny] * chi); setrow(ny + 1, 0., 1., 0., 0.); }
    } else if (f == 1) {
        const double t = c.temp1 * c.nu_v_scale;
        for (int j = 2; j <= ny; ++j) {
            L[j] = -t / (DYF[j - 1] * DY[j]);
            D[j] = 1. + t / (DYF[j] * DY[j]) + t / (DYF[j - 1] * DY[j]);
            U[j] = -t / (DYF[j] * DY[j]);
            K[j] = 0;
        }
        if (lo == 0) { setrow(1, 0., 1., 0., clo); setrow(2, 0., 1., 0., clo); }
        else { setrow(1, 0., -1., 1., DYF[1] * clo); }
        setrow(0, 0., 1., 0., 0.);
        if (hi == 0) { setrow(ny + 1, 0., 1., 0., chi); setrow(ny, 0., 1., 0., chi); }
        else { setrow(ny + 1, -1., 1., 0., DYF[ny] * chi); }
    } else {
        const double t = c.temp1 * c.nu_v_scale;
        for (int j = 2; j <= ny; ++j) {
            L[j] = -t / (DY[j] * DYF[j]);
            D[j] = 1. - t * (-1. / (DY[j + 1] * DYF[j]) - 1. / (DY[j] * DYF[j]));
            U[j] = -t / (DY[j + 1] * DYF[j]);
            K[j] = 0;
        }
        if (lo == 0) { setrow(0, 0., 1., 0., 0.); setrow(1, 0., 1., 0., clo); }
        else { setrow(0, 0., 1., 0., 0.); setrow(1, 0., -1., 1., DY[2] * clo); }
        if (hi == 0) { setrow(ny + 1, 0., 1., 0., 0.); setrow(ny, 0., 1., 0., chi); }
        else { setrow(ny, -1., 1., 0., DY[ny] * chi); setrow(ny + 1, 0., 1., 0., 0.); }
    }
    // THOMAS_FORWARD_REAL_MPI with NPROCY = 1: rows 1..NY+1 eliminated
    // (mpi.f:668-694); L becomes the multiplier, D the pivot.
    for (int j = 1; j <= ny + 1; ++j) {
        L[j] = -L[j] / D[j - 1];
        D[j] = D[j] + L[j] * U[j - 1];
    }
    L[0] = 0.0;
}

cudaError_t launch_cn_coef(const Dims& d, const CnArgs& a, double* mult, double* piv, double* cup,
                           double* bcv, signed char* kind, const int* bc_type, const double* bc_c1,
                           cudaStream_t st) {
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
    k_cn_coef<<<1, 32, 0, st>>>(c, mult, piv, cup, bcv, kind);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// K4: Fourier RHS assembly (channel.f:77-293, 581-595), explicit half of the
// CN y terms (channel.f:606-626, 737-747), and the CN solves (forward sweep
// ascending, back substitution descending) for every field of one column.
// ---------------------------------------------------------------------------
template <int NTH, typename TN>
__global__ void __launch_bounds__(128) k_cn(CnArgs a, const TN* __restrict__ nl) {
    constexpr int F = 3 + NTH;
    const Dims& d = a.d;
    const int kx = blockIdx.x * 32 + threadIdx.x;
    const int m = blockIdx.y * 4 + threadIdx.y;
    if (kx >= d.nkxp || m >= d.nkzt) return;
    const size_t ps = (size_t)d.nkzt * d.ldx;
    const size_t fs = ps * d.nyp;
    const size_t col = (size_t)m * d.ldx + kx;
    const int ny = d.ny, nyp = d.nyp;
    const bool zero_mode = (kx == 0 && m == 0);
    const double KX = a.kx[kx], KZ = a.kz[m];
    const double k2 = pow(KX * KX + KZ * KZ, a.beta);
    double2* cu = a.cu + col;
    double2* cf = a.cf + col;
    const double2* cp = a.cp + col;
    const TN* nlc = nl + col;
    const double2 zero = make_double2(0.0, 0.0);

    double2 w[F][3];     // CU(j-1), CU(j), CU(j+1) of every field
#pragma unroll
    for (int f = 0; f < F; ++f) {
        w[f][0] = zero;
        w[f][1] = cu[f * fs];
        w[f][2] = cu[f * fs + ps];
    }
    double2 cpm = zero, cpj = cp[0];
    double2 gprev[F], g0[F];

    for (int j = 0; j <= ny + 1; ++j) {
        const double dyj = a.dy[j], dyj1 = (j + 1 < nyp) ? a.dy[j + 1] : 1.0;
        const double dyfj = a.dyf[j], dyfjm = (j > 0) ? a.dyf[j - 1] : 0.0;
#pragma unroll
        for (int f = 0; f < F; ++f) {
            const int row = f * nyp + j;
            const int knd = a.kind[row];
            double2 G = zero;
            if (j >= a.cf_lo[f] && j <= a.cf_hi[f]) {
                const double2 u = w[f][1];
                double2 CF;
                if (f == 0) {
                    CF = (-a.nu * k2) * u + a.i_ro * w[2][1];
#pragma unroll
                    for (int n = 0; n < NTH; ++n) CF = CF + (a.ri[n] * a.grav_x) * w[3 + n][1];
                } else if (f == 2) {
                    CF = (-a.nu * k2) * u - a.i_ro * w[0][1];
#pragma unroll
                    for (int n = 0; n < NTH; ++n) CF = CF + (a.ri[n] * a.grav_z) * w[3 + n][1];
                } else if (f == 1) {
                    CF = (-a.nu * k2) * u;
                    if (!zero_mode) {
#pragma unroll
                        for (int n = 0; n < NTH; ++n)
                            CF = CF + (a.ri[n] * a.grav_y) *
                                          ((dyfjm * w[3 + n][1] + dyfj * w[3 + n][0]) / (2.0 * dyj));
                    }
                } else {
                    const int n = f - 3;
                    CF = (-(a.nu / a.pr[n]) * k2) * u - a.drhodx[n] * w[0][1] - a.drhodz[n] * w[2][1];
                }
                CF = CF + ldn<TN>(nlc + f * fs + j * ps);
                double2 R = u;
                if (a.rk_step > 1) R = R + a.temp3 * cf[f * fs + j * ps];
                if (a.store_cf) cf[f * fs + j * ps] = CF;
                if (knd == 0) {
                    if (f == 0) {
                        R = R - a.temp4 * ik(KX, cpj);
                        if (zero_mode) R.x -= a.forcing;
                    } else if (f == 2) {
                        R = R - a.temp4 * ik(KZ, cpj);
                    } else if (f == 1) {
                        R = R - a.temp4 * ((cpj - cpm) / dyj);
                    }
                    R = R + a.temp5 * CF;
                    double2 ex;
                    if (f == 1)
                        ex = ((w[f][2] - u) / dyfj - (u - w[f][0]) / dyfjm) / dyj;
                    else
                        ex = ((w[f][2] - u) / dyj1 - (u - w[f][0]) / dyj) / dyfj;
                    const double c = (f >= 3) ? (a.temp1 / a.pr[f - 3]) * a.nu_v_scale : a.temp1 * a.nu_v_scale;
                    G = R + c * ex;
                }
            }
            if (knd != 0) G = zero_mode ? make_double2(a.bcv[row], 0.0) : zero;
            if (j == 0) {
                g0[f] = G;
                gprev[f] = G;
            } else {
                G = G + a.mult[row] * gprev[f];
                gprev[f] = G;
                cu[f * fs + j * ps] = G;
            }
        }
        // slide the window
#pragma unroll
        for (int f = 0; f < F; ++f) {
            w[f][0] = w[f][1];
            w[f][1] = w[f][2];
            w[f][2] = (j + 2 <= ny + 1) ? cu[f * fs + (j + 2) * ps] : zero;
        }
        cpm = cpj;
        cpj = (j + 1 <= ny + 1) ? cp[(j + 1) * ps] : zero;
    }
    // back substitution (THOMAS_BACKWARD_REAL_MPI, mpi.f:778-800)
    double2 xn[F];
    for (int j = ny + 1; j >= 0; --j) {
#pragma unroll
        for (int f = 0; f < F; ++f) {
            const int row = f * nyp + j;
            const double2 gj = (j == 0) ? g0[f] : cu[f * fs + j * ps];
            const double pv = a.piv[row];
            double2 x;
            if (j == ny + 1) x = gj / pv;
            else if (pv != 0.0) x = (gj - a.cup[row] * xn[f]) / pv;
            else x = zero;
            xn[f] = x;
            if (j >= a.cb_lo[f]) cu[f * fs + j * ps] = x;
        }
    }
}

template <typename TN>
cudaError_t launch_cn(const CnArgs& a, const TN* nl, cudaStream_t st) {
    dim3 block(32, 4);
    dim3 grid((a.d.nkxp + 31) / 32, (a.d.nkzt + 3) / 4);
    switch (a.d.nth) {
        case 0: k_cn<0, TN><<<grid, block, 0, st>>>(a, nl); break;
        case 1: k_cn<1, TN><<<grid, block, 0, st>>>(a, nl); break;
        case 2: k_cn<2, TN><<<grid, block, 0, st>>>(a, nl); break;
        case 3: k_cn<3, TN><<<grid, block, 0, st>>>(a, nl); break;
        case 4: k_cn<4, TN><<<grid, block, 0, st>>>(a, nl); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}
template cudaError_t launch_cn<cpx<float>>(const CnArgs&, const cpx<float>*, cudaStream_t);
template cudaError_t launch_cn<cpx<double>>(const CnArgs&, const cpx<double>*, cudaStream_t);

// ---------------------------------------------------------------------------
// K5: REM_DIV_CHAN (channel.f:1103-1214) per column with the boundary rows
// of APPLY_BC_REM_DIV_MPI (mpi.f:1239-1278) and the guarded complex Thomas
// of mpi.f:700-865; then the velocity correction and the pressure update
// CP += phi/h (channel.f:1059-1065).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_remdiv(RemDivArgs a) {
    const Dims& d = a.d;
    const int kx = blockIdx.x * 32 + threadIdx.x;
    const int m = blockIdx.y * 4 + threadIdx.y;
    if (kx >= d.nkxp || m >= d.nkzt) return;
    const size_t ps = (size_t)d.nkzt * d.ldx;
    const size_t fs = ps * d.nyp;
    const size_t col = (size_t)m * d.ldx + kx;
    const int ny = d.ny;
    const bool zero_mode = (kx == 0 && m == 0);
    const double KX = a.kx[kx], KZ = a.kz[m];
    const double K2 = KX * KX + KZ * KZ;
    double2* u1 = a.cu + col;
    double2* u2 = a.cu + fs + col;
    double2* u3 = a.cu + 2 * fs + col;
    double* bs = a.bsc + col;
    double2* gs = a.gsc + col;
    const double2 zero = make_double2(0.0, 0.0);
    // row 1 (BC), then forward elimination over rows 2..NY
    double bprev = 1.0, cprev = zero_mode ? 0.0 : -1.0;
    double2 gprev = zero;
    bs[ps] = bprev;
    gs[ps] = gprev;
    double2 u2j = u2[2 * ps];
    for (int j = 2; j <= ny; ++j) {
        double A, B, C;
        double2 G;
        if (j < ny) {
            A = 1. / (a.dy[j] * a.dyf[j]);
            B = -KX * KX - KZ * KZ - 1. / (a.dy[j + 1] * a.dyf[j]) - 1. / (a.dy[j] * a.dyf[j]);
            C = 1. / (a.dy[j + 1] * a.dyf[j]);
            const double2 u2n = u2[(j + 1) * ps];
            G = ik(KX, u1[j * ps]) + (u2n - u2j) / a.dyf[j] + ik(KZ, u3[j * ps]);
            u2j = u2n;
        } else {
            A = 1.; B = -1.; C = 0.; G = zero;
        }
        (void)K2;
        const double Ap = (bprev != 0.0) ? -A / bprev : 0.0;
        B = B + Ap * cprev;
        G = G + Ap * gprev;
        bs[j * ps] = B;
        gs[j * ps] = G;
        bprev = B;
        cprev = C;
        gprev = G;
    }
    // back substitution, corrections and pressure update, descending
    double2 xn = zero;   // phi(j+1)
    for (int j = ny; j >= 1; --j) {
        const double B = bs[j * ps];
        const double2 G = gs[j * ps];
        double2 x;
        if (j == ny) x = (B != 0.0) ? G / B : zero;
        else {
            const double C = (j == 1) ? (zero_mode ? 0.0 : -1.0) : 1. / (a.dy[j + 1] * a.dyf[j]);
            x = (B != 0.0) ? (G - C * xn) / B : zero;
        }
        a.phi[col + j * ps] = x;
        u1[j * ps] = u1[j * ps] - ik(KX, x);
        u3[j * ps] = u3[j * ps] - ik(KZ, x);
        if (j + 1 <= ny) u2[(j + 1) * ps] = u2[(j + 1) * ps] - (xn - x) / a.dy[j + 1];
        if (a.update_cp && j + 1 <= ny) a.cp[col + (j + 1) * ps] = a.cp[col + (j + 1) * ps] + a.inv_h * xn;
        xn = x;
    }
}

cudaError_t launch_remdiv(const RemDivArgs& a, cudaStream_t st) {
    dim3 block(32, 4);
    dim3 grid((a.d.nkxp + 31) / 32, (a.d.nkzt + 3) / 4);
    k_remdiv<<<grid, block, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace dgpu
