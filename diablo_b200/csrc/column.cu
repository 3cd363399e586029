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

// Rows are set up in shared memory (one thread per field, in the order of
// the reference), eliminated there, then copied out by the whole block.
__global__ void __launch_bounds__(256) k_cn_coef(CoefParams c, double* mult, double* piv, double* cup,
                                                 double* bcv, signed char* kind) {
    extern __shared__ double sh[];
    const int ny = c.d.ny, nyp = c.d.nyp, nf = c.d.nf;
    double* sL = sh;
    double* sD = sL + nf * nyp;
    double* sU = sD + nf * nyp;
    double* sV = sU + nf * nyp;
    signed char* sK = reinterpret_cast<signed char*>(sV + nf * nyp);
    const double* DY = c.dy;
    const double* DYF = c.dyf;
    for (int e = threadIdx.x; e < nf * nyp; e += blockDim.x) {
        const int f = e / nyp, j = e % nyp;
        double l = 0.0, dd = 1.0, u = 0.0;
        signed char k = 1;
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
        sL[e] = l; sD[e] = dd; sU[e] = u; sV[e] = 0.0; sK[e] = k;
    }
    __syncthreads();
    const int f = threadIdx.x;
    if (f < nf) {
        double* L = sL + f * nyp;
        double* D = sD + f * nyp;
        double* U = sU + f * nyp;
        double* V = sV + f * nyp;
        signed char* K = sK + f * nyp;
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
        // THOMAS_FORWARD_REAL_MPI with NPROCY = 1: rows 1..NY+1 eliminated
        // (mpi.f:668-694); L becomes the multiplier, D the pivot.
        double dprev = D[0];
        for (int j = 1; j <= ny + 1; ++j) {
            const double m = -L[j] / dprev;
            L[j] = m;
            dprev = D[j] + m * U[j - 1];
            D[j] = dprev;
        }
        L[0] = 0.0;
    }
    __syncthreads();
    // pivots are stored as reciprocals; a zero pivot maps to 0, which gives
    // the x = 0 of the guarded back substitution (mpi.f:790-794)
    for (int e = threadIdx.x; e < nf * nyp; e += blockDim.x) {
        mult[e] = sL[e]; piv[e] = sD[e] != 0.0 ? 1.0 / sD[e] : 0.0; cup[e] = sU[e]; bcv[e] = sV[e];
        kind[e] = sK[e];
    }
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
    const size_t smem = (sizeof(double) * 4 + 1) * (size_t)d.nf * d.nyp;
    cudaFuncSetAttribute(k_cn_coef, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_cn_coef<<<1, 256, smem, st>>>(c, mult, piv, cup, bcv, kind);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// K5: REM_DIV_CHAN (channel.f:1103-1214) per column with the boundary rows
// of APPLY_BC_REM_DIV_MPI (mpi.f:1239-1278) and the guarded complex Thomas
// of mpi.f:700-865; then the velocity correction and the pressure update
// CP += phi/h (channel.f:1059-1065).
// ---------------------------------------------------------------------------
// Two lanes per column: the phi systems have real coefficients, so the real
// and the imaginary part are solved by neighbouring lanes; the products with
// i*k that mix the parts read the partner lane's value by a shuffle.
__device__ __forceinline__ double part_of(double2 v, int part) { return part ? v.y : v.x; }

__global__ void __launch_bounds__(128) k_remdiv(RemDivArgs a) {
    const Dims& d = a.d;
    const int part = threadIdx.x & 1;
    const int ncol = d.nkxp * d.nkzt;
    const int g = (blockIdx.x * 128 + threadIdx.x) >> 1;
    const bool active = g < ncol;
    const int gg = active ? g : ncol - 1;
    const int kx = gg % d.nkxp, m = gg / d.nkxp;
    const size_t ps = d.splane();
    const size_t fs = ps * d.nyp;
    const size_t col = (size_t)m * d.ldx + kx;
    const int ny = d.ny;
    const bool zero_mode = (kx == 0 && m == 0);
    const double KX = a.kx[kx], KZ = a.kz[m];
    const double sgn = part ? 1.0 : -1.0;   // (i K v) of part: re -> -K v.y, im -> +K v.x
    const double2* u1 = a.cu + col;
    const double2* u2 = a.cu + fs + col;
    const double2* u3 = a.cu + 2 * fs + col;
    double* pu1 = reinterpret_cast<double*>(a.cu + col) + part;
    double* pu2 = reinterpret_cast<double*>(a.cu + fs + col) + part;
    double* pu3 = reinterpret_cast<double*>(a.cu + 2 * fs + col) + part;
    double* pcp = reinterpret_cast<double*>(a.cp + col) + part;
    double* pphi = reinterpret_cast<double*>(a.phi + col) + part;
    double* bs = a.bsc + col;
    double* gs = reinterpret_cast<double*>(a.gsc + col) + part;
    // row 1 (BC rows of APPLY_BC_REM_DIV_MPI), then rows 2..NY
    double bprev = 1.0, cprev = zero_mode ? 0.0 : -1.0, gprev = 0.0;
    if (active) {
        if (part == 0) bs[ps] = bprev;
        gs[2 * ps] = gprev;
    }
    double2 u2j = active ? u2[2 * ps] : make_double2(0, 0);
    double2 u1n = active ? u1[2 * ps] : make_double2(0, 0);
    double2 u3n = active ? u3[2 * ps] : make_double2(0, 0);
    double2 u2n = active ? u2[3 * ps] : make_double2(0, 0);
    for (int j = 2; j <= ny; ++j) {
        const double2 u1j = u1n, u3j = u3n, u2p = u2n;
        if (active && j + 1 <= ny) {
            u1n = u1[(size_t)(j + 1) * ps];
            u3n = u3[(size_t)(j + 1) * ps];
            u2n = u2[(size_t)(j + 2) * ps];
        }
        double A, B, C, G;
        if (j < ny) {
            A = 1. / (a.dy[j] * a.dyf[j]);
            B = -KX * KX - KZ * KZ - 1. / (a.dy[j + 1] * a.dyf[j]) - 1. / (a.dy[j] * a.dyf[j]);
            C = 1. / (a.dy[j + 1] * a.dyf[j]);
            G = sgn * KX * part_of(u1j, part ^ 1) + (part_of(u2p, part) - part_of(u2j, part)) / a.dyf[j] +
                sgn * KZ * part_of(u3j, part ^ 1);
            u2j = u2p;
        } else {
            A = 1.; B = -1.; C = 0.; G = 0.;
        }
        const double Ap = (bprev != 0.0) ? -A / bprev : 0.0;
        B = B + Ap * cprev;
        G = G + Ap * gprev;
        if (active) {
            if (part == 0) bs[(size_t)j * ps] = B;
            gs[2 * (size_t)j * ps] = G;
        }
        bprev = B;
        cprev = C;
        gprev = G;
    }
    // back substitution, corrections and pressure update, descending
    double xn = 0.0;   // phi(j+1) of this part
    double bn = active ? bs[(size_t)ny * ps] : 1.0, gn = active ? gs[2 * (size_t)ny * ps] : 0.0;
    for (int j = ny; j >= 1; --j) {
        const double B = bn, G = gn;
        if (active && j - 1 >= 1) {
            bn = bs[(size_t)(j - 1) * ps];
            gn = gs[2 * (size_t)(j - 1) * ps];
        }
        double x;
        if (j == ny) x = (B != 0.0) ? G / B : 0.0;
        else {
            const double C = (j == 1) ? (zero_mode ? 0.0 : -1.0) : 1. / (a.dy[j + 1] * a.dyf[j]);
            x = (B != 0.0) ? (G - C * xn) / B : 0.0;
        }
        const double xo = __shfl_xor_sync(0xffffffffu, x, 1);   // the other part of phi(j)
        if (active) {
            pphi[2 * (size_t)j * ps] = x;
            // CU1 -= i KX phi, CU3 -= i KZ phi  (part re: +K phi.im, part im: -K phi.re)
            pu1[2 * (size_t)j * ps] -= sgn * KX * xo;
            pu3[2 * (size_t)j * ps] -= sgn * KZ * xo;
            if (j + 1 <= ny) {
                pu2[2 * (size_t)(j + 1) * ps] -= (xn - x) / a.dy[j + 1];
                if (a.update_cp) pcp[2 * (size_t)(j + 1) * ps] += a.inv_h * xn;
            }
        }
        xn = x;
    }
}

cudaError_t launch_remdiv(const RemDivArgs& a, cudaStream_t st) {
    const int ncol = a.d.nkxp * a.d.nkzt;
    k_remdiv<<<(2 * ncol + 127) / 128, 128, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace dgpu
