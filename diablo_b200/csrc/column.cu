// column.cu -- the standalone REM_DIV_CHAN projection (FP64), one pair of
// lanes per Fourier column (kx, kz): REM_DIV_CHAN called on its own and the
// projection that follows COURANT at a CFL substage.
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
