// poisson_stats.cu -- POISSON_P_CHAN (channel.f:1217-1453) and the plane
// statistics of SAVE_STATS_CHAN (save_stats.f:104-347, 452-536) on the
// device, in FP64.
//
// POISSON_P_CHAN forms RHS = sum_ij (du_i/dx_j)(du_j/dx_i) from nine
// gradient fields through physical space.  The reference transforms each of
// the five product groups forward separately and sums in Fourier space;
// the forward transform is linear, so here the products are summed in
// physical space and transformed once (equal to round-off, same 2/3
// truncation).  The buoyancy term and the tridiagonal solve with the
// APPLY_BC_POISSON_MPI rows (mpi.f:1280-1315) follow per Fourier column.
#include <cuda_runtime.h>

#include "kernels.cuh"
#include "launch.h"

namespace dgpu {

namespace {
__device__ __forceinline__ double2 ikd(double K, double2 a) { return make_double2(-K * a.y, K * a.x); }
}  // namespace

// One gradient field of POISSON_P_CHAN (rows J = 2..NY, zero elsewhere).
//  kind 0: ikx CU1            1: (CU2(j+1)-CU2(j))/DYF(j)   2: ikz CU3
//       3: (CU1(j+1)-CU1(j-1))/(2 DYF(j))   4: ikx (CU2(j)+CU2(j+1))/2
//       5: (CU3(j+1)-CU3(j-1))/(2 DYF(j))   6: ikz (CU2(j)+CU2(j+1))/2
//       7: ikz CU1            8: ikx CU3
__global__ void k_grad_field(Dims d, int kind, const double2* __restrict__ cu, double2* __restrict__ out,
                             const double* __restrict__ kx, const double* __restrict__ kz,
                             const double* __restrict__ dyf) {
    const size_t ps = d.splane();
    const size_t fs = ps * d.nyp;
    const size_t n = fs;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(e / ps);
        const size_t col = e % ps;
        const int m = (int)(col / d.ldx), i = (int)(col % d.ldx);
        double2 v = make_double2(0.0, 0.0);
        if (j >= 2 && j <= d.ny && m < d.nkzt && i < d.nkxp) {
            const double2* u1 = cu + col;
            const double2* u2 = cu + fs + col;
            const double2* u3 = cu + 2 * fs + col;
            const double KX = kx[i], KZ = kz[m];
            switch (kind) {
                case 0: v = ikd(KX, u1[j * ps]); break;
                case 1: { const double2 a = u2[(j + 1) * ps], b = u2[j * ps];
                          v = make_double2((a.x - b.x) / dyf[j], (a.y - b.y) / dyf[j]); } break;
                case 2: v = ikd(KZ, u3[j * ps]); break;
                case 3: { const double2 a = u1[(j + 1) * ps], b = u1[(j - 1) * ps];
                          v = make_double2((a.x - b.x) / (2. * dyf[j]), (a.y - b.y) / (2. * dyf[j])); } break;
                case 4: { const double2 a = u2[j * ps], b = u2[(j + 1) * ps];
                          v = ikd(KX * 0.5, make_double2(a.x + b.x, a.y + b.y)); } break;
                case 5: { const double2 a = u3[(j + 1) * ps], b = u3[(j - 1) * ps];
                          v = make_double2((a.x - b.x) / (2. * dyf[j]), (a.y - b.y) / (2. * dyf[j])); } break;
                case 6: { const double2 a = u2[j * ps], b = u2[(j + 1) * ps];
                          v = ikd(KZ * 0.5, make_double2(a.x + b.x, a.y + b.y)); } break;
                case 7: v = ikd(KZ, u1[j * ps]); break;
                default: v = ikd(KX, u3[j * ps]); break;
            }
        }
        out[e] = v;
    }
}

// acc (+)= alpha * a * b on physical planes 2..NY (P layout [J][z][x]).
__global__ void k_phys_fma(Dims d, double* __restrict__ acc, const double* __restrict__ a,
                           const double* __restrict__ b, double alpha, int init) {
    const size_t plane = (size_t)d.nz * d.nx;
    const size_t n0 = 2 * plane, n1 = (size_t)(d.ny + 1) * plane;
    for (size_t e = n0 + blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n1; e += (size_t)gridDim.x * blockDim.x) {
        const double v = alpha * a[e] * b[e];
        acc[e] = init ? v : acc[e] + v;
    }
}

// Per column: buoyancy term (non-(0,0) modes), rows of the Poisson system,
// guarded forward elimination over rows 2..NY and back substitution
// (mpi.f:700-865); CP(J) = solution, J = 1..NY.  Two lanes per column: lane
// 0 the real, lane 1 the imaginary part (the coefficients are real).
__global__ void __launch_bounds__(128) k_poisson_column(PoissonArgs a) {
    const Dims d = a.d;
    const int part = threadIdx.x & 1;
    const int ncol = d.nkxp * d.nkzt;
    const int g = (int)((blockIdx.x * 128 + threadIdx.x) >> 1);
    const bool active = g < ncol;
    const int gg = active ? g : ncol - 1;
    const int i = gg % d.nkxp, m = gg / d.nkxp;
    const size_t ps = d.splane(), fs = ps * d.nyp, col = (size_t)m * d.ldx + i;
    const int ny = d.ny;
    const bool zero_mode = (i == 0 && m == 0);
    const double KX = a.kx[i], KZ = a.kz[m];
    const double* pr = reinterpret_cast<const double*>(a.rhs + col) + part;
    double* pb = a.bsc + col;
    double* pg = reinterpret_cast<double*>(a.gsc + col) + part;
    // row 1 is the BC row; rows 2..NY-1 carry G = -RHS; row NY is a BC row
    double bprev = 1.0, cprev = zero_mode ? 0.0 : -1.0, gprev = 0.0;
    if (active) {
        pb[ps] = bprev;          // both lanes store the same pivot
        pg[2 * ps] = gprev;
    }
    for (int j = 2; j <= ny; ++j) {
        double A, B, C, G = 0.0;
        if (j < ny) {
            A = 1. / (a.dy[j] * a.dyf[j]);
            B = -KX * KX - KZ * KZ - 1. / (a.dy[j + 1] * a.dyf[j]) - 1. / (a.dy[j] * a.dyf[j]);
            C = 1. / (a.dy[j + 1] * a.dyf[j]);
            if (active) {
                double r = pr[2 * (size_t)j * ps];
                if (!zero_mode)
                    for (int n = 0; n < d.nth; ++n) {
                        const double* t = reinterpret_cast<const double*>(a.cth + (size_t)n * fs + col) + part;
                        r += a.ri[n] * (t[2 * (size_t)(j + 1) * ps] - t[2 * (size_t)(j - 1) * ps]) /
                             (a.gyf[j + 1] - a.gyf[j - 1]);
                    }
                G = -1. * r;
            }
        } else {
            A = 1.; B = -1.; C = 0.;
        }
        const double Ap = (bprev != 0.0) ? -A / bprev : 0.0;
        B = B + Ap * cprev;
        G = G + Ap * gprev;
        if (active) {
            pb[(size_t)j * ps] = B;
            pg[2 * (size_t)j * ps] = G;
        }
        bprev = B;
        cprev = C;
        gprev = G;
    }
    if (!active) return;
    double* pcp = reinterpret_cast<double*>(a.cp + col) + part;
    double xn = 0.0;
    for (int j = ny; j >= 1; --j) {
        const double B = pb[(size_t)j * ps], G = pg[2 * (size_t)j * ps];
        double x;
        if (j == ny) x = (B != 0.0) ? G / B : 0.0;
        else {
            const double C = (j == 1) ? (zero_mode ? 0.0 : -1.0) : 1. / (a.dy[j + 1] * a.dyf[j]);
            x = (B != 0.0) ? (G - C * xn) / B : 0.0;
        }
        pcp[2 * (size_t)j * ps] = x;
        xn = x;
    }
}

// FP64 plane sums for SAVE_STATS_CHAN: one block per plane j = 1..NY over
// physical U1, U2, U3 (and TH of scalar 1), with the mean profiles ume..thme.
// out[s*(NY+2)+j]: 0 urms^2 1 vrms^2 2 wrms^2 3 uv 4 uw 5 wv 6 shear 7 th^2 8 thv
// (sums over the plane; the host divides, takes square roots).
__global__ void __launch_bounds__(256) k_stats_planes(Dims d, const double* __restrict__ u1,
                                                      const double* __restrict__ u2, const double* __restrict__ u3,
                                                      const double* __restrict__ th, const double* __restrict__ me,
                                                      const double* __restrict__ dy, const double* __restrict__ dyf,
                                                      double* __restrict__ out) {
    __shared__ double red[9][256];
    const int j = 1 + blockIdx.x;
    const int nyp = d.nyp;
    const double* ume = me;
    const double* vme = me + nyp;
    const double* wme = me + 2 * nyp;
    const double* thme = me + 3 * nyp;
    const size_t plane = (size_t)d.nz * d.nx;
    double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (size_t e = threadIdx.x; e < plane; e += 256) {
        const size_t c = (size_t)j * plane + e, cm = c - plane, cpp = c + plane;
        const double a1 = u1[c] - ume[j], a2 = u2[c] - vme[j], a3 = u3[c] - wme[j];
        const double a2p = u2[cpp] - vme[j + 1];
        s[0] += a1 * a1;
        s[1] += 0.5 * (a2 * a2 + a2p * a2p);
        s[2] += a3 * a3;
        s[3] += (dyf[j - 1] * a1 + dyf[j] * (u1[cm] - ume[j - 1])) / (2.0 * dy[j]) * a2;
        s[4] += a1 * a3;
        s[5] += (dyf[j - 1] * a3 + dyf[j] * (u3[cm] - wme[j - 1])) / (2.0 * dy[j]) * a2;
        const double g1 = (u1[cpp] - u1[cm]) / (2.0 * dyf[j]), g3 = (u3[cpp] - u3[cm]) / (2.0 * dyf[j]);
        s[6] += g1 * g1 + g3 * g3;
        if (th) {
            const double t = th[c] - thme[j];
            s[7] += t * t;
            s[8] += t * (0.5 * (u2[c] + u2[cpp]) - 0.5 * (vme[j] + vme[j + 1]));
        }
    }
    for (int k = 0; k < 9; ++k) red[k][threadIdx.x] = s[k];
    __syncthreads();
    for (int st = 128; st > 0; st >>= 1) {
        if (threadIdx.x < st)
            for (int k = 0; k < 9; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x < 9) out[threadIdx.x * nyp + j] = red[threadIdx.x][0];
}

// One Fourier field of the remaining SAVE_STATS_CHAN profiles on rows
// J = 1..NY (zero on rows 0 and NY+1), from CU (after APPLY_BC_VEL) or from
// one scalar CS:
//  kind 0: omega_x = (CU3(j+1)-CU3(j-1))/(2 DYF(j)) - ikz (CU2(j+1)+CU2(j))/2
//       1: omega_y = ikz CU1 - ikx CU3                     (save_stats.f:270-322)
//       2: omega_z = ikx (CU2(j+1)+CU2(j))/2 - (CU1(j+1)-CU1(j-1))/(2 DYF(j))
//    3..5: ikx CU1, ikx CU2, ikx CU3   6..8: ikz CU1, ikz CU2, ikz CU3
//          (the gradients of tkebudget_chan, save_stats.f:957-1135)
//   9..11: ikx CS, (CS(j+1)-CS(j-1))/(GYF(j+1)-GYF(j-1)), ikz CS
//          (the scalar gradient of pe_diss, save_stats.f:465-474)
__global__ void k_stats_spec(Dims d, int kind, const double2* __restrict__ cu, const double2* __restrict__ cs,
                             double2* __restrict__ out, const double* __restrict__ kx, const double* __restrict__ kz,
                             const double* __restrict__ dyf, const double* __restrict__ gyf) {
    const size_t ps = d.splane();
    const size_t fs = ps * d.nyp;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < fs; e += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(e / ps);
        const size_t col = e % ps;
        const int m = (int)(col / d.ldx), i = (int)(col % d.ldx);
        double2 v = make_double2(0.0, 0.0);
        if (j >= 1 && j <= d.ny && m < d.nkzt && i < d.nkxp) {
            const double2* u1 = cu + col;
            const double2* u2 = cu + fs + col;
            const double2* u3 = cu + 2 * fs + col;
            const double KX = kx[i], KZ = kz[m];
            auto ddy = [&](const double2* f) {
                const double2 a = f[(j + 1) * ps], b = f[(j - 1) * ps];
                return make_double2((a.x - b.x) / (2. * dyf[j]), (a.y - b.y) / (2. * dyf[j]));
            };
            auto avg2 = [&]() {
                const double2 a = u2[(j + 1) * ps], b = u2[j * ps];
                return make_double2(0.5 * (a.x + b.x), 0.5 * (a.y + b.y));
            };
            switch (kind) {
                case 0: { const double2 a = ddy(u3), b = ikd(KZ, avg2());
                          v = make_double2(a.x - b.x, a.y - b.y); } break;
                case 1: { const double2 a = ikd(KZ, u1[j * ps]), b = ikd(KX, u3[j * ps]);
                          v = make_double2(a.x - b.x, a.y - b.y); } break;
                case 2: { const double2 a = ikd(KX, avg2()), b = ddy(u1);
                          v = make_double2(a.x - b.x, a.y - b.y); } break;
                case 3: v = ikd(KX, u1[j * ps]); break;
                case 4: v = ikd(KX, u2[j * ps]); break;
                case 5: v = ikd(KX, u3[j * ps]); break;
                case 6: v = ikd(KZ, u1[j * ps]); break;
                case 7: v = ikd(KZ, u2[j * ps]); break;
                case 8: v = ikd(KZ, u3[j * ps]); break;
                case 9: v = ikd(KX, cs[col + j * ps]); break;
                case 10: { const double2 a = cs[col + (j + 1) * ps], b = cs[col + (j - 1) * ps];
                           const double g = gyf[j + 1] - gyf[j - 1];
                           v = make_double2((a.x - b.x) / g, (a.y - b.y) / g); } break;
                default: v = ikd(KZ, cs[col + j * ps]); break;
            }
        }
        out[e] = v;
    }
}

// Plane sums of one term of the statistics over physical planes j = jlo..jhi
// (one block per plane, FP64): acc[j] = (init ? 0 : acc[j]) + sum_{x,z} term.
//  mode 0: f(j)^2
//       1: (DYF(j-1) f(j)^2 + DYF(j) f(j-1)^2) / (2 DY(j))   (GYF values at GY)
//       2: (((u(j)-m(j)) - (u(j-1)-m(j-1))) / DY(j))^2      (du/dy, dw/dy)
//       3: (((u(j+1)-m(j)) - (u(j-1)-m(j-1))) * rg(j))^2    (dv/dy, rg = 1/(GY(j+1)-GY(j-1)))
//       4: |f(j)-m(j)|^2                                    (thrms)
//       5: (f(j)-m(j)) ((u(j)+u(j+1))/2 - (m2(j)+m2(j+1))/2) (thv)
__global__ void __launch_bounds__(256) k_plane_terms(Dims d, int mode, const double* __restrict__ f,
                                                     const double* __restrict__ u, const double* __restrict__ m,
                                                     const double* __restrict__ m2, const double* __restrict__ dy,
                                                     const double* __restrict__ dyf, const double* __restrict__ rg,
                                                     int jlo, double* __restrict__ acc, int init) {
    __shared__ double red[256];
    const int j = jlo + blockIdx.x;
    const size_t plane = (size_t)d.nz * d.nx;
    const size_t c0 = (size_t)j * plane;
    double s = 0.0;
    for (size_t e = threadIdx.x; e < plane; e += 256) {
        const size_t c = c0 + e;
        double t;
        switch (mode) {
            case 0: t = f[c] * f[c]; break;
            case 1: { const double a = f[c], b = f[c - plane];
                      t = (dyf[j - 1] * a * a + dyf[j] * b * b) / (2.0 * dy[j]); } break;
            case 2: { const double g = ((u[c] - m[j]) - (u[c - plane] - m[j - 1])) / dy[j]; t = g * g; } break;
            case 3: { const double g = ((u[c + plane] - m[j]) - (u[c - plane] - m[j - 1])) * rg[j]; t = g * g; } break;
            case 4: { const double a = fabs(f[c] - m[j]); t = a * a; } break;
            default: t = (f[c] - m[j]) * (0.5 * (u[c] + u[c + plane]) - 0.5 * (m2[j] + m2[j + 1])); break;
        }
        s += t;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int st = 128; st > 0; st >>= 1) {
        if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0) acc[j] = (init ? 0.0 : acc[j]) + red[0];
}

cudaError_t launch_stats_spec(const Dims& d, int kind, const double2* cu, const double2* cs, double2* out,
                              const double* kx, const double* kz, const double* dyf, const double* gyf,
                              cudaStream_t st) {
    k_stats_spec<<<1184, 256, 0, st>>>(d, kind, cu, cs, out, kx, kz, dyf, gyf);
    return cudaGetLastError();
}

cudaError_t launch_plane_terms(const Dims& d, int mode, const double* f, const double* u, const double* m,
                               const double* m2, const double* dy, const double* dyf, const double* rg, int jlo,
                               int jhi, double* acc, int init, cudaStream_t st) {
    if (jhi < jlo) return cudaSuccess;
    k_plane_terms<<<jhi - jlo + 1, 256, 0, st>>>(d, mode, f, u, m, m2, dy, dyf, rg, jlo, acc, init);
    return cudaGetLastError();
}

cudaError_t launch_grad_field(const Dims& d, int kind, const double2* cu, double2* out, const double* kx,
                              const double* kz, const double* dyf, cudaStream_t st) {
    k_grad_field<<<1184, 256, 0, st>>>(d, kind, cu, out, kx, kz, dyf);
    return cudaGetLastError();
}

cudaError_t launch_phys_fma(const Dims& d, double* acc, const double* a, const double* b, double alpha, int init,
                            cudaStream_t st) {
    k_phys_fma<<<1184, 256, 0, st>>>(d, acc, a, b, alpha, init);
    return cudaGetLastError();
}

cudaError_t launch_poisson_column(const PoissonArgs& a, cudaStream_t st) {
    const int ncol = a.d.nkxp * a.d.nkzt;
    k_poisson_column<<<(2 * ncol + 127) / 128, 128, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_stats_planes(const Dims& d, const double* u1, const double* u2, const double* u3,
                                const double* th, const double* me, const double* dy, const double* dyf, double* out,
                                cudaStream_t st) {
    k_stats_planes<<<d.ny, 256, 0, st>>>(d, u1, u2, u3, th, me, dy, dyf, out);
    return cudaGetLastError();
}

}  // namespace dgpu
