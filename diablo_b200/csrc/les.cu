// les.cu -- the constant-Smagorinsky LES branch of RK_CHAN_1 on the device
// (for/les.f:1-267, 280-336; for/channel.f:303-384, 631-660, 748-760 and the
// eddy-viscosity rows of the CN matrices, channel.f:793-805, 862-874,
// 927-939, 991-1003).
//
// With an eddy viscosity that varies in x and z the CN systems differ from
// column to column in physical space, so this branch follows the reference's
// own order: right-hand sides in Fourier space, the subgrid model in physical
// space, the CN half-step and the tridiagonal solves per physical column
// (i,k), then the forward transforms and the projection.  The kernels here
// are the elementwise and column steps; the transforms are the FFT kernels of
// transforms.cu.  Everything is FP64.
//
// Layouts: spectral S[f][J][m][kx] (padded, see kernels.cuh); physical
// P[f][J][z][x] with pitch NX, pf = (NY+2)*NZ*NX doubles per field.
#include <cuda_runtime.h>

#include "../../include/diablo_gpu.h"
#include "kernels.cuh"
#include "launch.h"

namespace dgpu {
namespace {

__device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 operator*(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
__device__ __forceinline__ double2 operator/(double2 a, double s) { return make_double2(a.x / s, a.y / s); }
// i*K*a, the reference's CIKX(I)*A with CIKX = (0,KX)
__device__ __forceinline__ double2 ik(double K, double2 a) { return make_double2(-K * a.y, K * a.x); }

// Retained spectral entry of a flat index over (J, m, kx); false for padding.
__device__ __forceinline__ bool spec_index(const Dims& d, size_t g, int& J, int& m, int& kx) {
    const size_t ps = d.splane();
    if (g >= ps * (size_t)d.nyp) return false;
    J = (int)(g / ps);
    const size_t r = g % ps;
    m = (int)(r / d.ldx);
    kx = (int)(r % d.ldx);
    return kx < d.nkxp && m < d.nkzt;
}

constexpr int TB = 256;
inline unsigned blocks(size_t n) { return (unsigned)((n + TB - 1) / TB); }
inline size_t spec_items(const Dims& d) { return d.splane() * (size_t)d.nyp; }
__host__ __device__ inline size_t plane_pts(const Dims& d) { return (size_t)d.nz * d.nx; }

// ---------------------------------------------------------------------------
// Fourier-space right-hand sides before the subgrid model (channel.f:88-293):
// CR = CU + zeta h CF_old - h grad P (- h PX0 on the mean of CR1), and the new
// CF from the horizontal viscous, Coriolis, buoyancy and background-gradient
// terms, on the rows each field forms them.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(TB) k_les_pre(CnArgs a, const double* __restrict__ k2, double2* __restrict__ r) {
    const Dims& d = a.d;
    int J, m, kx;
    if (!spec_index(d, (size_t)blockIdx.x * TB + threadIdx.x, J, m, kx)) return;
    const size_t ps = d.splane(), fs = ps * d.nyp;
    const size_t o = (size_t)J * ps + (size_t)m * d.ldx + kx;
    const bool z0 = kx == 0 && m == 0;
    const double KX = a.kx[kx], KZ = a.kz[m], K2 = k2[(size_t)m * d.ldx + kx];
    for (int f = 0; f < d.nf; ++f) {
        if (J < a.cf_lo[f] || J > a.cf_hi[f]) continue;
        const double2 u = a.cu[(size_t)f * fs + o];
        double2 R = u;
        if (a.rk_step > 1) R = R + a.temp3 * a.cf[(size_t)f * fs + o];
        double2 CF;
        if (f < 3) {
            const double2 cp = a.cp[o];
            if (f == 0) R = R - a.temp4 * ik(KX, cp);
            else if (f == 2) R = R - a.temp4 * ik(KZ, cp);
            else R = R - a.temp4 * ((cp - a.cp[o - ps]) / a.dy[J]);
            if (f == 0 && z0) R.x -= a.forcing;
            CF = (-a.nu * K2) * u;
            if (f == 0) CF = CF + a.i_ro * a.cu[2 * fs + o];
            if (f == 2) CF = CF - a.i_ro * a.cu[o];
            for (int n = 0; n < d.nth; ++n) {
                const double2 th = a.cu[(size_t)(3 + n) * fs + o];
                if (f == 1) {
                    if (!z0) {
                        const double2 thm = a.cu[(size_t)(3 + n) * fs + o - ps];
                        CF = CF + ((a.ri[n] * a.grav_y) * (a.dyf[J - 1] * th + a.dyf[J] * thm)) / (2.0 * a.dy[J]);
                    }
                } else {
                    CF = CF + (a.ri[n] * (f == 0 ? a.grav_x : a.grav_z)) * th;
                }
            }
        } else {
            const int n = f - 3;
            CF = (-(a.nu / a.pr[n]) * K2) * u;
            CF = CF - a.drhodx[n] * a.cu[o] - a.drhodz[n] * a.cu[2 * fs + o];
        }
        r[(size_t)f * fs + o] = R;
        a.cf[(size_t)f * fs + o] = CF;
    }
}

// APPLY_BC_LES (les.f:805-865) on the state's CU1 / CU3, one thread per
// retained (kx,kz) column: Neumann walls copy the last interior row outward.
__global__ void __launch_bounds__(TB) k_les_bc(Dims d, double2* __restrict__ cu, int u_top, int w_top, int u_bot,
                                               int w_bot) {
    const size_t ps = d.splane(), g = (size_t)blockIdx.x * TB + threadIdx.x;
    if (g >= ps) return;
    const int kx = (int)(g % d.ldx), m = (int)(g / d.ldx);
    if (kx >= d.nkxp || m >= d.nkzt) return;
    const size_t fs = ps * d.nyp;
    const int ny = d.ny;
    double2* f1 = cu + g;
    double2* f3 = cu + 2 * fs + g;
    auto at = [&](double2* f, int j) -> double2& { return f[(size_t)j * ps]; };
    if (u_top == 1) { at(f1, ny) = at(f1, ny - 1); at(f1, ny + 1) = at(f1, ny); }
    if (w_top == 1) { at(f3, ny) = at(f3, ny - 1); at(f3, ny + 1) = at(f3, ny); }
    if (u_bot == 1) { at(f1, 1) = at(f1, 2); at(f1, 0) = at(f1, 1); }
    if (w_bot == 1) { at(f3, 1) = at(f3, 2); at(f3, 0) = at(f3, 1); }
}

// compute_strain_chan (les.f:526-569): S_11, S_22, S_33, S_13 on rows 1..NY
// and S_12, S_23 on rows 1..NY+1 into six spectral fields; other rows zero.
__global__ void __launch_bounds__(TB) k_les_strain(Dims d, const double2* __restrict__ cu, const double* __restrict__ kxw,
                                                   const double* __restrict__ kzw, const double* __restrict__ dy,
                                                   const double* __restrict__ dyf, double2* __restrict__ sij) {
    int J, m, kx;
    if (!spec_index(d, (size_t)blockIdx.x * TB + threadIdx.x, J, m, kx)) return;
    const size_t ps = d.splane(), fs = ps * d.nyp;
    const size_t o = (size_t)J * ps + (size_t)m * d.ldx + kx;
    const double KX = kxw[kx], KZ = kzw[m];
    const double2 zero = make_double2(0.0, 0.0);
    const double2* u1 = cu;
    const double2* u2 = cu + fs;
    const double2* u3 = cu + 2 * fs;
    double2 s1 = zero, s2 = zero, s3 = zero, s4 = zero, s5 = zero, s6 = zero;
    if (J >= 1 && J <= d.ny) {
        s1 = ik(KX, u1[o]);
        s2 = (u2[o + ps] - u2[o]) / dyf[J];
        s3 = ik(KZ, u3[o]);
        s5 = 0.5 * (ik(KZ, u1[o]) + ik(KX, u3[o]));
    }
    if (J >= 1) {
        s4 = 0.5 * ((u1[o] - u1[o - ps]) / dy[J] + ik(KX, u2[o]));
        s6 = 0.5 * (ik(KZ, u2[o]) + (u3[o] - u3[o - ps]) / dy[J]);
    }
    sij[o] = s1;
    sij[fs + o] = s2;
    sij[2 * fs + o] = s3;
    sij[3 * fs + o] = s4;
    sij[4 * fs + o] = s5;
    sij[5 * fs + o] = s6;
}

// The subgrid model at every physical point (les.f:113-227, 307-322):
// |S| at GYF and GY points with the mean shear removed, tau = |S| S_ij (the
// GY components without their implicit dU/dy part), NU_T = C_s^2 Delta^2 |S|
// with GHOST_LES's zero rows, and the cross-term integrands
// NU_T dU1/dy, NU_T dU3/dy.  sij: S_11, S_22, S_33, S_12, S_13, S_23
// (physical, rows 0..NY+1); out: tau_11, tau_33, tau_12, tau_13, tau_23, C1,
// C3.  The means are the (0,0) modes of the state's CU1 and CU3.
__global__ void __launch_bounds__(TB) k_les_sgs(Dims d, const double* __restrict__ sij, const double* __restrict__ u,
                                                const double2* __restrict__ cu, const double* __restrict__ dy,
                                                const double* __restrict__ dyf, const double* __restrict__ delta_y,
                                                double* __restrict__ out, double* __restrict__ nut) {
    const size_t pp = plane_pts(d), pf = pp * d.nyp;
    const size_t g = (size_t)blockIdx.x * TB + threadIdx.x;
    if (g >= pf) return;
    const int J = (int)(g / pp);
    const size_t col = g % pp;
    const int ny = d.ny;
    const size_t ps = d.splane(), fs = ps * d.nyp;
    auto S = [&](int q, int j) { return sij[(size_t)q * pf + (size_t)j * pp + col]; };
    auto U = [&](int c, int j) { return u[(size_t)c * pf + (size_t)j * pp + col]; };
    auto ub = [&](int c, int j) { return cu[(size_t)c * fs + (size_t)j * ps].x; };
    double t11 = S(0, J), t33 = S(2, J), t13 = S(4, J), t12 = S(3, J), t23 = S(5, J);
    if (J >= 2 && J <= ny) {
        const double a4 = 0.5 * (S(3, J + 1) + S(3, J) - 0.5 * (ub(0, J) - ub(0, J - 1)) / dy[J] -
                                 0.5 * (ub(0, J + 1) - ub(0, J)) / dy[J + 1]);
        const double a6 = 0.5 * (S(5, J + 1) + S(5, J) - 0.5 * (ub(2, J) - ub(2, J - 1)) / dy[J] -
                                 0.5 * (ub(2, J + 1) - ub(2, J)) / dy[J + 1]);
        const double s1 = S(0, J), s2 = S(1, J), s3 = S(2, J), s5 = S(4, J);
        const double sm = sqrt(2.0 * (s1 * s1) + 4.0 * (a4 * a4) + 4.0 * (s5 * s5) + 2.0 * (s2 * s2) +
                               4.0 * (a6 * a6) + 2.0 * (s3 * s3));
        t11 = sm * s1;
        t13 = sm * s5;
        t33 = sm * s3;
    }
    double sg = 0.0;
    if (J >= 2) {
        const double w0 = dyf[J - 1], w1 = dyf[J], h2 = 2.0 * dy[J];
        const double g1 = (S(0, J) * w0 + S(0, J - 1) * w1) / h2;
        const double g5 = (S(4, J) * w0 + S(4, J - 1) * w1) / h2;
        const double g2 = (S(1, J) * w0 + S(1, J - 1) * w1) / h2;
        const double g3 = (S(2, J) * w0 + S(2, J - 1) * w1) / h2;
        const double b4 = S(3, J) - 0.5 * (ub(0, J) - ub(0, J - 1)) / dy[J];
        const double b6 = S(5, J) - 0.5 * (ub(2, J) - ub(2, J - 1)) / dy[J];
        sg = sqrt(2.0 * (g1 * g1) + 4.0 * (b4 * b4) + 4.0 * (g5 * g5) + 2.0 * (g2 * g2) + 4.0 * (b6 * b6) +
                  2.0 * (g3 * g3));
        t12 = sg * (S(3, J) - 0.5 * (U(0, J) - U(0, J - 1)) / dy[J]);
        t23 = sg * (S(5, J) - 0.5 * (U(2, J) - U(2, J - 1)) / dy[J]);
    }
    const double nt = (J >= 3 && J <= ny - 1) ? -0.5 * delta_y[J] * sg : 0.0;
    double c1 = 0.0, c3 = 0.0;
    if (J >= 2 && J <= ny) {
        c1 = nt * (U(0, J) - U(0, J - 1)) / dy[J];
        c3 = nt * (U(2, J) - U(2, J - 1)) / dy[J];
    }
    out[g] = t11;
    out[pf + g] = t33;
    out[2 * pf + g] = t12;
    out[3 * pf + g] = t13;
    out[4 * pf + g] = t23;
    out[5 * pf + g] = c1;
    out[6 * pf + g] = c3;
    nut[g] = nt;
}

// APPLY_BC_VEL_PHYS_LOWER / _UPPER (channel.f:2495-2660) on physical U1..U3,
// one thread per (x,z) column.
__global__ void __launch_bounds__(TB) k_phys_bc_vel(Dims d, double* __restrict__ u, const double* __restrict__ dy,
                                                    const double* __restrict__ dyf, diablo_params p) {
    const size_t pp = plane_pts(d), pf = pp * d.nyp;
    const size_t g = (size_t)blockIdx.x * TB + threadIdx.x;
    if (g >= pp) return;
    const int ny = d.ny;
    double* u1 = u + g;
    double* u2 = u + pf + g;
    double* u3 = u + 2 * pf + g;
    auto at = [&](double* f, int j) -> double& { return f[(size_t)j * pp]; };
    if (p.u_bc_ymin == 0) { at(u1, 0) = p.u_bc_ymin_c1; at(u1, 1) = p.u_bc_ymin_c1; }
    else { at(u1, 1) = at(u1, 2) - dy[2] * p.u_bc_ymin_c1; at(u1, 0) = at(u1, 1) - dy[1] * p.u_bc_ymin_c1; }
    if (p.w_bc_ymin == 0) { at(u3, 0) = p.w_bc_ymin_c1; at(u3, 1) = p.w_bc_ymin_c1; }
    else { at(u3, 1) = at(u3, 2) - dy[2] * p.w_bc_ymin_c1; at(u3, 0) = at(u3, 1) - dy[1] * p.w_bc_ymin_c1; }
    if (p.v_bc_ymin == 0) { at(u2, 1) = 2.0 * p.v_bc_ymin_c1 - at(u2, 2); at(u2, 0) = at(u2, 1); }
    else { at(u2, 1) = at(u2, 2) - dyf[1] * p.v_bc_ymin_c1; at(u2, 0) = at(u2, 1) - dyf[1] * p.v_bc_ymin_c1; }
    if (p.u_bc_ymax == 0) { at(u1, ny) = p.u_bc_ymax_c1; at(u1, ny + 1) = p.u_bc_ymax_c1; }
    else { at(u1, ny) = at(u1, ny - 1) + dy[ny] * p.u_bc_ymax_c1; at(u1, ny + 1) = at(u1, ny) + dy[ny] * p.u_bc_ymax_c1; }
    if (p.w_bc_ymax == 0) { at(u3, ny) = p.w_bc_ymax_c1; at(u3, ny + 1) = p.w_bc_ymax_c1; }
    else { at(u3, ny) = at(u3, ny - 1) + dy[ny] * p.w_bc_ymax_c1; at(u3, ny + 1) = at(u3, ny) + dy[ny] * p.w_bc_ymax_c1; }
    if (p.v_bc_ymax == 0) at(u2, ny + 1) = 2.0 * p.v_bc_ymax_c1 - at(u2, ny);
    else at(u2, ny + 1) = at(u2, ny) + dy[ny] * p.v_bc_ymax_c1;
}

// CF_i -= d tau_ij / dx_j (les.f:235-304) and the cross terms (les.f:307-336).
// tau: the seven forward-transformed fields of k_les_sgs; the filter widths
// Delta_YF (GYF) and Delta_Y (GY) scale them on the reference's rows.
__global__ void __launch_bounds__(TB) k_les_tau_cf(Dims d, const double2* __restrict__ tau, double2* __restrict__ cf,
                                                   const double* __restrict__ kxw, const double* __restrict__ kzw,
                                                   const double* __restrict__ dyf, const double* __restrict__ delta_yf,
                                                   const double* __restrict__ delta_y) {
    int J, m, kx;
    if (!spec_index(d, (size_t)blockIdx.x * TB + threadIdx.x, J, m, kx)) return;
    const int ny = d.ny;
    if (J < 2 || J > ny) return;
    const size_t ps = d.splane(), fs = ps * d.nyp;
    const size_t o = (size_t)J * ps + (size_t)m * d.ldx + kx;
    const double KX = kxw[kx], KZ = kzw[m];
    auto T = [&](int q, int j) { return tau[(size_t)q * fs + o + (size_t)(j - J) * ps]; };
    if (J <= ny - 1) {   // J1 = JSTART, J2 = NY-1 with NPROCY = 1 (les.f:46-59)
        const double2 c11 = delta_yf[J] * T(0, J), c33 = delta_yf[J] * T(1, J), c13 = delta_yf[J] * T(3, J);
        const double2 c12 = delta_y[J] * T(2, J), c12p = delta_y[J + 1] * T(2, J + 1);
        const double2 c23 = delta_y[J] * T(4, J), c23p = delta_y[J + 1] * T(4, J + 1);
        double2* f1 = cf + o;
        double2* f3 = cf + 2 * fs + o;
        *f1 = *f1 - ik(KX, c11) - (c12p - c12) / dyf[J] - ik(KZ, c13);
        *f3 = *f3 - ik(KX, c13) - (c23p - c23) / dyf[J] - ik(KZ, c33);
    }
    double2* f2 = cf + fs + o;
    double2 v = *f2 - ik(KX, delta_y[J] * T(2, J)) - ik(KZ, delta_y[J] * T(4, J));
    v = v + ik(KX, T(5, J));
    v = v + ik(KZ, T(6, J));
    *f2 = v;
}

// i k_x CTH and i k_z CTH of one scalar on rows 1..NY+1 (channel.f:328-357).
__global__ void __launch_bounds__(TB) k_les_kgrad(Dims d, const double2* __restrict__ cth, const double* __restrict__ kxw,
                                                  const double* __restrict__ kzw, double2* __restrict__ out) {
    int J, m, kx;
    if (!spec_index(d, (size_t)blockIdx.x * TB + threadIdx.x, J, m, kx)) return;
    const size_t ps = d.splane(), fs = ps * d.nyp;
    const size_t o = (size_t)J * ps + (size_t)m * d.ldx + kx;
    const double2 zero = make_double2(0.0, 0.0);
    const double2 t = cth[o];
    out[o] = J >= 1 ? ik(kxw[kx], t) : zero;
    out[fs + o] = J >= 1 ? ik(kzw[m], t) : zero;
}

// KAPPA_T * (two physical fields) on rows 1..NY+1 (channel.f:336-342, 360-366).
__global__ void __launch_bounds__(TB) k_les_kmul(Dims d, double* __restrict__ a, const double* __restrict__ nut) {
    const size_t pp = plane_pts(d), pf = pp * d.nyp;
    const size_t g = (size_t)blockIdx.x * TB + threadIdx.x;
    if (g >= pf || g < pp) return;
    a[g] = nut[g] * a[g];
    a[pf + g] = nut[g] * a[pf + g];
}

// CFTH += i k_x (KAPPA_T dTH/dx)^ + i k_z (KAPPA_T dTH/dz)^ on the scalar's
// rows (channel.f:344-350, 368-374).
__global__ void __launch_bounds__(TB) k_les_kcf(Dims d, const double2* __restrict__ g2, double2* __restrict__ cfth,
                                                const double* __restrict__ kxw, const double* __restrict__ kzw, int j0,
                                                int j1) {
    int J, m, kx;
    if (!spec_index(d, (size_t)blockIdx.x * TB + threadIdx.x, J, m, kx)) return;
    if (J < j0 || J > j1) return;
    const size_t ps = d.splane(), fs = ps * d.nyp;
    const size_t o = (size_t)J * ps + (size_t)m * d.ldx + kx;
    const double2 v = cfth[o] + ik(kxw[kx], g2[o]);
    cfth[o] = v + ik(kzw[m], g2[fs + o]);
}

// CF += the nonlinear terms; CR += beta h CF (channel.f:581-595, 708-711).
__global__ void __launch_bounds__(TB) k_les_post(CnArgs a, const double2* __restrict__ nl, double2* __restrict__ r) {
    const Dims& d = a.d;
    int J, m, kx;
    if (!spec_index(d, (size_t)blockIdx.x * TB + threadIdx.x, J, m, kx)) return;
    const size_t ps = d.splane(), fs = ps * d.nyp;
    const size_t o = (size_t)J * ps + (size_t)m * d.ldx + kx;
    for (int f = 0; f < d.nf; ++f) {
        if (J < a.cf_lo[f] || J > a.cf_hi[f]) continue;
        const size_t q = (size_t)f * fs + o;
        const double2 cf = a.cf[q] + nl[q];
        a.cf[q] = cf;
        r[q] = r[q] + a.temp5 * cf;
    }
}

// The explicit half of CN in y and the eddy-viscosity terms, in physical
// space (channel.f:606-660, 737-760): R_f += TEMP1 (nu_v) d2/dy2 f +
// TEMP2 d/dy(NU_T df/dy).  u holds the physical fields, r the physical RHS.
__global__ void __launch_bounds__(TB) k_les_explicit(LesArgs a, const double* __restrict__ u, double* __restrict__ r,
                                                     const double* __restrict__ nut) {
    const Dims& d = a.d;
    const size_t pp = plane_pts(d), pf = pp * d.nyp;
    const size_t g = (size_t)blockIdx.x * TB + threadIdx.x;
    if (g >= pf) return;
    const int J = (int)(g / pp);
    const double* dy = a.dy;
    const double* dyf = a.dyf;
    for (int f = 0; f < d.nf; ++f) {
        if (J < a.j_lo[f] || J > a.j_hi[f]) continue;   // j_lo >= 1, j_hi <= NY
        const double* F = u + (size_t)f * pf + g;
        const double fm = F[-(ptrdiff_t)pp], f0 = F[0], fp = F[pp];
        const double nm = nut[g - pp], n0 = nut[g], np = nut[g + pp];
        double v = r[(size_t)f * pf + g];
        if (f == 1) {
            v = v + a.temp1 * a.nu_v_scale * (((fp - f0) / dyf[J] - (f0 - fm) / dyf[J - 1]) / dy[J]);
            v = v + a.temp2 * ((0.5 * (n0 + np) * (fp - f0) / dyf[J] - 0.5 * (n0 + nm) * (f0 - fm) / dyf[J - 1]) / dy[J]);
        } else {
            const double c = f < 3 ? a.temp1 * a.nu_v_scale : (a.temp1 / a.pr[f - 3]) * a.nu_v_scale;
            v = v + c * (((fp - f0) / dy[J + 1] - (f0 - fm) / dy[J]) / dyf[J]);
            v = v + a.temp2 * ((np * (fp - f0) / dy[J + 1] - n0 * (f0 - fm) / dy[J]) / dyf[J]);
        }
        r[(size_t)f * pf + g] = v;
    }
}

// One row of a CN system in physical space: the interior row with the
// eddy-viscosity terms (channel.f:786-805, 851-874, 916-939, 980-1003), then
// the BC rows of APPLY_BC_TH_*, APPLY_BC_2_*, APPLY_BC_1_* / _3_*
// (channel.f:1660-2202) written over it, in the reference's order.  Rows
// outside the system are the identity with a zero right-hand side.  The
// grid metrics come from the reciprocal row tables (RT_E*), so a row costs
// no division.
__device__ __forceinline__ void les_row(const LesArgs& a, int f, int j, double n0, double np, double nm, double rv,
                                        double& L, double& D, double& U, double& V) {
    const int ny = a.d.ny;
    const int nyp = a.d.nyp;
    L = 0.0; D = 1.0; U = 0.0; V = 0.0;
    if (j >= a.j_lo[f] && j <= a.j_hi[f]) {
        const double t2 = a.temp2;
        if (f == 1) {
            const double em = a.rows[RT_E2M * nyp + j], ep = a.rows[RT_E2P * nyp + j];
            const double c = a.temp1 * a.nu_v_scale;
            const double sm = t2 * 0.5 * (n0 + nm), sp = t2 * 0.5 * (n0 + np);
            L = -c * em - sm * em;
            D = 1. + c * ep + c * em + sp * ep + sm * em;
            U = -c * ep - sp * ep;
        } else {
            const double em = a.rows[RT_E1M * nyp + j], ep = a.rows[RT_E1P * nyp + j];
            const double c = f < 3 ? a.temp1 * a.nu_v_scale : a.temp1 / a.pr[f - 3] * a.nu_v_scale;
            L = -c * em - t2 * n0 * em;
            D = 1. + c * ep + c * em + t2 * np * ep + t2 * n0 * em;
            U = -c * ep - t2 * np * ep;
        }
        V = rv;
    }
    auto set = [&](double l, double dd, double u, double v) { L = l; D = dd; U = u; V = v; };
    const int bmin = a.bc_type[f][0], bmax = a.bc_type[f][1];
    const double cmin = a.bc_c1[f][0], cmax = a.bc_c1[f][1];
    if (f == 1) {   // APPLY_BC_2_LOWER / _UPPER
        if (bmin == 0) {
            if (j == 1 || j == 2) set(0.0, 1.0, 0.0, cmin);
        } else if (j == 1) {
            set(0.0, -1.0, 1.0, a.dyf[1] * cmin);
        }
        if (j == 0) set(0.0, 1.0, 0.0, 0.0);
        if (bmax == 0) {
            if (j == ny + 1 || j == ny) set(0.0, 1.0, 0.0, cmax);
        } else if (j == ny + 1) {
            set(-1.0, 1.0, 0.0, a.dyf[ny] * cmax);
        }
    } else {        // U1, U3 and the scalars share the GYF-point rows
        if (j == 0) set(0.0, 1.0, 0.0, 0.0);
        if (j == 1) {
            if (bmin == 0) set(0.0, 1.0, 0.0, cmin);
            else set(0.0, -1.0, 1.0, a.dy[2] * cmin);
        }
        if (j == ny + 1) set(0.0, 1.0, 0.0, 0.0);
        if (j == ny) {
            if (bmax == 0) set(0.0, 1.0, 0.0, cmax);
            else set(-1.0, 1.0, 0.0, a.dy[ny] * cmax);
        }
    }
}

// THOMAS_FORWARD/BACKWARD_REAL_MPI (mpi.f:630-697, 757-809) with NPROCY = 1,
// one thread per physical (x,z) column and field (blockIdx.y): forward
// elimination over rows 1..NY+1, the eliminated right-hand side written over
// the right-hand side r and the pivots kept in piv; back substitution from
// NY+1 down to 0 (zero where a pivot is zero), the result written on the
// rows the reference copies back.
__global__ void __launch_bounds__(TB) k_les_solve(LesArgs a, double* __restrict__ r, const double* __restrict__ nut,
                                                  double* __restrict__ piv, double* __restrict__ out) {
    const Dims& d = a.d;
    const size_t pp = plane_pts(d), pf = pp * d.nyp;
    const size_t g = (size_t)blockIdx.x * TB + threadIdx.x;
    const int f = blockIdx.y;
    if (g >= pp) return;
    const int ny = d.ny;
    r += (size_t)f * pf;
    piv += (size_t)f * pf;
    out += (size_t)f * pf;
    double L, D, U, V;
    double nm = 0.0, n0 = nut[g], np = nut[pp + g];
    les_row(a, f, 0, n0, np, nm, r[g], L, D, U, V);
    double Bp = D, Gp = V, Up = U;
    piv[g] = Bp;
    r[g] = Gp;
    for (int j = 1; j <= ny + 1; ++j) {
        const size_t q = (size_t)j * pp + g;
        nm = n0;
        n0 = np;
        np = j + 1 <= ny + 1 ? nut[q + pp] : 0.0;
        les_row(a, f, j, n0, np, nm, r[q], L, D, U, V);
        const double A = -L / Bp;
        Bp = D + A * Up;
        Gp = V + A * Gp;
        Up = U;
        piv[q] = Bp;
        r[q] = Gp;
    }
    double x = Gp / Bp;
    if (ny + 1 >= a.out_lo[f]) out[(size_t)(ny + 1) * pp + g] = x;
    np = 0.0;
    n0 = nut[(size_t)(ny + 1) * pp + g];
    nm = nut[(size_t)ny * pp + g];
    for (int j = ny; j >= 0; --j) {
        const size_t q = (size_t)j * pp + g;
        np = n0;
        n0 = nm;
        nm = j >= 1 ? nut[q - pp] : 0.0;
        les_row(a, f, j, n0, np, nm, 0.0, L, D, U, V);
        const double b = piv[q];
        x = b != 0.0 ? (r[q] - U * x) / b : 0.0;
        if (j >= a.out_lo[f]) out[q] = x;
    }
}

// ---------------------------------------------------------------------------
// Dynamic Smagorinsky (LES_MODEL_TYPE 2).  The reference stops for this model
// type (les.f:269-272); the model is this library's: Germano's identity with
// Lilly's least squares over each x-z plane at GYF points J = 2..NY,
//   L_ij = (u_i u_j)^ - u^_i u^_j,  M_ij = R |S^| S^_ij - (|S| S_ij)^,
//   (C Delta^2)(J) = max(0, -<L_ij M_ij> / (2 <M_ij M_ij>)),
// ^ the 5-point test filter of les_filter_chan (les.f:572-712) in x then z,
// R = (Delta^/Delta)^2, |S| and |S^| with the mean shear removed.
//
// k_dyn_sums: one block per (32 x-points, 8 z-points, plane).  The ten base
// values of the 36 x 12 points the stencils reach (periodic) are computed
// into shared memory; the x-filtered 21 quantities of the 32 x 12 points
// follow; each thread z-filters its point, forms L_ij M_ij and M_ij M_ij,
// and the block's sums are added to the plane's.
// ---------------------------------------------------------------------------
constexpr int DX_T = 32, DZ_T = 8, DX_S = DX_T + 4, DZ_S = DZ_T + 4, NB = 10, NQ = 21;

__global__ void __launch_bounds__(256) k_dyn_sums(Dims d, const double* __restrict__ sij, const double* __restrict__ u,
                                                  const double2* __restrict__ cu, const double* __restrict__ dy,
                                                  double R, double* __restrict__ sums) {
    extern __shared__ __align__(16) unsigned char smem[];
    double* sb = reinterpret_cast<double*>(smem);   // [NB][DZ_S][DX_S]
    double* sx = sb + NB * DZ_S * DX_S;              // [NQ][DZ_S][DX_T]
    __shared__ double red[2][8];
    const int nx = d.nx, nz = d.nz;
    const int i0 = blockIdx.x * DX_T, k0 = blockIdx.y * DZ_T, J = 2 + blockIdx.z;
    const size_t pp = plane_pts(d), pf = pp * d.nyp;
    const size_t ps = d.splane(), fs = ps * d.nyp;
    auto ub = [&](int c, int j) { return cu[(size_t)c * fs + (size_t)j * ps].x; };
    const double dm1 = 0.5 * (ub(0, J) - ub(0, J - 1)) / dy[J], dp1 = 0.5 * (ub(0, J + 1) - ub(0, J)) / dy[J + 1];
    const double dm3 = 0.5 * (ub(2, J) - ub(2, J - 1)) / dy[J], dp3 = 0.5 * (ub(2, J + 1) - ub(2, J)) / dy[J + 1];
    const double m1 = dm1 + dp1, m3 = dm3 + dp3;
    for (int e = threadIdx.x; e < DZ_S * DX_S; e += 256) {
        const int kk = e / DX_S, ii = e % DX_S;
        const int i = (i0 - 2 + ii + nx) % nx, k = (k0 - 2 + kk + nz) % nz;
        const size_t c = (size_t)k * nx + i;
        auto S = [&](int q, int j) { return sij[(size_t)q * pf + (size_t)j * pp + c]; };
        auto U = [&](int q, int j) { return u[(size_t)q * pf + (size_t)j * pp + c]; };
        const double s11 = S(0, J), s22 = S(1, J), s33 = S(2, J), s13 = S(4, J);
        const double a4 = 0.5 * (S(3, J + 1) + S(3, J) - dm1 - dp1);
        const double a6 = 0.5 * (S(5, J + 1) + S(5, J) - dm3 - dp3);
        const double sm = sqrt(2.0 * (s11 * s11) + 4.0 * (a4 * a4) + 4.0 * (s13 * s13) + 2.0 * (s22 * s22) +
                               4.0 * (a6 * a6) + 2.0 * (s33 * s33));
        const double v[NB] = {U(0, J), 0.5 * (U(1, J) + U(1, J + 1)), U(2, J), s11, s22, s33,
                              0.5 * (S(3, J) + S(3, J + 1)), s13, 0.5 * (S(5, J) + S(5, J + 1)), sm};
#pragma unroll
        for (int q = 0; q < NB; ++q) sb[(q * DZ_S + kk) * DX_S + ii] = v[q];
    }
    __syncthreads();
    // the 21 quantities of each point, filtered in x (les.f:656-662 order)
    const double W[5] = {1.0 / 8.0, 1.0 / 4.0, 1.0 / 4.0, 1.0 / 4.0, 1.0 / 8.0};
    for (int e = threadIdx.x; e < DZ_S * DX_T; e += 256) {
        const int kk = e / DX_T, tx = e % DX_T;
        double acc[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) acc[q] = 0.0;
#pragma unroll
        for (int t = 0; t < 5; ++t) {
            const int ii = tx + t;
            double b[NB];
#pragma unroll
            for (int q = 0; q < NB; ++q) b[q] = sb[(q * DZ_S + kk) * DX_S + ii];
            const double v[NQ] = {b[0], b[1], b[2], b[0] * b[0], b[1] * b[1], b[2] * b[2], b[0] * b[1], b[0] * b[2],
                                  b[1] * b[2], b[3], b[4], b[5], b[6], b[7], b[8],
                                  b[9] * b[3], b[9] * b[4], b[9] * b[5], b[9] * b[6], b[9] * b[7], b[9] * b[8]};
#pragma unroll
            for (int q = 0; q < NQ; ++q) acc[q] = t == 0 ? W[0] * v[q] : acc[q] + W[t] * v[q];
        }
#pragma unroll
        for (int q = 0; q < NQ; ++q) sx[(q * DZ_S + kk) * DX_T + tx] = acc[q];
    }
    __syncthreads();
    const int tx = threadIdx.x % DX_T, tz = threadIdx.x / DX_T;
    double num = 0.0, den = 0.0;
    if (i0 + tx < nx && k0 + tz < nz) {
        double h[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            double a = W[0] * sx[(q * DZ_S + tz) * DX_T + tx];
#pragma unroll
            for (int t = 1; t < 5; ++t) a = a + W[t] * sx[(q * DZ_S + tz + t) * DX_T + tx];
            h[q] = a;
        }
        const double a12 = h[12] - 0.5 * m1, a23 = h[14] - 0.5 * m3;
        const double sh = sqrt(2.0 * (h[9] * h[9]) + 4.0 * (a12 * a12) + 4.0 * (h[13] * h[13]) + 2.0 * (h[10] * h[10]) +
                               4.0 * (a23 * a23) + 2.0 * (h[11] * h[11]));
        const double L11 = h[3] - h[0] * h[0], L22 = h[4] - h[1] * h[1], L33 = h[5] - h[2] * h[2];
        const double L12 = h[6] - h[0] * h[1], L13 = h[7] - h[0] * h[2], L23 = h[8] - h[1] * h[2];
        const double M11 = R * sh * h[9] - h[15], M22 = R * sh * h[10] - h[16], M33 = R * sh * h[11] - h[17];
        const double M12 = R * sh * h[12] - h[18], M13 = R * sh * h[13] - h[19], M23 = R * sh * h[14] - h[20];
        num = L11 * M11 + L22 * M22 + L33 * M33 + 2.0 * (L12 * M12 + L13 * M13 + L23 * M23);
        den = M11 * M11 + M22 * M22 + M33 * M33 + 2.0 * (M12 * M12 + M13 * M13 + M23 * M23);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        num += __shfl_down_sync(0xffffffffu, num, o);
        den += __shfl_down_sync(0xffffffffu, den, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { red[0][w] = num; red[1][w] = den; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int q = 0; q < 8; ++q) { a += red[0][q]; b += red[1][q]; }
        atomicAdd(sums + 2 * J, a);
        atomicAdd(sums + 2 * J + 1, b);
    }
}

// (C Delta^2)(J) from the plane sums, then the widths that replace the
// constant model's: Delta_YF = -2 C Delta^2 at GYF points, Delta_Y its
// interpolation to GY points (the end planes take the nearest value).
__global__ void k_dyn_widths(Dims d, const double* __restrict__ sums, const double* __restrict__ dy,
                             const double* __restrict__ dyf, double* __restrict__ widths) {
    const int ny = d.ny, nyp = d.nyp;
    auto cd = [&](int j) {
        j = j < 2 ? 2 : j > ny ? ny : j;
        const double num = sums[2 * j], den = sums[2 * j + 1];
        const double c = den > 0.0 ? -0.5 * num / den : 0.0;
        return c > 0.0 ? c : 0.0;
    };
    for (int j = threadIdx.x; j < nyp; j += blockDim.x) {
        widths[j] = j >= 1 ? -2.0 * cd(j) : 0.0;
        double cg = 0.0;
        if (j >= 3 && j <= ny) cg = (cd(j) * dyf[j - 1] + cd(j - 1) * dyf[j]) / (2.0 * dy[j]);
        else if (j == 2 || j == ny + 1) cg = cd(j);
        widths[nyp + j] = j >= 2 ? -2.0 * cg : 0.0;
    }
}

// ---------------------------------------------------------------------------
// Samples for the learned closure: from physical U1..U3, at GYF points
// J = 2..NY-1 and every `stride`-th x and z point, the features and targets
// of a w x w top-hat filter in x and z (periodic; w odd), one thread per
// sample.  U2 is averaged to GYF before filtering.  The gradients
// g_ij = d(ubar_i)/dx_j (i-major; centred differences over one cell in x and
// z, over GYF(J+-1) in y) enter in dimensionless form: features g_ij / G
// with G = |g|, then y+ = (distance to the nearer of GYF(1), GYF(NY)) / NU
// and Delta = (w DX DYF(J) w DZ)^(1/3); the stress scale is s = Delta^2 G^2.
// Targets (when t is given): tau_ij / s, tau_ij = bar(u_i u_j) - ubar_i
// ubar_j in the order 11, 22, 33, 12, 13, 23 (zero where s = 0).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(TB) k_sgs_samples(Dims d, const double* __restrict__ u, const double* __restrict__ gyf,
                                                    const double* __restrict__ dyf, double dx, double dz, double nu,
                                                    int w, int stride, float* __restrict__ x, float* __restrict__ t,
                                                    float* __restrict__ sc) {
    const int nx = d.nx, nz = d.nz, ny = d.ny;
    const int nxs = (nx + stride - 1) / stride, nzs = (nz + stride - 1) / stride;
    const long long ns = (long long)(ny - 2) * nzs * nxs;
    const long long s = (long long)blockIdx.x * TB + threadIdx.x;
    if (s >= ns) return;
    const int ii = (int)(s % nxs), kk = (int)((s / nxs) % nzs), J = 2 + (int)(s / ((long long)nxs * nzs));
    const int i = ii * stride, k = kk * stride;
    const size_t pp = plane_pts(d), pf = pp * d.nyp;
    const int hw = (w - 1) / 2;
    const double inv = 1.0 / ((double)w * w);
    auto raw = [&](int c, int j, int ia, int ka) -> double {
        ia = ((ia % nx) + nx) % nx;
        ka = ((ka % nz) + nz) % nz;
        const size_t o = (size_t)j * pp + (size_t)ka * nx + ia;
        return c == 1 ? 0.5 * (u[pf + o] + u[pf + o + pp]) : u[(size_t)c * pf + o];
    };
    auto bar = [&](int c, int j, int ic, int kc) {
        double a = 0.0;
        for (int dk = -hw; dk <= hw; ++dk)
            for (int di = -hw; di <= hw; ++di) a += raw(c, j, ic + di, kc + dk);
        return a * inv;
    };
    float* xo = x + s * 11;
    const double hy = gyf[J + 1] - gyf[J - 1];
    double gr[9], g2 = 0.0;
    if (w == 1) {
        // unfiltered (the LES features): neighbours once, no modulo per access
        const int ip = i + 1 < nx ? i + 1 : 0, im = i > 0 ? i - 1 : nx - 1;
        const int kp = k + 1 < nz ? k + 1 : 0, km = k > 0 ? k - 1 : nz - 1;
        const size_t o = (size_t)J * pp + (size_t)k * nx + i;
        const size_t oxp = (size_t)J * pp + (size_t)k * nx + ip, oxm = (size_t)J * pp + (size_t)k * nx + im;
        const size_t ozp = (size_t)J * pp + (size_t)kp * nx + i, ozm = (size_t)J * pp + (size_t)km * nx + i;
        const double r2x = 0.5 / dx, r2z = 0.5 / dz, rhy = 1.0 / hy;
        for (int c = 0; c < 3; ++c) {
            auto at = [&](size_t q) { return c == 1 ? 0.5 * (u[pf + q] + u[pf + q + pp]) : u[(size_t)c * pf + q]; };
            gr[3 * c + 0] = (at(oxp) - at(oxm)) * r2x;
            gr[3 * c + 1] = (at(o + pp) - at(o - pp)) * rhy;
            gr[3 * c + 2] = (at(ozp) - at(ozm)) * r2z;
        }
    } else {
        for (int c = 0; c < 3; ++c) {
            gr[3 * c + 0] = (bar(c, J, i + 1, k) - bar(c, J, i - 1, k)) / (2.0 * dx);
            gr[3 * c + 1] = (bar(c, J + 1, i, k) - bar(c, J - 1, i, k)) / hy;
            gr[3 * c + 2] = (bar(c, J, i, k + 1) - bar(c, J, i, k - 1)) / (2.0 * dz);
        }
    }
    for (int q = 0; q < 9; ++q) g2 += gr[q] * gr[q];
    const double G = sqrt(g2), ig = G > 0.0 ? 1.0 / G : 0.0;
    for (int q = 0; q < 9; ++q) xo[q] = (float)(gr[q] * ig);
    const double dwall = fmin(gyf[J] - gyf[1], gyf[ny] - gyf[J]);
    const double delta = cbrt((double)w * dx * dyf[J] * (double)w * dz);
    xo[9] = (float)(dwall / nu);
    xo[10] = (float)delta;
    const double scale = delta * delta * g2;
    sc[s] = (float)scale;
    if (!t) return;
    float* to = t + s * 6;
    double ub[3] = {bar(0, J, i, k), bar(1, J, i, k), bar(2, J, i, k)};
    double pr[6] = {0, 0, 0, 0, 0, 0};
    for (int dk = -hw; dk <= hw; ++dk)
        for (int di = -hw; di <= hw; ++di) {
            const double a = raw(0, J, i + di, k + dk), b = raw(1, J, i + di, k + dk), c = raw(2, J, i + di, k + dk);
            pr[0] += a * a; pr[1] += b * b; pr[2] += c * c; pr[3] += a * b; pr[4] += a * c; pr[5] += b * c;
        }
    const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
    const double is = scale > 0.0 ? 1.0 / scale : 0.0;
    for (int q = 0; q < 6; ++q) to[q] = (float)((pr[q] * inv - ub[pa[q]] * ub[pb[q]]) * is);
}

// The closure's stresses at GYF points J = 2..NY-1 (the network's
// dimensionless output y [n][6] in the sampler's order times the sample's
// scale s, every x and z point) into physical fields: tau_11,
// tau_22, tau_33, tau_13 at GYF points; tau_12, tau_23 interpolated to GY
// points J = 3..NY-1 with the weights of the GY interpolation of channel.f
// (DYF(J-1), DYF(J)); all other rows zero.  out: 6 fields [J][z][x].
__global__ void __launch_bounds__(TB) k_mlp_tau_fields(Dims d, const float* __restrict__ tau,
                                                       const float* __restrict__ sc, const double* __restrict__ dy,
                                                       const double* __restrict__ dyf, double* __restrict__ out) {
    const size_t pp = plane_pts(d), pf = pp * d.nyp;
    const size_t g = (size_t)blockIdx.x * TB + threadIdx.x;
    if (g >= pf) return;
    const int J = (int)(g / pp), ny = d.ny;
    const size_t col = g % pp;
    auto T = [&](int q, int j) {
        const size_t e = (size_t)(j - 2) * pp + col;
        return (double)(tau[e * 6 + q] * sc[e]);
    };
    const bool f = J >= 2 && J <= ny - 1;
    out[g] = f ? T(0, J) : 0.0;              // 11
    out[pf + g] = f ? T(1, J) : 0.0;         // 22
    out[2 * pf + g] = f ? T(2, J) : 0.0;     // 33
    out[3 * pf + g] = f ? T(4, J) : 0.0;     // 13
    const bool gy = J >= 3 && J <= ny - 1;
    const double w0 = gy ? dyf[J - 1] : 0.0, w1 = gy ? dyf[J] : 0.0, h2 = 2.0 * dy[J];
    out[4 * pf + g] = gy ? (T(3, J) * w0 + T(3, J - 1) * w1) / h2 : 0.0;   // 12 at GY
    out[5 * pf + g] = gy ? (T(5, J) * w0 + T(5, J - 1) * w1) / h2 : 0.0;   // 23 at GY
}

// CF_i -= d tau_ij / dx_j for the closure's stresses (all explicit): tau
// holds the forward transforms of k_mlp_tau_fields' six fields.
__global__ void __launch_bounds__(TB) k_mlp_tau_cf(Dims d, const double2* __restrict__ tau, double2* __restrict__ cf,
                                                   const double* __restrict__ kxw, const double* __restrict__ kzw,
                                                   const double* __restrict__ dy, const double* __restrict__ dyf) {
    int J, m, kx;
    if (!spec_index(d, (size_t)blockIdx.x * TB + threadIdx.x, J, m, kx)) return;
    const int ny = d.ny;
    if (J < 2 || J > ny) return;
    const size_t ps = d.splane(), fs = ps * d.nyp;
    const size_t o = (size_t)J * ps + (size_t)m * d.ldx + kx;
    const double KX = kxw[kx], KZ = kzw[m];
    auto T = [&](int q, int j) { return tau[(size_t)q * fs + o + (size_t)(j - J) * ps]; };
    if (J <= ny - 1) {
        double2* f1 = cf + o;
        double2* f3 = cf + 2 * fs + o;
        *f1 = *f1 - ik(KX, T(0, J)) - (T(4, J + 1) - T(4, J)) / dyf[J] - ik(KZ, T(3, J));
        *f3 = *f3 - ik(KX, T(3, J)) - (T(5, J + 1) - T(5, J)) / dyf[J] - ik(KZ, T(2, J));
    }
    double2* f2 = cf + fs + o;
    *f2 = *f2 - ik(KX, T(4, J)) - (T(1, J) - T(1, J - 1)) / dy[J] - ik(KZ, T(5, J));
}

// COURANT's velocity limit (courant.f:35-47) over physical rows 1..NY of the
// fields the physical solves left (they are not band-limited, so the limit
// is taken on them rather than on their transforms).  Non-negative doubles
// order like their bit patterns, so the minimum is an integer atomicMin.
__global__ void __launch_bounds__(TB) k_les_cfl(Dims d, const double* __restrict__ u, const double* __restrict__ dy,
                                                double cfl, double dx, double dz, double* dtmin) {
    __shared__ double red[TB];
    const size_t pp = plane_pts(d), pf = pp * d.nyp;
    const size_t n = pp * (size_t)d.ny;
    double m = __longlong_as_double(0x7ff0000000000000LL);   // +inf
    for (size_t g = (size_t)blockIdx.x * TB + threadIdx.x; g < n; g += (size_t)gridDim.x * TB) {
        const size_t q = g + pp;
        const int J = (int)(q / pp);
        const double tx = cfl * dx / fabs(u[q]);
        const double ty = cfl * dy[J] / fabs(u[pf + q]);
        const double tz = cfl * dz / fabs(u[2 * pf + q]);
        m = fmin(m, fmin(tx, fmin(ty, tz)));
    }
    red[threadIdx.x] = m;
    __syncthreads();
    for (int s = TB / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] = fmin(red[threadIdx.x], red[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0)
        atomicMin(reinterpret_cast<unsigned long long*>(dtmin), (unsigned long long)__double_as_longlong(red[0]));
}

}  // namespace

cudaError_t launch_les_pre(const CnArgs& a, const double* k2, double2* r, cudaStream_t st) {
    k_les_pre<<<blocks(spec_items(a.d)), TB, 0, st>>>(a, k2, r);
    return cudaGetLastError();
}

cudaError_t launch_les_bc(const Dims& d, double2* cu, const diablo_params& p, cudaStream_t st) {
    k_les_bc<<<blocks(d.splane()), TB, 0, st>>>(d, cu, p.u_bc_ymax, p.w_bc_ymax, p.u_bc_ymin, p.w_bc_ymin);
    return cudaGetLastError();
}

cudaError_t launch_les_strain(const Dims& d, const double2* cu, const double* kx, const double* kz, const double* dy,
                              const double* dyf, double2* sij, cudaStream_t st) {
    k_les_strain<<<blocks(spec_items(d)), TB, 0, st>>>(d, cu, kx, kz, dy, dyf, sij);
    return cudaGetLastError();
}

cudaError_t launch_les_sgs(const Dims& d, const double* sij, const double* u, const double2* cu, const double* dy,
                           const double* dyf, const double* delta_y, double* out, double* nut, cudaStream_t st) {
    k_les_sgs<<<blocks(plane_pts(d) * d.nyp), TB, 0, st>>>(d, sij, u, cu, dy, dyf, delta_y, out, nut);
    return cudaGetLastError();
}

cudaError_t launch_phys_bc_vel(const Dims& d, double* u, const double* dy, const double* dyf, const diablo_params& p,
                               cudaStream_t st) {
    k_phys_bc_vel<<<blocks(plane_pts(d)), TB, 0, st>>>(d, u, dy, dyf, p);
    return cudaGetLastError();
}

cudaError_t launch_les_tau_cf(const Dims& d, const double2* tau, double2* cf, const double* kx, const double* kz,
                              const double* dyf, const double* delta_yf, const double* delta_y, cudaStream_t st) {
    k_les_tau_cf<<<blocks(spec_items(d)), TB, 0, st>>>(d, tau, cf, kx, kz, dyf, delta_yf, delta_y);
    return cudaGetLastError();
}

cudaError_t launch_les_kgrad(const Dims& d, const double2* cth, const double* kx, const double* kz, double2* out,
                             cudaStream_t st) {
    k_les_kgrad<<<blocks(spec_items(d)), TB, 0, st>>>(d, cth, kx, kz, out);
    return cudaGetLastError();
}

cudaError_t launch_les_kmul(const Dims& d, double* a, const double* nut, cudaStream_t st) {
    k_les_kmul<<<blocks(plane_pts(d) * d.nyp), TB, 0, st>>>(d, a, nut);
    return cudaGetLastError();
}

cudaError_t launch_les_kcf(const Dims& d, const double2* g2, double2* cfth, const double* kx, const double* kz, int j0,
                           int j1, cudaStream_t st) {
    k_les_kcf<<<blocks(spec_items(d)), TB, 0, st>>>(d, g2, cfth, kx, kz, j0, j1);
    return cudaGetLastError();
}

cudaError_t launch_les_post(const CnArgs& a, const double2* nl, double2* r, cudaStream_t st) {
    k_les_post<<<blocks(spec_items(a.d)), TB, 0, st>>>(a, nl, r);
    return cudaGetLastError();
}

cudaError_t launch_les_explicit(const LesArgs& a, const double* u, double* r, const double* nut, cudaStream_t st) {
    k_les_explicit<<<blocks(plane_pts(a.d) * a.d.nyp), TB, 0, st>>>(a, u, r, nut);
    return cudaGetLastError();
}

cudaError_t launch_les_solve(const LesArgs& a, double* r, const double* nut, double* piv, double* out,
                             cudaStream_t st) {
    dim3 grid(blocks(plane_pts(a.d)), a.d.nf);
    k_les_solve<<<grid, TB, 0, st>>>(a, r, nut, piv, out);
    return cudaGetLastError();
}

cudaError_t launch_dyn_widths(const Dims& d, const double* sij, const double* u, const double2* cu, const double* dy,
                              const double* dyf, double R, double* sums, double* widths, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(sums, 0, sizeof(double) * 2 * d.nyp, st);
    if (e != cudaSuccess) return e;
    const size_t smem = sizeof(double) * ((size_t)NB * DZ_S * DX_S + (size_t)NQ * DZ_S * DX_T);
    cudaFuncSetAttribute(k_dyn_sums, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 grid((d.nx + DX_T - 1) / DX_T, (d.nz + DZ_T - 1) / DZ_T, d.ny - 1);
    k_dyn_sums<<<grid, 256, smem, st>>>(d, sij, u, cu, dy, R, sums);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_dyn_widths<<<1, 256, 0, st>>>(d, sums, dy, dyf, widths);
    return cudaGetLastError();
}

cudaError_t launch_sgs_samples(const Dims& d, const double* u, const double* gyf, const double* dyf, double dx,
                               double dz, double nu, int w, int stride, float* x, float* t, float* sc, cudaStream_t st) {
    const int nxs = (d.nx + stride - 1) / stride, nzs = (d.nz + stride - 1) / stride;
    const long long ns = (long long)(d.ny - 2) * nzs * nxs;
    if (ns <= 0) return cudaSuccess;
    k_sgs_samples<<<(unsigned)((ns + TB - 1) / TB), TB, 0, st>>>(d, u, gyf, dyf, dx, dz, nu, w, stride, x, t, sc);
    return cudaGetLastError();
}

cudaError_t launch_mlp_tau_fields(const Dims& d, const float* tau, const float* sc, const double* dy, const double* dyf,
                                  double* out, cudaStream_t st) {
    k_mlp_tau_fields<<<blocks(plane_pts(d) * d.nyp), TB, 0, st>>>(d, tau, sc, dy, dyf, out);
    return cudaGetLastError();
}

cudaError_t launch_mlp_tau_cf(const Dims& d, const double2* tau, double2* cf, const double* kx, const double* kz,
                              const double* dy, const double* dyf, cudaStream_t st) {
    k_mlp_tau_cf<<<blocks(spec_items(d)), TB, 0, st>>>(d, tau, cf, kx, kz, dy, dyf);
    return cudaGetLastError();
}

cudaError_t launch_les_cfl(const Dims& d, const double* u, const double* dy, double cfl, double dx, double dz,
                           double* dtmin, cudaStream_t st) {
    const size_t n = plane_pts(d) * (size_t)d.ny;
    unsigned nb = blocks(n);
    if (nb > 148 * 8) nb = 148 * 8;
    k_les_cfl<<<nb, TB, 0, st>>>(d, u, dy, cfl, dx, dz, dtmin);
    return cudaGetLastError();
}

}  // namespace dgpu
