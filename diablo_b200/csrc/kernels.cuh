// kernels.cuh -- device data layouts and kernel argument blocks.
//
// Device layouts (all row-major, fastest index last):
//   spectral  S[f][J][m][kx]   complex, J in [0,NY+1], m in [0,TNKZ] (the
//             packed kz of FFT_XZ_TO_FOURIER, mpi.f:1530-1539), kx in
//             [0,NKX]; rows padded to ldx (a multiple of 16) and the kz rows
//             of a plane padded to an even count nkzp, all padding zero.
//             State (CU, CP, CF) is FP64; the nonlinear term NL is the
//             transform type T.
//   x-spectrum X[f][J][z][kx]  complex<T>: after the inverse z transform,
//             kx in [0,NKX] (+ zero padding to ldx), z in [0,NZ).
//   products  Y[p][J][z][kx]   complex<T>: x spectra of the products.
//   physical  P[J][z][x]       real, pitch NX (transform API only).
#pragma once

#include "fft.cuh"

namespace dgpu {

constexpr int MAXF = 3 + 4;   // fields: U1, U2, U3, TH(1..N_TH)

struct Dims {
    int nx, ny, nz, nth, nf, np;
    int nkx, nkz, tnkz, nkxp, nkzt, ldx, nyp;
    int nkzp;   // kz rows per plane in the S layout: nkzt padded to even, so
                // that a plane (nkzp*ldx elements) is a multiple of 32 columns
    __host__ __device__ size_t splane() const { return (size_t)nkzp * ldx; }
};

// Offset of element (plane J, column g = m*ldx + kx) within one field of a
// spectral array, in the S layout or in the pair-blocked layout that CF
// takes on the Fourier-space path: column pairs (g, g+1) with g even, each
// pair's NY+2 rows contiguous ([pair][J][2]), so that the column kernel,
// which handles one pair per block and is CF's only reader and writer there,
// reads and writes it as one contiguous run.
__host__ __device__ __forceinline__ size_t spec_at(const Dims& d, bool pair_blocked, int J, size_t g) {
    return pair_blocked ? (g >> 1) * (size_t)(2 * d.nyp) + (size_t)J * 2 + (g & 1) : (size_t)J * d.splane() + g;
}

// Per-instance arrays of a batched launch over a group of instances of equal
// shape (the transform kernels' *_b entries): instance i of the group reads
// its own state, scratch and grid tables through entry i.
struct InstPtrs {
    const double2* cu;    // state (S layout, nf fields)
    void* xb;             // x spectra X
    void* yb;             // product spectra Y
    void* nl;             // nonlinear term NL
    const double* dy;
    const double* dyf;
    const double* kx;
    const double* kz;
    int jlo_prod;         // first product plane
};

// Everything K4 (the column kernel) needs besides the arrays.
struct CnArgs {
    Dims d;
    double2* cu;          // S, nf fields (in: CU old, out: CU after the CN solves)
    double2* cf;          // S, nf fields (in: CF old, out: CF new)
    const double2* cp;    // S, 1 field
    const double* kx;     // KX(0..ldx-1), zero beyond NKX
    const double* kz;     // KZ(0..TNKZ)
    const double* dy;     // DY(0..NY+1)
    const double* dyf;    // DYF(0..NY+1)
    const double* bcv;    // [nf][nyp] RHS of BC rows for the (0,0) mode
    const signed char* kind;  // [nf][nyp] 0: interior row, 1: BC row
    int cf_lo[MAXF], cf_hi[MAXF];   // rows where CF is formed
    int cb_lo[MAXF];                // first row copied back (last is NY+1)
    double temp1, temp3, temp4, temp5;
    double nu, beta, nu_v_scale, i_ro, grav_x, grav_y, grav_z;
    double ri[4], pr[4], drhodx[4], drhodz[4];
    double forcing;       // value subtracted from CR1(0,0,j) (F_TYPE 1/2), already * TEMP4
    int rk_step;
    int store_cf;
};

// Everything the CN row set-up needs (k_cn_part).
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

// Per-row grid metrics shared by all columns (reciprocals computed once, so
// the column sweeps multiply instead of divide):
enum RowTab {
    RT_RDY = 0,    // 1/DY(j)
    RT_RDYF,       // 1/DYF(j)                          (0 where DYF(j) = 0)
    RT_E1P,        // 1/(DY(j+1) DYF(j))   U1/U3/TH stencil, phi rows C(j)
    RT_E1M,        // 1/(DY(j) DYF(j))     U1/U3/TH stencil, phi rows A(j)
    RT_E2P,        // 1/(DYF(j) DY(j))     U2 stencil
    RT_E2M,        // 1/(DYF(j-1) DY(j))   U2 stencil
    RT_BY0,        // DYF(j-1)/(2 DY(j))   weight of TH(j) at GY(j)
    RT_BY1,        // DYF(j)/(2 DY(j))     weight of TH(j-1) at GY(j)
    RT_COUNT
};

// The column kernel (colpart.cu): CnArgs plus the projection.
struct ColArgs {
    CnArgs cn;
    const double* k2;     // (KX^2+KZ^2)**BETA per padded column [m][kx]
    const double* rows;   // [RT_COUNT][nyp] row tables
    const double* phitab; // per column: partition factors of the phi system
    double2* phi;         // S, phi (J = 1..NY), written when store_phi
    double inv_h;         // 1/TEMP4
    int project;          // run the REM_DIV projection
    int update_cp;        // CP += phi/h on J = 2..NY
    int store_phi;
    int* nan_flag;        // set to 1 when a new CU value is not finite (may be null)
    int pair_blocked;     // CF is in the pair-blocked layout (spec_at)
    int mean_split;       // the nonlinear term lacks the mean x mean products: add them to
                          // the (0,0) mode in FP64 on the product planes jlo_prod..NY
    int jlo_prod;
};

// One instance of a batched column launch (launch_colpart_b).
struct ColJob {
    ColArgs A;
    const void* nl;       // nonlinear term, the transform type
    const double* tabs;   // CN partition tables of the substage
};

struct RemDivArgs {
    Dims d;
    double2* cu;          // S, velocity fields 0..2
    double2* cp;          // S
    double2* phi;         // S, phi (J = 1..NY)
    const double* rows;   // [RT_COUNT][nyp] reciprocal row tables
    const double* phitab; // per-column phi partition factors (k_phi_part)
    const double* kx;
    const double* kz;
    const double* dy;
    const double* dyf;
    double inv_h;         // 1/TEMP4 for the pressure update
    int update_cp;        // CP += phi/h on J = 2..NY
    int* nan_flag;        // set to 1 when a new velocity value is not finite (may be null)
};

// Physical-space CN steps of the LES branch (les.cu).
struct LesArgs {
    Dims d;
    const double* dy;
    const double* dyf;
    const double* rows;             // [RT_COUNT][nyp] reciprocal row tables
    double temp1, temp2, nu_v_scale;
    double pr[4];
    int j_lo[MAXF], j_hi[MAXF];     // interior rows of each field's system
    int out_lo[MAXF];               // first row copied back (the last is NY+1)
    int bc_type[MAXF][2];
    double bc_c1[MAXF][2];
};

// POISSON_P_CHAN column solve (poisson_stats.cu).
struct PoissonArgs {
    Dims d;
    const double2* rhs;   // S, sum_ij (du_i/dx_j)(du_j/dx_i) on J = 2..NY-1
    const double2* cth;   // S, N_TH scalar fields
    double2* cp;          // S, receives CP on J = 1..NY
    double* bsc;          // scratch pivots  [J][m][kx]
    double2* gsc;         // scratch RHS     [J][m][kx]
    const double* kx;
    const double* kz;
    const double* dy;
    const double* dyf;
    const double* gyf;
    double ri[4];
};

}  // namespace dgpu
