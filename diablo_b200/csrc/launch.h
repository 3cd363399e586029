// launch.h -- host-side launchers of the device kernels.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "../../include/diablo_gpu.h"
#include "kernels.cuh"

namespace dgpu {

// Planes [j0, j0+nplanes) of fields [0,nfields) of S (FP64 spectral) ->
// X (x-spectrum, type T): unpack kz, backward z transform (mpi.f:1562-1577).
// skip_mean: leave out the (0,0) mode, so X is the fluctuation about the
// plane mean (the FP32 transform path; the mean stays FP64).
template <typename T>
cudaError_t launch_zinv(const Dims& d, const double2* S, size_t s_fstride, void* X, size_t x_fstride,
                        int nfields, int j0, int nplanes, const FftPlan& pz, const void* twz,
                        cudaStream_t st, int skip_mean = 0);

// Fused per z-row: backward x transform of the fields at planes jlo-1..jhi+1,
// the 8 + 3*N_TH physical products of RK_CHAN_1 (channel.f:410-571,
// 670-720) at planes jlo..jhi, forward x transform with 1/NX and truncation
// to kx <= NKX (mpi.f:1493-1508), combined into 2 outputs per field
// (ikx*Pa + Pflux, Pz) -> Y.
// pm/twm: plan and table of the NX/2-point complex FFT; twn: table of NX.
// means (S layout, field stride means_fstride): when given, X holds each
// field's fluctuation about its plane mean (launch_zinv with skip_mean) and
// the products are formed without their mean x mean part, which only the
// (0,0) mode carries (the column kernel adds it in FP64).
template <typename T>
cudaError_t launch_products(const Dims& d, const void* X, void* Y, int jlo, int jhi, int chunk,
                            const double* dy, const double* dyf, const double* kx, const FftPlan& pm,
                            const void* twm, const void* twn, cudaStream_t st, const double2* means = nullptr,
                            size_t means_fstride = 0);

// The same products for NX = 512 in FP32 (products_hw.cu): one block per
// z-row, one half-warp per field, register-resident 256-point transforms.
bool products_hw_supported(const Dims& d);
size_t products_hw_smem(const Dims& d);
cudaError_t launch_products_hw(const Dims& d, const void* X, void* Y, int jlo, int jhi, int chunk, const double* dy,
                               const double* dyf, const double* kx, const void* twm, const void* twn, cudaStream_t st,
                               const double2* means, size_t means_fstride);
// Batched form (see launch_zinv_b); the state of each instance gives the plane means.
cudaError_t launch_products_hw_b(const Dims& d, const InstPtrs* ip, int ninst, int jlo_min, int jhi, int chunk,
                                 const void* twm, const void* twn, cudaStream_t st, size_t means_fstride);

// Per plane (zp planes per block, 0 = default): forward z transform of the 2
// product outputs of every field,
// kz packing and 1/NZ (mpi.f:1526-1540), then NL = -(first) - ikz (second)
// -> NL (type T, S layout).
template <typename T>
cudaError_t launch_zfwd_nl(const Dims& d, const void* Y, void* NL, int jlo, int jhi, int zp,
                           const double* kx, const double* kz, const FftPlan& pz, const void* twz,
                           cudaStream_t st);

// Batched forms of the three transform kernels: one launch for the ninst
// instances of a group of equal shape, whose arrays come from the device
// table ip (InstPtrs).  jlo_min: the smallest first product plane of the group.
template <typename T>
cudaError_t launch_zinv_b(const Dims& d, const InstPtrs* ip, int ninst, size_t s_fstride, size_t x_fstride,
                          const FftPlan& pz, const void* twz, cudaStream_t st, int skip_mean);
template <typename T>
cudaError_t launch_products_b(const Dims& d, const InstPtrs* ip, int ninst, int jlo_min, int jhi, int chunk,
                              const FftPlan& pm, const void* twm, const void* twn, cudaStream_t st, int mean_split,
                              size_t means_fstride);
template <typename T>
cudaError_t launch_zfwd_nl_b(const Dims& d, const InstPtrs* ip, int ninst, int jlo_min, int jhi, int zp,
                             const FftPlan& pz, const void* twz, cudaStream_t st);

// Transform-API helpers (one field at a time, FP64):
// X -> physical rows P (c2r, unnormalised, Nyquist and kx > NKX zero).
cudaError_t launch_xinv(const Dims& d, const void* X, double* P, int j0, int nplanes,
                        const FftPlan& pm, const void* twm, const void* twn, cudaStream_t st);
// physical rows P -> X (r2c, 1/NX, truncation).
cudaError_t launch_xfwd(const Dims& d, const double* P, void* X, int j0, int nplanes,
                        const FftPlan& pm, const void* twm, const void* twn, cudaStream_t st);
// X -> S (forward z transform, 1/NZ, kz packing) for one field.
cudaError_t launch_zfwd_pack(const Dims& d, const void* X, double2* S, int j0, int nplanes,
                             const FftPlan& pz, const void* twz, cudaStream_t st);

// Column kernels (FP64).
// CN rows of every field and their partition factors (column-independent),
// the BC-row values of the (0,0) mode and the row kinds.
cudaError_t launch_cn_part(const Dims& d, const CnArgs& a, double* tabs, double* bcv, signed char* kind,
                           const int* bc_type, const double* bc_c1, cudaStream_t st);
// doubles of the partition tables per field
size_t part_table_doubles(int nyp);
// rows per CN block of the partition solve (0 when NY+2 > 544)
int part_rows(int nyp);
// Per-column partition factors of the phi system (built once per instance).
size_t phi_table_doubles(const Dims& d);
cudaError_t launch_phi_part(const Dims& d, const double* rows, const double* kx, const double* kz, double* tab,
                            cudaStream_t st);
// One pass per column pair: RHS, CN solves, projection and pressure update.
template <typename TN>
cudaError_t launch_colpart(const ColArgs& a, const TN* nl, const double* tabs, cudaStream_t st);
template <typename TN>
size_t colpart_smem(const Dims& d);
// Batched form for a group of equal shape (ColJob table on the device).
template <typename TN>
cudaError_t launch_colpart_b(const Dims& d, const ColJob* jobs, int ninst, bool pair_blocked, cudaStream_t st);
cudaError_t launch_remdiv(const RemDivArgs& a, cudaStream_t st);

// CFL minimum (courant.f:35-47) over planes 1..NY of the physical velocity
// obtained from X (3 fields, FP64).  Result: atomically min-ed into *dtmin.
cudaError_t launch_cfl(const Dims& d, const void* X, size_t x_fstride, const FftPlan& pm,
                       const void* twm, const void* twn, const double* dy, double cfl, double dx,
                       double dz, double* dtmin, cudaStream_t st);
// POISSON_P_CHAN and SAVE_STATS_CHAN pieces (poisson_stats.cu, FP64).
// One velocity-gradient field of the pressure source into S (kinds 0..8).
cudaError_t launch_grad_field(const Dims& d, int kind, const double2* cu, double2* out, const double* kx,
                              const double* kz, const double* dyf, cudaStream_t st);
// acc (+)= alpha*a*b on physical planes 2..NY.
cudaError_t launch_phys_fma(const Dims& d, double* acc, const double* a, const double* b, double alpha, int init,
                            cudaStream_t st);
cudaError_t launch_poisson_column(const PoissonArgs& a, cudaStream_t st);
// Plane sums of the second-order statistics, planes 1..NY (th may be null).
cudaError_t launch_stats_planes(const Dims& d, const double* u1, const double* u2, const double* u3,
                                const double* th, const double* me, const double* dy, const double* dyf, double* out,
                                cudaStream_t st);
// One Fourier field of the vorticity / dissipation / scalar-gradient
// statistics on rows 1..NY (kinds 0..11, see k_stats_spec).
cudaError_t launch_stats_spec(const Dims& d, int kind, const double2* cu, const double2* cs, double2* out,
                              const double* kx, const double* kz, const double* dyf, const double* gyf,
                              cudaStream_t st);
// acc[j] (+)= plane sum of one statistics term (modes 0..5), planes jlo..jhi.
cudaError_t launch_plane_terms(const Dims& d, int mode, const double* f, const double* u, const double* m,
                               const double* m2, const double* dy, const double* dyf, const double* rg, int jlo,
                               int jhi, double* acc, int init, cudaStream_t st);
// filter_chan (filter.f:1-98) on one scalar field of the S layout; fnx, fnz
// are NX and NZ as the reference's FLOAT() gives them.
cudaError_t launch_filter_chan(const Dims& d, double2* cth, const double* kx, const double* kz, double lx,
                               double lz, double fnx, double fnz, cudaStream_t st);
// Constant-Smagorinsky LES branch (les.cu, FP64).  Spectral kernels run over
// the retained modes of planes 0..NY+1, physical ones over P[J][z][x].
cudaError_t launch_les_pre(const CnArgs& a, const double* k2, double2* r, cudaStream_t st);
cudaError_t launch_les_bc(const Dims& d, double2* cu, const diablo_params& p, cudaStream_t st);
cudaError_t launch_les_strain(const Dims& d, const double2* cu, const double* kx, const double* kz, const double* dy,
                              const double* dyf, double2* sij, cudaStream_t st);
cudaError_t launch_les_sgs(const Dims& d, const double* sij, const double* u, const double2* cu, const double* dy,
                           const double* dyf, const double* delta_y, double* out, double* nut, cudaStream_t st);
cudaError_t launch_phys_bc_vel(const Dims& d, double* u, const double* dy, const double* dyf, const diablo_params& p,
                               cudaStream_t st);
cudaError_t launch_les_tau_cf(const Dims& d, const double2* tau, double2* cf, const double* kx, const double* kz,
                              const double* dyf, const double* delta_yf, const double* delta_y, cudaStream_t st);
cudaError_t launch_les_kgrad(const Dims& d, const double2* cth, const double* kx, const double* kz, double2* out,
                             cudaStream_t st);
cudaError_t launch_les_kmul(const Dims& d, double* a, const double* nut, cudaStream_t st);
cudaError_t launch_les_kcf(const Dims& d, const double2* g2, double2* cfth, const double* kx, const double* kz, int j0,
                           int j1, cudaStream_t st);
cudaError_t launch_les_post(const CnArgs& a, const double2* nl, double2* r, cudaStream_t st);
cudaError_t launch_les_explicit(const LesArgs& a, const double* u, double* r, const double* nut, cudaStream_t st);
// All fields' column solves; r (nf physical fields) is overwritten, piv holds
// nf fields of pivots, out receives the solution rows.
cudaError_t launch_les_solve(const LesArgs& a, double* r, const double* nut, double* piv, double* out,
                             cudaStream_t st);
// Dynamic Smagorinsky widths: plane sums of L_ij M_ij and M_ij M_ij (sums,
// 2*(NY+2) doubles, zeroed here), then widths[0..NY+1] = Delta_YF and
// widths[NY+2..] = Delta_Y.  sij: the six physical strain fields, u: U1..U3.
cudaError_t launch_dyn_widths(const Dims& d, const double* sij, const double* u, const double2* cu, const double* dy,
                              const double* dyf, double R, double* sums, double* widths, cudaStream_t st);
// Closure samples (features [n][11], targets [n][6], scales [n]; t may be
// null) of a w x w x-z top-hat
// filter at GYF points J = 2..NY-1 and every stride-th x and z point.
cudaError_t launch_sgs_samples(const Dims& d, const double* u, const double* gyf, const double* dyf, double dx,
                               double dz, double nu, int w, int stride, float* x, float* t, float* sc, cudaStream_t st);
// The closure's stresses ([n][6] at GYF rows 2..NY-1) to six physical fields
// (11, 22, 33, 13 at GYF; 12, 23 at GY), and their divergence into CF.
cudaError_t launch_mlp_tau_fields(const Dims& d, const float* tau, const float* sc, const double* dy, const double* dyf,
                                  double* out, cudaStream_t st);
cudaError_t launch_mlp_tau_cf(const Dims& d, const double2* tau, double2* cf, const double* kx, const double* kz,
                              const double* dy, const double* dyf, cudaStream_t st);
// COURANT's velocity minimum over physical rows 1..NY of U1..U3 (u: 3 fields).
cudaError_t launch_les_cfl(const Dims& d, const double* u, const double* dy, double cfl, double dx, double dz,
                           double* dtmin, cudaStream_t st);
// The learned closure's forward pass on device arrays (mlp.cu): x [n][11]
// features in physical units -> y [n][6] stresses; mlp is a diablo_mlp handle.
cudaError_t launch_mlp_forward(const void* mlp, const float* x, long long n, float* y, cudaStream_t st);
// rows transformed together by the products kernel for a given NX
int products_group(int nx);
// Record the one-line message returned by diablo_gpu_last_error; returns code.
int set_error(int code, const std::string& msg);
}  // namespace dgpu
