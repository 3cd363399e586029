/*
 * diablo_oracle.h -- CPU FP64 restatement of DIABLO's channel timestep.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the correctness oracle for the GPU
 * library: it is used by tests/, by __graft_entry__.smoke() and by the
 * cpu_baseline leg of bench.py, as the checker and never as the product.
 *
 * It restates, routine by routine, the reference's MPI build with
 * NPROCY = NPROCZ = 1 (the only channel build that links, since the serial
 * stubs in dummy_code/mpi_serial.f lack FFT_XZ_*), keeping the Fortran
 * COMMON layouts and the EQUIVALENCE aliasing (U1<->CU1, S1<->CS1, ...) of
 * for/header:222-258.  FFTW 3.3.10 (the third-party transform the reference
 * links, for/Makefile:78) is restated by its published definition: forward
 * DFT with exp(-2 pi i jk/n), backward with exp(+2 pi i jk/n), both
 * unnormalised; the c2r transform reads the half spectrum and ignores the
 * imaginary parts of the DC and Nyquist bins.
 *
 * Parity status: the reference cannot be built here (no Fortran compiler,
 * no FFTW/MPI/HDF5), so whole-step outputs are NOT pinned against reference
 * runs ("parity unpinned" at the step level).  What is pinned: the transform
 * conventions against numpy.fft (an independent implementation of the same
 * DFT definition), the y-grid construction against the reference's own
 * KH_test/grid.h5, and the physics known-answer tests of the test suite.
 */
#ifndef DIABLO_ORACLE_H
#define DIABLO_ORACLE_H

#include <stddef.h>
#include "../include/diablo_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_state orc_state;

/* Array identifiers for orc_array(). */
enum {
    ORC_U1 = 0, ORC_U2, ORC_U3, ORC_P, ORC_R1, ORC_R2, ORC_R3,
    ORC_F1, ORC_F2, ORC_F3, ORC_S1,
    ORC_TH, ORC_CTH, ORC_FTH, ORC_CFTH, ORC_RTH, ORC_CRTH,
    ORC_GY, ORC_GYF, ORC_DY, ORC_DYF, ORC_KX, ORC_KZ,
    ORC_NU_T,
    ORC_NARRAYS
};

/* Allocate and initialise (CREATE_GRID_CHAN spacing, INIT_CHAN_MPI ranges,
 * INIT_FFT wavenumbers, RK coefficients of diablo_io.f:116-124).
 * gy, gyf: GY(0:NY+1), GYF(0:NY+1). */
orc_state* orc_create(const diablo_params* p, const double* gy, const double* gyf,
                      double delta_t);
void orc_destroy(orc_state* s);
/* Pointer to an array of the state (Fortran layout, see diablo_gpu.h). */
double* orc_array(orc_state* s, int which);
size_t orc_array_doubles(orc_state* s, int which);
/* Scalars of /RUNTIME_VARS/ and /RKW3_PARAMS/. */
void orc_get_time(orc_state* s, double* time, double* delta_t, int* time_step,
                  double* h_bar);
void orc_set_time(orc_state* s, double time, double delta_t, int time_step);
void orc_set_threads(int n);

/* Routines of the reference, on the state. */
void orc_fft_xz_to_fourier(orc_state* s, double* v, double* vv, int jmin, int jmax);
void orc_fft_xz_to_physical(orc_state* s, double* vv, double* v, int jmin, int jmax);
void orc_rk_chan_1(orc_state* s, int rk_step);
void orc_rem_div_chan(orc_state* s);
void orc_poisson_p_chan(orc_state* s);
void orc_courant(orc_state* s);
void orc_apply_bc_vel(orc_state* s);
void orc_apply_bc_scalar(orc_state* s);
/* One time step of diablo.f:66-111 without I/O: three RK_CHAN_1 substages,
 * then TIME += DELTA_T and TIME_STEP += 1. */
void orc_step(orc_state* s);
/* filter_chan(n) of filter.f on scalar n (1..N_TH). */
void orc_filter_chan(orc_state* s, int n);
/* Statistics of SAVE_STATS_CHAN (DIABLO_STAT_* profiles, NY+2 each). */
void orc_stats(orc_state* s, double* profiles);
/* Every mean.h5 / tke.h5 profile: chan DIABLO_NMEAN*(NY+2), scal
 * N_TH*DIABLO_NSCAL*(NY+2), eps NY+2 (or NULL), as diablo_gpu_mean_stats. */
void orc_mean_stats(orc_state* s, double* chan, double* scal, double* eps);
/* USER_RHS_CHAN_FOURIER (kind 0, channel.f:297) / USER_RHS_CHAN_PHYSICAL
 * (kind 1, channel.f:578): fn(user) runs at that point of orc_rk_chan_1 and
 * may change CF1..CF3, CFTH through orc_array; NULL removes it. */
void orc_set_user_rhs(orc_state* s, int kind, void (*fn)(void*), void* user);
/* tkebudget_chan_les's epsilon_sgs (plane sums, NY+2 values, rows 1..NY). */
void orc_epsilon_sgs(orc_state* s, double* out);
/* tkebudget_chan's 3-D dissipation field F1 (rows 2..NY-1), physical layout. */
void orc_epsilon_field(orc_state* s, double* F1);
/* Parameters of the learned closure (LES_MODEL_TYPE 4), in the layout of the
 * GPU library's diablo_mlp_set_params; NULL removes it. */
void orc_set_mlp(orc_state* s, const float* params);
/* Plain complex DFT of length n (interleaved), sign -1 or +1, unnormalised;
 * exposed for the transform-convention tests. */
int orc_cdft(int n, double* data, int sign);

#ifdef __cplusplus
}
#endif
#endif
