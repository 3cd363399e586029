/*
 * diablo_gpu.h -- C ABI of the B200 (sm_100a) channel timestep library.
 *
 * The library replaces the body of DIABLO's channel solver step for the
 * Fortran host: RK_CHAN_1 (for/channel.f:62-1073) together with the x/z
 * transform wrappers FFT_XZ_TO_FOURIER / FFT_XZ_TO_PHYSICAL
 * (for/mpi.f:1477-1606), the projection REM_DIV_CHAN (for/channel.f:1103-1214),
 * the restart pressure solve POISSON_P_CHAN (for/channel.f:1217-1453) and the
 * CFL step COURANT (for/courant.f:1-66).  In the reference all of these take
 * no arguments and talk through COMMON blocks; here the COMMON state that
 * RK_CHAN_1 reads and writes lives on the device inside an opaque handle, and
 * the host moves it in and out with the upload / download calls.
 *
 * Conventions
 *  - Every pointer argument is a HOST pointer.  No torch or CUDA types appear.
 *  - Fourier-space arrays use the Fortran layout of the COMMON arrays
 *    CU1(0:NXP,0:NZ+1,0:NY+1) (for/header:236-249): COMPLEX*16 stored as
 *    interleaved (re,im) doubles, column-major, NXP = NX/2.  Only the
 *    dealiased block I in [0,NKX], K in [0,TNKZ] (NKX=NX/3, TNKZ=2*(NZ/3)) is
 *    read or written; the other entries of a host array are left untouched
 *    on download and ignored on upload, as every Fourier-space loop of the
 *    reference only visits that block.
 *  - Physical-space arrays use the layout U1(0:NX+1,0:NZ+1,0:NY+1) REAL*8
 *    (for/header:222-229, NPROCZ=1 so NZP=NZ).
 *  - Return value: 0 on success, a negative DIABLO_E* code on failure.
 *    diablo_gpu_last_error() gives a one-line message for the last failure
 *    on the calling thread.
 *  - One handle = one channel instance = one CUDA stream.  Calls on the same
 *    handle must not overlap in time (the reference is single-threaded).
 */
#ifndef DIABLO_GPU_H
#define DIABLO_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define DIABLO_OK            0
#define DIABLO_EINVAL       -1   /* bad dimensions or parameters, null pointer */
#define DIABLO_ERADIX       -2   /* NX or NZ is not a product of 2, 3 and 5 */
#define DIABLO_ECUDA        -3   /* a CUDA runtime call failed */
#define DIABLO_ENOTSUP      -4   /* feature not supported (RK_CHAN_2, LES_MODEL_TYPE 3) */
#define DIABLO_ENAN         -5   /* a non-finite value was found in the state: the kernels
                                    that write CU flag it on the device, and the next call
                                    that synchronises (diablo_gpu_synchronize,
                                    download_state, COURANT inside rk_chan_1 or
                                    diablo_gpu_courant) returns it once */
#define DIABLO_ENOMEM       -6   /* device allocation failed */
#define DIABLO_ETIMEOUT     -7   /* a bounded wait inside a kernel gave up; reserved: no
                                    kernel of this library waits on another block, stream
                                    or device, so no call returns it */

#define DIABLO_MAX_TH        4   /* largest N_TH the library accepts */

#define DIABLO_PREC_FP64     0   /* every kernel in FP64 */
#define DIABLO_PREC_FP32SPLIT 1  /* transforms + products in FP32; solves, state, (0,0) mode in FP64 */

/* Run parameters: grid_def + input.dat + input_chan.dat (for/diablo_io.f:11-46,
 * for/channel.f:1466-1509).  Names follow the Fortran variables. */
typedef struct diablo_params {
    /* grid_def (for/grid_def) */
    int nx, ny, nz, n_th;
    /* input.dat */
    double nu, beta, lx, ly, lz;
    double nu_v_scale;
    int variable_dt, update_dt;
    double cfl;
    int les;                       /* LES flag of input.dat */
    int create_new_flow;
    /* input_chan.dat */
    double i_ro;
    double grav_x, grav_y, grav_z;
    int f_type;
    double ubulk0, px0, omega0, amp_omega0;
    int u_bc_ymin, v_bc_ymin, w_bc_ymin;
    int u_bc_ymax, v_bc_ymax, w_bc_ymax;
    double u_bc_ymin_c1, v_bc_ymin_c1, w_bc_ymin_c1;
    double u_bc_ymax_c1, v_bc_ymax_c1, w_bc_ymax_c1;
    int th_bc_ymin[DIABLO_MAX_TH], th_bc_ymax[DIABLO_MAX_TH];
    double th_bc_ymin_c1[DIABLO_MAX_TH], th_bc_ymax_c1[DIABLO_MAX_TH];
    double ri[DIABLO_MAX_TH], pr[DIABLO_MAX_TH];
    double drhodx[DIABLO_MAX_TH], drhodz[DIABLO_MAX_TH];
    /* library options */
    int precision;                 /* DIABLO_PREC_* */
    /* input_chan.dat LES_MODEL_TYPE (for/channel.f:1477): 1 the constant
     * Smagorinsky model of for/les.f; 2 a dynamic Smagorinsky model of this
     * library (the reference stops for 2 and 3, for/les.f:269-272); 4 the
     * learned closure (diablo_gpu_set_sgs_mlp), the dynamic model without one */
    int les_model_type;
} diablo_params;

/* Create a channel instance on the current CUDA device.
 * gy, gyf, dy, dyf: GY(0:NY+1), GYF(0:NY+1), DY(0:NY+1), DYF(0:NY+1) of
 * /GRID_PARAMS/ (for/header:205-207) as set by CREATE_GRID_CHAN
 * (for/channel.f:1564-1655).  Replaces INIT_FFT's plans and wavenumbers
 * (for/fft.f:55-143) and INIT_CHAN_MPI's JSTART/JEND (for/mpi.f:1013-1081). */
int diablo_gpu_create(const diablo_params* p, const double* gy, const double* gyf,
                      const double* dy, const double* dyf, void** handle);
int diablo_gpu_destroy(void* handle);

/* Copy the RK_CHAN_1 inputs from host COMMON arrays to the device.
 * cu1..cp: CU1, CU2, CU3, CP; cth: CTH(...,1:N_TH) (N_TH consecutive arrays);
 * cf1..cfth: CF1, CF2, CF3, CFTH (may be NULL: the device copy is zeroed,
 * which is what RK_STEP=1 needs). */
int diablo_gpu_upload_state(void* handle, const double* cu1, const double* cu2,
                            const double* cu3, const double* cp, const double* cth,
                            const double* cf1, const double* cf2, const double* cf3,
                            const double* cfth);
/* Copy the device state back into host COMMON arrays (any pointer may be NULL). */
int diablo_gpu_download_state(void* handle, double* cu1, double* cu2, double* cu3,
                              double* cp, double* cth, double* cf1, double* cf2,
                              double* cf3, double* cfth);

/* One RK substage: the body of RK_CHAN_1 (for/channel.f:62-1073), including
 * the REM_DIV_CHAN projection and the pressure update (channel.f:1055-1065),
 * and COURANT at rk_step 3 when variable_dt and mod(time_step,update_dt)==0
 * (channel.f:1037-1040).  h_bar/beta_bar/zeta_bar are /RKW3_PARAMS/
 * (for/header:173-174).  delta_t and h_bar are updated in place when
 * COURANT runs, exactly as courant.f:49-62 updates DELTA_T and H_BAR.
 * With p.les set (LES_MODEL_TYPE 1, FP64) the substage includes the
 * constant-Smagorinsky branch (for/les.f:1-336, channel.f:303-384 and the
 * eddy-viscosity terms) once LES and (not CREATE_NEW_FLOW or
 * time_step > 100), and then solves the CN systems per physical column as
 * the reference does. */
int diablo_gpu_rk_chan_1(void* handle, int rk_step, int time_step, double time,
                         double* delta_t, double* h_bar, const double* beta_bar,
                         const double* zeta_bar);
/* NU_T(0:NX+1,0:NZP+1,0:NY+1) of COMMON /LES_VARS/ (for/header:164-168) in
 * the host physical layout (entries with I >= NX or K >= NZ untouched): the
 * eddy viscosity at GY points of the last LES substage, zero before the
 * first.  DIABLO_EINVAL without LES. */
int diablo_gpu_download_nu_t(void* handle, double* nu_t);
/* RK_CHAN_2 (for/channel.f:1076-1100) is a stub in the reference that prints
 * "not supported" and stops; this returns DIABLO_ENOTSUP. */
int diablo_gpu_rk_chan_2(void* handle);

/* FFT_XZ_TO_FOURIER(V,VV,JMIN,JMAX) (for/mpi.f:1477-1542) on host arrays:
 * v is a physical array, vv a Fourier array; planes jmin..jmax. */
int diablo_gpu_fft_xz_to_fourier(void* handle, const double* v, double* vv,
                                 int jmin, int jmax);
/* FFT_XZ_TO_PHYSICAL(VV,V,JMIN,JMAX) (for/mpi.f:1547-1606) on host arrays. */
int diablo_gpu_fft_xz_to_physical(void* handle, const double* vv, double* v,
                                  int jmin, int jmax);

/* REM_DIV_CHAN (for/channel.f:1103-1214) on the device state; phi is kept
 * on the device and returned by diablo_gpu_download_phi. */
int diablo_gpu_rem_div_chan(void* handle);
int diablo_gpu_download_phi(void* handle, double* phi);
/* POISSON_P_CHAN (for/channel.f:1217-1453) on the device state (CU -> CP). */
int diablo_gpu_poisson_p_chan(void* handle);
/* APPLY_BC_VEL_MPI (for/mpi.f:1317-1331) on the device state. */
int diablo_gpu_apply_bc_vel(void* handle);
/* COURANT (for/courant.f:1-66) on the device state's physical velocity. */
int diablo_gpu_courant(void* handle, double* delta_t, double* h_bar);

/* Plane statistics of SAVE_STATS_CHAN (for/save_stats.f:104-347,452-536) in
 * FP64 for the current state.  profiles receives DIABLO_NSTATS*(NY+2)
 * doubles, profile s at [s*(NY+2) + j]; see DIABLO_STAT_* for s. */
#define DIABLO_STAT_UME     0
#define DIABLO_STAT_VME     1
#define DIABLO_STAT_WME     2
#define DIABLO_STAT_URMS    3
#define DIABLO_STAT_VRMS    4
#define DIABLO_STAT_WRMS    5
#define DIABLO_STAT_UV      6
#define DIABLO_STAT_UW      7
#define DIABLO_STAT_WV      8
#define DIABLO_STAT_DUDY    9
#define DIABLO_STAT_DWDY   10
#define DIABLO_STAT_CP     11
#define DIABLO_STAT_SHEAR  12
#define DIABLO_STAT_THME   13   /* scalar 1 */
#define DIABLO_STAT_DTHDY  14
#define DIABLO_STAT_THRMS  15
#define DIABLO_STAT_THV    16
#define DIABLO_NSTATS      17
int diablo_gpu_stats(void* handle, double* profiles);

/* Every profile SAVE_STATS_CHAN writes to mean.h5 and tke.h5
 * (for/save_stats.f:104-536, 937-1135), in FP64, for the current state
 * (after APPLY_BC_VEL, as the reference does).
 *  chan:    DIABLO_NMEAN*(NY+2) doubles: profiles 0..12 as DIABLO_STAT_UME..
 *           DIABLO_STAT_SHEAR, then the rms vorticity components omega_x,
 *           omega_y, omega_z (save_stats.f:270-347), rows 1..NY.
 *  scal:    N_TH*DIABLO_NSCAL*(NY+2) doubles (may be null when N_TH = 0):
 *           per scalar n, thme, dthdy, thrms, thv and pe_diss (the mean
 *           square scalar gradient, save_stats.f:465-536) at
 *           [(n*DIABLO_NSCAL + s)*(NY+2) + j].
 *  epsilon: NY+2 doubles or null: the pseudo-dissipation of tkebudget_chan
 *           (save_stats.f:937-1135), NU <du_i/dx_j du_i/dx_j>, on rows
 *           2..NY-1.  Rows 1 and NY are 0: there the reference's value
 *           depends on work-array contents left by earlier calls.
 * The reference's mean.h5 stores omega_y in the omega_z dataset
 * (save_stats.f:421-423); this entry returns the true omega_z and leaves
 * that choice to the writer.  Replaces the statistics part of
 * SAVE_STATS_CHAN; its HDF5 writes stay on the host. */
#define DIABLO_MEAN_OMEGA_X 13
#define DIABLO_MEAN_OMEGA_Y 14
#define DIABLO_MEAN_OMEGA_Z 15
#define DIABLO_NMEAN        16
#define DIABLO_SCAL_THME     0
#define DIABLO_SCAL_DTHDY    1
#define DIABLO_SCAL_THRMS    2
#define DIABLO_SCAL_THV      3
#define DIABLO_SCAL_PE_DISS  4
#define DIABLO_NSCAL         5
int diablo_gpu_mean_stats(void* handle, double* chan, double* scal, double* epsilon);

/* USER_RHS_CHAN_FOURIER and USER_RHS_CHAN_PHYSICAL (for/user_rhs.f:1-122),
 * which RK_CHAN_1 calls at for/channel.f:297 and :578 so that a user can
 * add terms to the right-hand sides CF1..CF3, CFTH (empty in the reference).
 * Here the user's host callback gets device pointers and the handle's stream
 * and writes the terms to add; the library adds them to CF in every substage,
 * where the reference forms CF (rows JSTART..JEND, CF2 rows 2..NY).  Nothing
 * of this runs while no callback is set.
 *  DIABLO_USER_RHS_FOURIER:  cu holds CU1..CU3, CTH(1..N_TH) at the start of
 *    the substage; write Fourier-space terms into cf_add (zeroed).
 *  DIABLO_USER_RHS_PHYSICAL: u holds U1..U3, TH(1..N_TH) in physical space
 *    (planes 0..NY+1); write physical-space terms into f_add (zeroed); the
 *    library transforms them with FFT_XZ_TO_FOURIER and adds them to CF,
 *    the pattern of user_rhs.f:14-40.
 * Device layouts, FP64: Fourier field f, plane J, packed kz row m (0..TNKZ),
 * kx (0..NKX) is the complex element f*s_field + J*s_plane + m*s_row + kx
 * (interleaved re, im); physical field f, plane J, z, x is the double
 * f*p_field + J*p_plane + z*NX + x.  The callback enqueues its work on
 * `stream` (a cudaStream_t) or finishes it before returning.  In FP32-split
 * mode the Fourier-space terms join the nonlinear term and are rounded to
 * FP32 with it.  fn = NULL removes the hook.  No counterpart in the
 * reference's interface beyond the two subroutines; batched handles reject
 * hooks. */
typedef struct diablo_user_rhs_args {
    int rk_step, time_step;
    double time;
    int nx, ny, nz, n_th, nkx, tnkz;
    long long s_field, s_plane, s_row;    /* complex elements */
    long long p_field, p_plane;           /* doubles */
    const double* cu;
    double* cf_add;
    const double* u;                      /* physical hook only, else NULL */
    double* f_add;                        /* physical hook only, else NULL */
    void* stream;
} diablo_user_rhs_args;
typedef void (*diablo_user_rhs_fn)(void* user, const diablo_user_rhs_args* args);
#define DIABLO_USER_RHS_FOURIER  0
#define DIABLO_USER_RHS_PHYSICAL 1
int diablo_gpu_set_user_rhs(void* handle, int kind, diablo_user_rhs_fn fn, void* user);

/* The CUDA stream (a cudaStream_t) all work of the handle is queued on, as
 * an opaque pointer: callers may record timing events on it. */
int diablo_gpu_get_stream(void* handle, void** stream);
/* Kernel timing: with profiling on, every library launch is bracketed by
 * CUDA events on the handle's stream.  diablo_gpu_kernel_times waits for the
 * stream, then returns per kernel kind the number of launches and the summed
 * device time in ms since profiling was switched on (and restarts the
 * count).  Kinds: DIABLO_KERNEL_*; arrays hold DIABLO_NKERNELS entries. */
#define DIABLO_KERNEL_ZINV      0   /* inverse z transform of the state */
#define DIABLO_KERNEL_PRODUCTS  1   /* x transforms + nonlinear products */
#define DIABLO_KERNEL_ZFWD_NL   2   /* forward z transform + derivative combination */
#define DIABLO_KERNEL_CN_COEF   3   /* CN tridiagonal factors */
#define DIABLO_KERNEL_COLUMN    4   /* CN solves + projection + pressure update */
#define DIABLO_KERNEL_REMDIV    5   /* stand-alone projection */
#define DIABLO_KERNEL_CFL       6   /* CFL minimum */
#define DIABLO_KERNEL_OTHER     7   /* transform API, BCs, statistics */
#define DIABLO_NKERNELS         8
int diablo_gpu_set_profiling(void* handle, int on);
int diablo_gpu_kernel_times(void* handle, long long* launches, double* ms);

/* REM_DIV_CHAN for callers that cannot allocate device memory.  This entry
 * point has no counterpart in the reference: it exists for hosts that keep
 * CU1, CU2, CU3 in device memory they obtained themselves (OpenACC or CUDA
 * Fortran device arrays, a framework's memory pool) and cannot let a library
 * call cudaMalloc, because that memory is managed by the host's runtime or
 * pool and a second allocator would bypass it.  It allocates nothing: it
 * queues two small host-to-device copies of the grid metrics and one kernel
 * on `stream` (a cudaStream_t, NULL for the default stream) and keeps its
 * working storage in an 8 MiB array of static device memory that every GPU
 * loading this library holds until exit.
 *   p        sizes and LX, LZ (other fields unused)
 *   dy, dyf  HOST pointers to DY(0:NY+1), DYF(0:NY+1); pageable memory is
 *            read before the call returns, page-locked memory when the copy
 *            runs on `stream`, so keep it unchanged until then
 *   cu1..3   DEVICE pointers, Fortran layout (0:NXP,0:NZ+1,0:NY+1) complex;
 *            projected in place (dealiased block, J = 1..NY)
 *   phi      DEVICE pointer, same layout; receives phi on J = 1..NY
 * Limit: (NX/3+1)*(2*(NZ/3)+1)*(NY+2) + 2*(NY+2) <= 2^20, else
 * DIABLO_EINVAL.  The first call on a device looks up the static array's
 * address (cudaGetSymbolAddress); make that first call before any stream
 * capture.  All calls share the array: calls that may overlap on the GPU
 * race and must be serialised by the caller. */
int diablo_gpu_rem_div_chan_noalloc(const diablo_params* p, const double* dy, const double* dyf,
                                    double* cu1, double* cu2, double* cu3, double* phi,
                                    void* stream);

/* filter_chan(n) (for/filter.f:1-98) on the device scalar n (1..N_TH): the
 * sharpened raised-cosine filter in kx,kz on rows J = 0..NY and, for
 * I >= 1, K >= 1, the vertical compact filter with alpha = 0 (an explicit
 * 5-point stencil on J = 2..NY-1).  Row J = 0 keeps its horizontally
 * filtered value, where the reference copies an element of its work array
 * that it never sets. */
int diablo_gpu_filter_chan(void* handle, int n);

/* Launch shapes chosen by timing (no counterpart in the reference, which
 * has no GPU code): planes per block of the products and z-forward kernels.
 * Runs a few RK substages of the instance's own grid with each candidate and
 * restores the state afterwards; the result of a step does not depend on the
 * choice (the same arithmetic, only grouped differently).  prod_chunk and
 * zf_planes receive the chosen values (either may be NULL).  Allocates a
 * temporary copy of the state. */
int diablo_gpu_autotune(void* handle, int* prod_chunk, int* zf_planes);

/* nsteps RK3 steps (the three RK_CHAN_1 substages each, as in diablo.f:66-111
 * without statistics or I/O) of one instance, replayed from one CUDA graph of
 * a whole step.  Small grids spend most of a step launching kernels; the
 * graph launches a step at once.  No counterpart in the reference, whose time
 * loop calls the substages one by one.  The step must be static: VARIABLE_DT
 * 0, F_TYPE != 2, no user right-hand side, profiling off and, on the LES
 * branch, the subgrid model running (after the CREATE_NEW_FLOW spin-up of
 * 100 steps); otherwise DIABLO_ENOTSUP and the caller steps with
 * diablo_gpu_rk_chan_1.  h_bar, beta_bar, zeta_bar are the substage
 * coefficients of the fixed time step; time_step is the number of the step
 * before the first one taken.  The first call, and any call after a change of
 * the coefficients, of diablo_gpu_autotune's launch shapes or of the attached
 * network, runs one step directly and captures the next; later calls only
 * launch the graph.  Asynchronous on the handle's stream (diablo_gpu_synchronize
 * waits and reports DIABLO_ENAN).  The results equal nsteps calls of the
 * three substages. */
int diablo_gpu_step_graph(void* handle, int nsteps, int time_step, const double* h_bar, const double* beta_bar,
                          const double* zeta_bar);

/* Batched instances (configuration of many independent channels of uneven
 * sizes; the reference's ensemble driver, dummy_code/ensem_dummy.f, is an
 * empty stub).  diablo_gpu_batch_create captures one full RK3 step (the three
 * RK_CHAN_1 substages) of every handle into one CUDA graph, one stream branch
 * per instance, with the fixed time step delta_t[i] of instance i; each
 * diablo_gpu_batch_step then advances every instance by nsteps steps, one
 * graph launch per step.  Every instance must have variable_dt = 0 and no
 * time-dependent forcing (f_type != 2), else DIABLO_ENOTSUP.  The handles
 * stay owned by the caller and must outlive the batch; while the batch
 * exists, calls on its handles other than upload/download/synchronize are
 * not allowed to overlap a batch step. */
int diablo_gpu_batch_create(void* const* handles, const double* delta_t, int n, void** batch);
int diablo_gpu_batch_step(void* batch, int nsteps);
int diablo_gpu_batch_destroy(void* batch);

/* Wait for all work queued on the handle's stream. */
int diablo_gpu_synchronize(void* handle);
/* Sum over the last launches of the handle: number of kernels launched by
 * the library since creation (the counter is cumulative). */
long long diablo_gpu_kernel_launches(void* handle);
/* Short description of the last error on this thread. */
const char* diablo_gpu_last_error(void);

/* ------------------------------------------------------------------------ */
/* Learned subgrid-stress closure.  The reference has no counterpart: it is   */
/* this library's MLP from the 9 resolved velocity gradients du_i/dx_j        */
/* (i-major, divided by their norm G), the wall distance in viscous units y+  */
/* and the filter width Delta to the 6 stresses (tau_11, tau_22, tau_33,      */
/* tau_12, tau_13, tau_23) divided by Delta^2 G^2, through 3 hidden layers   */
/* of 64 GELU units (tanh form).  Weights and activations are BF16 on the     */
/* tensor cores with FP32 accumulation; parameters, gradients and the Adam    */
/* state are FP32 on the device.                                              */
/*                                                                            */
/* Parameter vector (DIABLO_MLP_NPARAM floats): W1[64][11] b1[64] W2[64][64]  */
/* b2[64] W3[64][64] b3[64] W4[6][64] b4[6] (the DIABLO_MLP_NTRAIN trained    */
/* entries), then input means [11], input scales [11] and output scales [6]:  */
/* the network maps (x - mean)/scale to tau / out_scale.                      */
/* ------------------------------------------------------------------------ */
#define DIABLO_MLP_NIN 11
#define DIABLO_MLP_NHIDDEN 64
#define DIABLO_MLP_NOUT 6
#define DIABLO_MLP_NTRAIN 9478
#define DIABLO_MLP_NPARAM 9506
int diablo_mlp_create(void** mlp);
int diablo_mlp_destroy(void* mlp);
/* Set all parameters (scales must be non-zero); resets the Adam state. */
int diablo_mlp_set_params(void* mlp, const float* params);
int diablo_mlp_get_params(void* mlp, float* params);
/* x: host [n][11] features; y: host [n][6] outputs (dimensionless stresses
 * in the closure's use). */
int diablo_mlp_forward(void* mlp, const float* x, long long n, float* y);
/* Loss sum_samples sum_outputs (y/out_scale - t/out_scale)^2 / (2n) and its
 * gradient with respect to the DIABLO_MLP_NTRAIN trained parameters.  With a
 * dissipation weight w (diablo_mlp_set_dissipation_weight, default 0) the
 * loss adds w/(2n) sum_samples (Pi(y) - Pi(t))^2, Pi(tau) = -sum_ij tau_ij
 * S_ij the subgrid dissipation of the dimensionless stresses, S_ij the
 * symmetric part of the sample's gradient features x[0..8] (g_ij, i-major):
 * it trains the network to transfer the right energy between the resolved
 * and subgrid scales, not only to match the stresses. */
int diablo_mlp_gradient(void* mlp, const float* x, const float* t, long long n, double* loss, float* grad);
/* Weight w >= 0 of the dissipation term of the loss (used by
 * diablo_mlp_gradient and diablo_mlp_train).  No counterpart in the
 * reference, like the rest of the closure. */
int diablo_mlp_set_dissipation_weight(void* mlp, float weight);
/* steps Adam steps (beta 0.9, 0.999, eps 1e-8, learning rate lr) on
 * consecutive mini-batches of `batch` samples, cycling through the n
 * samples as given (the caller shuffles); losses[s] (may be NULL) receives
 * each step's mini-batch loss before its update. */
int diablo_mlp_train(void* mlp, const float* x, const float* t, long long n, int batch, int steps, float lr,
                     double* losses);
/* Training samples from a channel instance's current state (the reference
 * has no counterpart): a width x width top-hat filter in x and z (periodic,
 * width odd) of the velocity, at GYF points J = 2..NY-1 and every stride-th
 * x and z point, J-major then z then x.  With g_ij = d ubar_i/dx_j
 * (i-major), G = |g| and Delta = (width DX DYF(J) width DZ)^(1/3):
 * x receives [n][11] features (g_ij / G, y+, Delta), scale [n] the stress
 * scale s = Delta^2 G^2 and t [n][6] the targets tau_ij / s, tau_ij =
 * bar(u_i u_j) - ubar_i ubar_j (11, 22, 33, 12, 13, 23); the closure's
 * network works in this dimensionless form.  n = (NY-2) ceil(NX/stride)
 * ceil(NZ/stride) is written to *n; arrays shorter than that (capacity
 * samples) give DIABLO_EINVAL with *n set. */
int diablo_gpu_sgs_samples(void* handle, int width, int stride, float* x, float* t, float* scale,
                           long long capacity, long long* n);
/* Attach a closure network to an LES instance (NULL detaches; the caller
 * keeps ownership and must not change its parameters while a substage that
 * uses it runs).  With LES_MODEL_TYPE 4, each LES substage then computes the
 * features of the resolved field (width 1, every point of rows 2..NY-1, as
 * diablo_gpu_sgs_samples), the network's outputs times Delta^2 G^2 as the
 * stresses, tau_12 and tau_23 interpolated to GY points, and
 * CF_i -= d tau_ij / dx_j explicitly, in place of the eddy-viscosity model
 * (NU_T stays zero); without a network type 4 runs the dynamic model.  The
 * reference has no counterpart. */
int diablo_gpu_set_sgs_mlp(void* handle, void* mlp);

#ifdef __cplusplus
}
#endif
#endif /* DIABLO_GPU_H */
