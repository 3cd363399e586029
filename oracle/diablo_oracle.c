/*
 * diablo_oracle.c -- CPU FP64 restatement of DIABLO's channel timestep.
 *
 * TEST INFRASTRUCTURE ONLY (see diablo_oracle.h): the checker for the GPU
 * library, never linked into it.  Each routine cites the reference routine
 * it restates; the loop structure, ranges, aliasing and in-place updates
 * follow the reference's NPROCY = NPROCZ = 1 MPI build so that round-off
 * aside the oracle produces the reference's numbers.
 */
#include "diablo_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

/* ------------------------------------------------------------------------ */
/* FFT: mixed-radix (2,3,4,5,8) self-sorting Stockham transform, FP64.        */
/* Restates the DFT that FFTW 3.3.10 computes (fft.f:73-89 plans,             */
/* mpi.f:1494,1528,1575,1602 executions): X_k = sum_j x_j exp(s 2 pi i jk/n). */
/* ------------------------------------------------------------------------ */
typedef struct {
    int n, nr, radix[40];
    cplx* w;          /* w[k] = exp(-2 pi i k / n) */
} fftplan;

static int plan_init(fftplan* P, int n) {
    P->n = n;
    P->nr = 0;
    int m = n;
    const int rads[5] = {8, 4, 2, 3, 5};
    for (int q = 0; q < 5; ++q)
        while (m % rads[q] == 0) { P->radix[P->nr++] = rads[q]; m /= rads[q]; }
    if (m != 1) return -1;
    P->w = (cplx*)malloc(sizeof(cplx) * (size_t)n);
    const double pi = 4.0 * atan(1.0);
    for (int k = 0; k < n; ++k) {
        double a = -2.0 * pi * (double)k / (double)n;
        P->w[k] = cos(a) + I * sin(a);
    }
    return 0;
}
static void plan_free(fftplan* P) { free(P->w); P->w = NULL; }

/* In-place transform of x (length n, contiguous); work has n entries. */
static void cfft(const fftplan* P, cplx* x, cplx* work, int sign) {
    const int n = P->n;
    cplx* d0 = x;
    cplx* d1 = work;
    int Ns = 1;
    for (int s = 0; s < P->nr; ++s) {
        const int R = P->radix[s];
        const int nR = n / R;
        const int tw = n / (Ns * R);      /* table step for the stage twiddle */
        const int rw = n / R;             /* table step for the radix-R kernel */
        for (int j = 0; j < nR; ++j) {
            cplx v[8], V[8];
            const int k = j % Ns;
            for (int r = 0; r < R; ++r) {
                cplx t = P->w[(k * r * tw) % n];
                if (sign > 0) t = conj(t);
                v[r] = d0[j + r * nR] * t;
            }
            for (int p = 0; p < R; ++p) {
                cplx acc = 0;
                for (int q = 0; q < R; ++q) {
                    cplx t = P->w[((p * q) % R) * rw];
                    if (sign > 0) t = conj(t);
                    acc += v[q] * t;
                }
                V[p] = acc;
            }
            const int idxD = (j / Ns) * Ns * R + k;
            for (int r = 0; r < R; ++r) d1[idxD + r * Ns] = V[r];
        }
        cplx* t = d0; d0 = d1; d1 = t;
        Ns *= R;
    }
    if (d0 != x) memcpy(x, d0, sizeof(cplx) * (size_t)n);
}

int orc_cdft(int n, double* data, int sign) {
    fftplan P;
    if (plan_init(&P, n)) return -1;
    cplx* work = (cplx*)malloc(sizeof(cplx) * (size_t)n);
    cfft(&P, (cplx*)data, work, sign);
    free(work);
    plan_free(&P);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* State: the COMMON blocks that the channel timestep touches.               */
/* ------------------------------------------------------------------------ */
struct orc_state {
    diablo_params p;
    int NX, NY, NZ, NTH, NXP, NZP, NKX, NKZ, TNKZ, NXM;
    int px, pz;           /* physical leading dims: NX+2, NZP+2 */
    int cx, cz;           /* complex leading dims: NXP+1, NZ+2 */
    size_t nreal;         /* doubles per 3-D field */
    double PI;
    double *GY, *GYF, *DY, *DYF;      /* 0..NY+1 */
    double DX, DZ;
    double *KX, *KX2, *KZ, *KZ2;      /* 0..NXP, 0..TNKZ */
    double H_BAR[3], BETA_BAR[3], ZETA_BAR[3];
    double DELTA_T, TIME;
    int TIME_STEP, RK_STEP;
    int JSTART, JEND, JSTART_TH[DIABLO_MAX_TH], JEND_TH[DIABLO_MAX_TH];
    /* EQUIVALENCE'd pairs share one buffer: U1<->CU1 etc. (header:245-255) */
    double *U1, *U2, *U3, *P, *R1, *R2, *R3, *F1, *F2, *F3, *S1;
    /* not equivalenced (header:256-258) */
    double *TH, *CTH, *FTH, *CFTH, *RTH, *CRTH;
    /* LES (allocated when p.les): NU_T at GY points, which also serves as
     * KAPPA_T (channel.f:314-322 copies it for every scalar); Sij<->CSij and
     * TEMP<->CTEMP share one buffer each as header_les:31-37 equivalences them */
    double *NU_T, *SIJ[6], *TEMP;
    float* MLP;           /* learned closure parameters (LES_MODEL_TYPE 4), or NULL */
    /* USER_RHS_CHAN_FOURIER / _PHYSICAL: called with the state as the
     * reference's user routines see it, or NULL (the reference's empty ones) */
    void (*user_fn[2])(void*);
    void* user_data[2];
    fftplan px_plan, pz_plan;
};

#define PH(a, i, k, j) ((a)[(size_t)(i) + (size_t)s->px * ((size_t)(k) + (size_t)s->pz * (size_t)(j))])
#define CX(a, i, k, j) (((cplx*)(a))[(size_t)(i) + (size_t)s->cx * ((size_t)(k) + (size_t)s->cz * (size_t)(j))])

static int g_threads = 0;
void orc_set_threads(int n) { g_threads = n; }
static int nthreads(void) {
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

orc_state* orc_create(const diablo_params* p, const double* gy, const double* gyf,
                      double delta_t) {
    orc_state* s = (orc_state*)calloc(1, sizeof(orc_state));
    s->p = *p;
    s->NX = p->nx; s->NY = p->ny; s->NZ = p->nz; s->NTH = p->n_th;
    s->NXP = p->nx / 2; s->NZP = p->nz;
    s->NKX = p->nx / 3; s->NKZ = p->nz / 3; s->TNKZ = 2 * s->NKZ;
    s->NXM = p->nx - 1;
    s->px = s->NX + 2; s->pz = s->NZP + 2;
    s->cx = s->NXP + 1; s->cz = s->NZ + 2;
    s->nreal = (size_t)s->px * s->pz * (s->NY + 2);
    s->PI = 4.0 * atan(1.0);
    if (plan_init(&s->px_plan, s->NX) || plan_init(&s->pz_plan, s->NZ)) {
        free(s);
        return NULL;
    }
    const int NY = s->NY;
    s->GY = (double*)calloc(NY + 2, sizeof(double));
    s->GYF = (double*)calloc(NY + 2, sizeof(double));
    s->DY = (double*)calloc(NY + 2, sizeof(double));
    s->DYF = (double*)calloc(NY + 2, sizeof(double));
    memcpy(s->GY, gy, sizeof(double) * (NY + 2));
    memcpy(s->GYF, gyf, sizeof(double) * (NY + 2));
    /* CREATE_GRID_CHAN grid spacing (channel.f:1566-1578, 1646-1652) */
    s->DX = p->lx / s->NX;
    s->DZ = p->lz / s->NZ;
    for (int j = 1; j <= NY + 1; ++j) s->DY[j] = s->GYF[j] - s->GYF[j - 1];
    for (int j = 1; j <= NY; ++j) s->DYF[j] = s->GY[j + 1] - s->GY[j];
    s->DYF[NY + 1] = s->DYF[NY];
    /* INIT_FFT wavenumbers (fft.f:77-100); NXPP = NXP for NPROCZ = 1 */
    s->KX = (double*)calloc(s->NXP + 1, sizeof(double));
    s->KX2 = (double*)calloc(s->NXP + 1, sizeof(double));
    s->KZ = (double*)calloc(s->TNKZ + 1, sizeof(double));
    s->KZ2 = (double*)calloc(s->TNKZ + 1, sizeof(double));
    for (int i = 0; i <= s->NXP - 1; ++i) {
        s->KX[i] = (double)i * (2.0 * s->PI) / p->lx;
        s->KX2[i] = s->KX[i] * s->KX[i];
    }
    for (int k = 0; k <= s->NKZ; ++k) s->KZ[k] = (double)k * (2.0 * s->PI) / p->lz;
    for (int k = 1; k <= s->NKZ; ++k) s->KZ[s->TNKZ + 1 - k] = -(double)k * (2.0 * s->PI) / p->lz;
    for (int k = 0; k <= s->TNKZ; ++k) s->KZ2[k] = s->KZ[k] * s->KZ[k];
    /* INIT_CHAN_MPI, RANKY = 0 branch (mpi.f:1024-1044): with NPROCY = 1 the
     * first branch is taken, so JEND = NY and JSTART = 2 whatever the BCs. */
    s->JSTART = 2;
    s->JEND = NY;
    for (int n = 0; n < s->NTH; ++n) {
        s->JEND_TH[n] = NY;
        s->JSTART_TH[n] = (p->th_bc_ymin[n] == 1) ? 1 : 2;
    }
    /* RK coefficients (diablo_io.f:116-124) */
    s->DELTA_T = delta_t;
    s->H_BAR[0] = delta_t * (8.0 / 15.0);
    s->H_BAR[1] = delta_t * (2.0 / 15.0);
    s->H_BAR[2] = delta_t * (5.0 / 15.0);
    s->BETA_BAR[0] = 1.0; s->BETA_BAR[1] = 25.0 / 8.0; s->BETA_BAR[2] = 9.0 / 4.0;
    s->ZETA_BAR[0] = 0.0; s->ZETA_BAR[1] = -17.0 / 8.0; s->ZETA_BAR[2] = -5.0 / 4.0;
    s->TIME = 0.0;
    s->TIME_STEP = 0;
    double** fields[11] = {&s->U1, &s->U2, &s->U3, &s->P, &s->R1, &s->R2, &s->R3,
                           &s->F1, &s->F2, &s->F3, &s->S1};
    for (int f = 0; f < 11; ++f) *fields[f] = (double*)calloc(s->nreal, sizeof(double));
    size_t nth = (size_t)(s->NTH > 0 ? s->NTH : 1);
    s->TH = (double*)calloc(s->nreal * nth, sizeof(double));
    s->CTH = (double*)calloc(s->nreal * nth, sizeof(double));
    s->FTH = (double*)calloc(s->nreal * nth, sizeof(double));
    s->CFTH = (double*)calloc(s->nreal * nth, sizeof(double));
    s->RTH = (double*)calloc(s->nreal * nth, sizeof(double));
    s->CRTH = (double*)calloc(s->nreal * nth, sizeof(double));
    if (p->les) {
        s->NU_T = (double*)calloc(s->nreal, sizeof(double));
        s->TEMP = (double*)calloc(s->nreal, sizeof(double));
        for (int q = 0; q < 6; ++q) s->SIJ[q] = (double*)calloc(s->nreal, sizeof(double));
    }
    return s;
}

void orc_destroy(orc_state* s) {
    if (!s) return;
    double* bufs[] = {s->GY, s->GYF, s->DY, s->DYF, s->KX, s->KX2, s->KZ, s->KZ2,
                      s->U1, s->U2, s->U3, s->P, s->R1, s->R2, s->R3, s->F1, s->F2,
                      s->F3, s->S1, s->TH, s->CTH, s->FTH, s->CFTH, s->RTH, s->CRTH,
                      s->NU_T, s->TEMP, s->SIJ[0], s->SIJ[1], s->SIJ[2], s->SIJ[3], s->SIJ[4],
                      s->SIJ[5], NULL};
    free(s->MLP);
    for (size_t q = 0; q < sizeof(bufs) / sizeof(bufs[0]); ++q) free(bufs[q]);
    plan_free(&s->px_plan);
    plan_free(&s->pz_plan);
    free(s);
}

double* orc_array(orc_state* s, int which) {
    switch (which) {
        case ORC_U1: return s->U1;   case ORC_U2: return s->U2;
        case ORC_U3: return s->U3;   case ORC_P: return s->P;
        case ORC_R1: return s->R1;   case ORC_R2: return s->R2;
        case ORC_R3: return s->R3;   case ORC_F1: return s->F1;
        case ORC_F2: return s->F2;   case ORC_F3: return s->F3;
        case ORC_S1: return s->S1;   case ORC_TH: return s->TH;
        case ORC_CTH: return s->CTH; case ORC_FTH: return s->FTH;
        case ORC_CFTH: return s->CFTH; case ORC_RTH: return s->RTH;
        case ORC_CRTH: return s->CRTH; case ORC_GY: return s->GY;
        case ORC_GYF: return s->GYF; case ORC_DY: return s->DY;
        case ORC_DYF: return s->DYF; case ORC_KX: return s->KX;
        case ORC_KZ: return s->KZ;
        case ORC_NU_T: return s->NU_T;
    }
    return NULL;
}

size_t orc_array_doubles(orc_state* s, int which) {
    if (which <= ORC_S1) return s->nreal;
    if (which <= ORC_CRTH) return s->nreal * (size_t)(s->NTH > 0 ? s->NTH : 1);
    if (which <= ORC_DYF) return (size_t)s->NY + 2;
    if (which == ORC_KX) return (size_t)s->NXP + 1;
    if (which == ORC_KZ) return (size_t)s->TNKZ + 1;
    if (which == ORC_NU_T) return s->NU_T ? s->nreal : 0;
    return 0;
}

void orc_get_time(orc_state* s, double* time, double* delta_t, int* time_step,
                  double* h_bar) {
    if (time) *time = s->TIME;
    if (delta_t) *delta_t = s->DELTA_T;
    if (time_step) *time_step = s->TIME_STEP;
    if (h_bar) memcpy(h_bar, s->H_BAR, sizeof(s->H_BAR));
}

void orc_set_time(orc_state* s, double time, double delta_t, int time_step) {
    s->TIME = time;
    s->TIME_STEP = time_step;
    s->DELTA_T = delta_t;
    s->H_BAR[0] = delta_t * (8.0 / 15.0);
    s->H_BAR[1] = delta_t * (2.0 / 15.0);
    s->H_BAR[2] = delta_t * (5.0 / 15.0);
}

/* ------------------------------------------------------------------------ */
/* FFT_XZ_TO_FOURIER (mpi.f:1477-1542) with NPROCZ = 1: the all-to-all is a  */
/* plain copy.  V and VV may alias (EQUIVALENCE), so the x transforms of all */
/* planes finish before VV is written, as in the reference.                  */
/* ------------------------------------------------------------------------ */
void orc_fft_xz_to_fourier(orc_state* s, double* V, double* VVd, int jmin, int jmax) {
    const int NX = s->NX, NZ = s->NZ, NZP = s->NZP, NXP = s->NXP;
    const int NKX = s->NKX, NKZ = s->NKZ;
    const int nh = NX / 2 + 1;
    const int nplanes = jmax - jmin + 1;
    if (nplanes <= 0) return;
    /* TMP(0:NX/2, 0:NZP-1, JMIN:JMAX) */
    cplx* TMP = (cplx*)malloc(sizeof(cplx) * (size_t)nh * NZP * nplanes);
#pragma omp parallel num_threads(nthreads())
    {
        cplx* row = (cplx*)malloc(sizeof(cplx) * NX);
        cplx* work = (cplx*)malloc(sizeof(cplx) * NX);
#pragma omp for collapse(2) schedule(static)
        for (int j = jmin; j <= jmax; ++j)
            for (int k = 0; k < NZP; ++k) {
                for (int i = 0; i < NX; ++i) row[i] = PH(V, i, k, j);
                cfft(&s->px_plan, row, work, -1);
                cplx* t = TMP + ((size_t)(j - jmin) * NZP + k) * nh;
                for (int i = 0; i <= NKX; ++i) t[i] = row[i] / NX;
                for (int i = NKX + 1; i <= NX / 2; ++i) t[i] = 0.0;
            }
        free(row);
        free(work);
    }
    cplx* VV = (cplx*)VVd;
    (void)VV;
#pragma omp parallel num_threads(nthreads())
    {
        cplx* col = (cplx*)malloc(sizeof(cplx) * NZ);
        cplx* work = (cplx*)malloc(sizeof(cplx) * NZ);
#pragma omp for schedule(static)
        for (int j = jmin; j <= jmax; ++j) {
            /* all-to-all copy: TMP2(I,K)=TMP_1A(I,K,J), I<NXP, K<NZ */
            for (int k = 0; k <= NZ - 1; ++k) {
                const cplx* t = TMP + ((size_t)(j - jmin) * NZP + k) * nh;
                for (int i = 0; i <= NXP - 1; ++i) CX(VVd, i, k, j) = t[i];
                CX(VVd, NXP, k, j) = 0.0;
            }
            for (int k = NZ; k <= NZ + 1; ++k)
                for (int i = 0; i <= NXP; ++i) CX(VVd, i, k, j) = 0.0;
            /* z transform (howmany NXP, stride NXP+1), forward */
            for (int i = 0; i <= NXP - 1; ++i) {
                for (int k = 0; k < NZ; ++k) col[k] = CX(VVd, i, k, j);
                cfft(&s->pz_plan, col, work, -1);
                for (int k = 0; k < NZ; ++k) CX(VVd, i, k, j) = col[k];
            }
            for (int k = 0; k <= NKZ; ++k)
                for (int i = 0; i <= NXP; ++i) CX(VVd, i, k, j) = CX(VVd, i, k, j) / NZ;
            for (int k = 1; k <= NKZ; ++k)
                for (int i = 0; i <= NXP; ++i)
                    CX(VVd, i, NKZ + k, j) = CX(VVd, i, NZ - 1 + k - NKZ, j) / NZ;
        }
        free(col);
        free(work);
    }
    free(TMP);
}

/* FFT_XZ_TO_PHYSICAL (mpi.f:1547-1606).  The kz unpacking happens in place
 * on the input array, as in the reference. */
void orc_fft_xz_to_physical(orc_state* s, double* VVd, double* V, int jmin, int jmax) {
    const int NX = s->NX, NZ = s->NZ, NZP = s->NZP, NXP = s->NXP;
    const int NKZ = s->NKZ;
    const int nh = NX / 2 + 1;
    const int nplanes = jmax - jmin + 1;
    if (nplanes <= 0) return;
    cplx* TMP = (cplx*)malloc(sizeof(cplx) * (size_t)nh * NZP * nplanes);
#pragma omp parallel num_threads(nthreads())
    {
        cplx* col = (cplx*)malloc(sizeof(cplx) * NZ);
        cplx* work = (cplx*)malloc(sizeof(cplx) * NZ);
#pragma omp for schedule(static)
        for (int j = jmin; j <= jmax; ++j) {
            for (int k = NKZ; k >= 1; --k)
                for (int i = 0; i <= NXP; ++i)
                    CX(VVd, i, NZ - 1 + k - NKZ, j) = CX(VVd, i, NKZ + k, j);
            for (int k = NKZ + 1; k <= NZ - NKZ - 1; ++k)
                for (int i = 0; i <= NXP; ++i) CX(VVd, i, k, j) = 0.0;
            for (int i = 0; i <= NXP - 1; ++i) {
                for (int k = 0; k < NZ; ++k) col[k] = CX(VVd, i, k, j);
                cfft(&s->pz_plan, col, work, +1);
                for (int k = 0; k < NZ; ++k) CX(VVd, i, k, j) = col[k];
            }
            /* all-to-all copy into TMP(0:NX/2, K, J); Nyquist zeroed */
            for (int k = 0; k <= NZP - 1; ++k) {
                cplx* t = TMP + ((size_t)(j - jmin) * NZP + k) * nh;
                for (int i = 0; i <= NX / 2 - 1; ++i) t[i] = CX(VVd, i, k, j);
                t[NX / 2] = 0.0;
            }
        }
        free(col);
        free(work);
    }
#pragma omp parallel num_threads(nthreads())
    {
        cplx* row = (cplx*)malloc(sizeof(cplx) * NX);
        cplx* work = (cplx*)malloc(sizeof(cplx) * NX);
#pragma omp for collapse(2) schedule(static)
        for (int j = jmin; j <= jmax; ++j)
            for (int k = 0; k < NZP; ++k) {
                const cplx* t = TMP + ((size_t)(j - jmin) * NZP + k) * nh;
                /* c2r: Hermitian extension; imaginary parts of the DC and
                 * Nyquist bins do not contribute to a real output. */
                row[0] = creal(t[0]);
                for (int i = 1; i < NX / 2; ++i) {
                    row[i] = t[i];
                    row[NX - i] = conj(t[i]);
                }
                row[NX / 2] = creal(t[NX / 2]);
                cfft(&s->px_plan, row, work, +1);
                for (int i = 0; i < NX; ++i) PH(V, i, k, j) = creal(row[i]);
            }
        free(row);
        free(work);
    }
    free(TMP);
}

/* ------------------------------------------------------------------------ */
/* Tridiagonal solvers of the MPI build with NPROCY = 1.                      */
/* ------------------------------------------------------------------------ */
/* THOMAS_FORWARD_REAL_MPI + THOMAS_BACKWARD_REAL_MPI (mpi.f:630-697,         */
/* 757-809) for RANKY = 0 = NPROCY-1, INY = NY, columns i < inx.  Arrays are  */
/* (0:INX-1, 0:INY+1) column-major.                                           */
static void thomas_real_mpi(double* A, double* B, double* C, double* G, int iny, int inx) {
#define M2(a, i, j) (a)[(size_t)(i) + (size_t)inx * (size_t)(j)]
    for (int j = 1; j <= iny; ++j)
        for (int i = 0; i < inx; ++i) {
            M2(A, i, j) = -M2(A, i, j) / M2(B, i, j - 1);
            M2(B, i, j) = M2(B, i, j) + M2(A, i, j) * M2(C, i, j - 1);
            M2(G, i, j) = M2(G, i, j) + M2(A, i, j) * M2(G, i, j - 1);
        }
    {
        const int j = iny + 1;
        for (int i = 0; i < inx; ++i) {
            M2(A, i, j) = -M2(A, i, j) / M2(B, i, j - 1);
            M2(B, i, j) = M2(B, i, j) + M2(A, i, j) * M2(C, i, j - 1);
            M2(G, i, j) = M2(G, i, j) + M2(A, i, j) * M2(G, i, j - 1);
        }
    }
    for (int i = 0; i < inx; ++i) {
        M2(G, i, iny + 1) = M2(G, i, iny + 1) / M2(B, i, iny + 1);
        for (int j = iny; j >= 0; --j) {
            if (M2(B, i, j) != 0.0)
                M2(G, i, j) = (M2(G, i, j) - M2(C, i, j) * M2(G, i, j + 1)) / M2(B, i, j);
            else
                M2(G, i, j) = 0.0;
        }
    }
#undef M2
}

/* THOMAS_FORWARD_COMPLEX_MPI + THOMAS_BACKWARD_COMPLEX_MPI (mpi.f:700-754,
 * 812-865) for RANKY = 0 = NPROCY-1: forward rows 2..INY with the B != 0
 * guard, backward from INY down to 1.  Columns 0..inx (inclusive). */
static void thomas_complex_mpi(double* A, double* B, double* C, cplx* G, int iny, int inx) {
    const int ld = inx + 1;
#define M2(a, i, j) (a)[(size_t)(i) + (size_t)ld * (size_t)(j)]
    for (int i = 0; i <= inx; ++i) {
        for (int j = 2; j <= iny; ++j) {
            if (M2(B, i, j - 1) != 0.0)
                M2(A, i, j) = -M2(A, i, j) / M2(B, i, j - 1);
            else
                M2(A, i, j) = 0.0;
            M2(B, i, j) = M2(B, i, j) + M2(A, i, j) * M2(C, i, j - 1);
            M2(G, i, j) = M2(G, i, j) + M2(A, i, j) * M2(G, i, j - 1);
        }
        if (M2(B, i, iny) != 0.0)
            M2(G, i, iny) = M2(G, i, iny) / M2(B, i, iny);
        else
            M2(G, i, iny) = 0.0;
        for (int j = iny - 1; j >= 1; --j) {
            if (M2(B, i, j) != 0.0)
                M2(G, i, j) = (M2(G, i, j) - M2(C, i, j) * M2(G, i, j + 1)) / M2(B, i, j);
            else
                M2(G, i, j) = 0.0;
        }
    }
#undef M2
}

/* ------------------------------------------------------------------------ */
/* Boundary-condition rows (channel.f:1660-2282), both walls applied since    */
/* NPROCY = 1 makes rank 0 both the lowest and the highest (mpi.f:1083-1237). */
/* Arrays (0:NX-1, 0:NY+1).                                                   */
/* ------------------------------------------------------------------------ */
#define MR(a, i, j) (a)[(size_t)(i) + (size_t)s->NX * (size_t)(j)]
static void set_row(orc_state* s, double* L, double* D, double* U, double* V, int j,
                    double l, double d, double u, double v) {
    for (int i = 0; i <= s->NXM; ++i) {
        MR(L, i, j) = l; MR(D, i, j) = d; MR(U, i, j) = u; MR(V, i, j) = v;
    }
}

/* APPLY_BC_1_LOWER / _UPPER and APPLY_BC_3_* share the same rows: U and W
 * are both at GYF points (channel.f:1660-1778, 1967-2086). */
static void bc_u13(orc_state* s, double* L, double* D, double* U, double* V,
                   int bmin, double cmin, int bmax, double cmax) {
    const int NY = s->NY;
    if (bmin == 0) {
        set_row(s, L, D, U, V, 0, 0.0, 1.0, 0.0, 0.0);
        set_row(s, L, D, U, V, 1, 0.0, 1.0, 0.0, cmin);
    } else {
        set_row(s, L, D, U, V, 0, 0.0, 1.0, 0.0, 0.0);
        set_row(s, L, D, U, V, 1, 0.0, -1.0, 1.0, s->DY[2] * cmin);
    }
    if (bmax == 0) {
        set_row(s, L, D, U, V, NY + 1, 0.0, 1.0, 0.0, 0.0);
        set_row(s, L, D, U, V, NY, 0.0, 1.0, 0.0, cmax);
    } else {
        set_row(s, L, D, U, V, NY, -1.0, 1.0, 0.0, s->DY[NY] * cmax);
        set_row(s, L, D, U, V, NY + 1, 0.0, 1.0, 0.0, 0.0);
    }
}

/* APPLY_BC_2_LOWER / APPLY_BC_2_UPPER (channel.f:1822-1934). */
static void bc_u2(orc_state* s, double* L, double* D, double* U, double* V) {
    const int NY = s->NY;
    const diablo_params* p = &s->p;
    if (p->v_bc_ymin == 0) {
        set_row(s, L, D, U, V, 1, 0.0, 1.0, 0.0, p->v_bc_ymin_c1);
        set_row(s, L, D, U, V, 2, 0.0, 1.0, 0.0, p->v_bc_ymin_c1);
    } else if (p->v_bc_ymin == 1) {
        set_row(s, L, D, U, V, 1, 0.0, -1.0, 1.0, s->DYF[1] * p->v_bc_ymin_c1);
    }
    set_row(s, L, D, U, V, 0, 0.0, 1.0, 0.0, 0.0);
    if (p->v_bc_ymax == 0) {
        set_row(s, L, D, U, V, NY + 1, 0.0, 1.0, 0.0, p->v_bc_ymax_c1);
        set_row(s, L, D, U, V, NY, 0.0, 1.0, 0.0, p->v_bc_ymax_c1);
    } else if (p->v_bc_ymax == 1) {
        set_row(s, L, D, U, V, NY + 1, -1.0, 1.0, 0.0, s->DYF[NY] * p->v_bc_ymax_c1);
    }
}

/* APPLY_BC_TH_LOWER / APPLY_BC_TH_UPPER (channel.f:2129-2202). */
static void bc_th(orc_state* s, double* L, double* D, double* U, double* V, int n) {
    const int NY = s->NY;
    const diablo_params* p = &s->p;
    if (p->th_bc_ymin[n] == 0) {
        set_row(s, L, D, U, V, 0, 0.0, 1.0, 0.0, 0.0);
        set_row(s, L, D, U, V, 1, 0.0, 1.0, 0.0, p->th_bc_ymin_c1[n]);
    } else {
        set_row(s, L, D, U, V, 1, 0.0, -1.0, 1.0, s->DY[2] * p->th_bc_ymin_c1[n]);
        set_row(s, L, D, U, V, 0, 0.0, 1.0, 0.0, 0.0);
    }
    if (p->th_bc_ymax[n] == 0) {
        set_row(s, L, D, U, V, NY + 1, 0.0, 1.0, 0.0, 0.0);
        set_row(s, L, D, U, V, NY, 0.0, 1.0, 0.0, p->th_bc_ymax_c1[n]);
    } else {
        set_row(s, L, D, U, V, NY, -1.0, 1.0, 0.0, s->DY[NY] * p->th_bc_ymax_c1[n]);
        set_row(s, L, D, U, V, NY + 1, 0.0, 1.0, 0.0, 0.0);
    }
}

/* Matrices persist across k (they are initialised once before the k loop
 * in the reference and rows not rewritten keep the previous k's factors).
 * That only matters when a BC type leaves a row unset (V_BC = 2); the loop
 * over k runs serially then so that the persistence is reproduced. */
static int serial_k(orc_state* s) {
    return s->p.v_bc_ymin == 2 || s->p.v_bc_ymax == 2;
}

typedef enum { SOLVE_TH, SOLVE_U2, SOLVE_U1, SOLVE_U3 } solve_kind;

/* One implicit CN solve over all (x,z) columns (channel.f:762-1029), with the
 * eddy viscosity / diffusivity rows of the LES build (channel.f:793-805,
 * 862-874, 927-939, 991-1003) when p.les. */
static void cn_solve(orc_state* s, solve_kind kind, int n, double TEMP1, double TEMP2) {
    const int NX = s->NX, NY = s->NY, NZP = s->NZP;
    const size_t msz = (size_t)NX * (NY + 2);
    double* field = kind == SOLVE_TH ? s->TH + (size_t)n * s->nreal
                  : kind == SOLVE_U2 ? s->U2 : kind == SOLVE_U1 ? s->U1 : s->U3;
    const double* rhs = kind == SOLVE_TH ? s->RTH + (size_t)n * s->nreal
                      : kind == SOLVE_U2 ? s->R2 : kind == SOLVE_U1 ? s->R1 : s->R3;
    const double nuv = s->p.nu_v_scale;
    const int nt = serial_k(s) ? 1 : nthreads();
#pragma omp parallel num_threads(nt)
    {
        double* L = (double*)malloc(sizeof(double) * msz);
        double* D = (double*)malloc(sizeof(double) * msz);
        double* U = (double*)malloc(sizeof(double) * msz);
        double* V = (double*)malloc(sizeof(double) * msz);
        for (size_t q = 0; q < msz; ++q) { L[q] = 0.0; D[q] = 1.0; U[q] = 0.0; V[q] = 0.0; }
#pragma omp for schedule(static)
        for (int k = 0; k <= NZP - 1; ++k) {
            int jlo, jhi, jc0, jc1;
            if (kind == SOLVE_TH) {
                const double c = TEMP1 / s->p.pr[n] * nuv;
                jlo = s->JSTART_TH[n]; jhi = s->JEND_TH[n];
                for (int j = jlo; j <= jhi; ++j)
                    for (int i = 0; i <= s->NXM; ++i) {
                        MR(L, i, j) = -c / (s->DY[j] * s->DYF[j]);
                        MR(D, i, j) = 1. + c / (s->DY[j + 1] * s->DYF[j]) + c / (s->DY[j] * s->DYF[j]);
                        MR(U, i, j) = -c / (s->DY[j + 1] * s->DYF[j]);
                        MR(V, i, j) = PH(rhs, i, k, j);
                    }
                if (s->p.les)
                    for (int j = jlo; j <= jhi; ++j)
                        for (int i = 0; i <= s->NXM; ++i) {
                            const double kj = PH(s->NU_T, i, k, j), kp = PH(s->NU_T, i, k, j + 1);
                            MR(L, i, j) = MR(L, i, j) - TEMP2 * kj / (s->DY[j] * s->DYF[j]);
                            MR(D, i, j) = MR(D, i, j) + TEMP2 * kp / (s->DY[j + 1] * s->DYF[j]) +
                                          TEMP2 * kj / (s->DY[j] * s->DYF[j]);
                            MR(U, i, j) = MR(U, i, j) - TEMP2 * kp / (s->DY[j + 1] * s->DYF[j]);
                        }
                bc_th(s, L, D, U, V, n);
                jc0 = jlo - 1; jc1 = jhi + 1;
            } else if (kind == SOLVE_U2) {
                for (int j = 2; j <= NY; ++j)
                    for (int i = 0; i <= s->NXM; ++i) {
                        MR(L, i, j) = -TEMP1 * nuv / (s->DYF[j - 1] * s->DY[j]);
                        MR(D, i, j) = 1. + TEMP1 * nuv / (s->DYF[j] * s->DY[j]) +
                                      TEMP1 * nuv / (s->DYF[j - 1] * s->DY[j]);
                        MR(U, i, j) = -TEMP1 * nuv / (s->DYF[j] * s->DY[j]);
                        MR(V, i, j) = PH(rhs, i, k, j);
                    }
                if (s->p.les)
                    for (int j = 2; j <= NY; ++j)
                        for (int i = 0; i <= s->NXM; ++i) {
                            const double nm = PH(s->NU_T, i, k, j) + PH(s->NU_T, i, k, j - 1);
                            const double np = PH(s->NU_T, i, k, j) + PH(s->NU_T, i, k, j + 1);
                            MR(L, i, j) = MR(L, i, j) - TEMP2 * 0.5 * nm / (s->DYF[j - 1] * s->DY[j]);
                            MR(D, i, j) = MR(D, i, j) + TEMP2 * 0.5 * np / (s->DYF[j] * s->DY[j]) +
                                          TEMP2 * 0.5 * nm / (s->DYF[j - 1] * s->DY[j]);
                            MR(U, i, j) = MR(U, i, j) - TEMP2 * 0.5 * np / (s->DYF[j] * s->DY[j]);
                        }
                bc_u2(s, L, D, U, V);
                jc0 = 1; jc1 = NY + 1;
            } else {
                jlo = s->JSTART; jhi = s->JEND;
                for (int j = jlo; j <= jhi; ++j)
                    for (int i = 0; i <= s->NXM; ++i) {
                        MR(L, i, j) = -TEMP1 * nuv / (s->DY[j] * s->DYF[j]);
                        MR(D, i, j) = 1. - TEMP1 * nuv * (-1. / (s->DY[j + 1] * s->DYF[j]) -
                                                          1. / (s->DY[j] * s->DYF[j]));
                        MR(U, i, j) = -TEMP1 * nuv / (s->DY[j + 1] * s->DYF[j]);
                        MR(V, i, j) = PH(rhs, i, k, j);
                    }
                if (s->p.les)
                    for (int j = jlo; j <= jhi; ++j)
                        for (int i = 0; i <= s->NXM; ++i) {
                            const double nj = PH(s->NU_T, i, k, j), nq = PH(s->NU_T, i, k, j + 1);
                            MR(L, i, j) = MR(L, i, j) - TEMP2 * nj / (s->DY[j] * s->DYF[j]);
                            MR(D, i, j) = MR(D, i, j) + TEMP2 * nq / (s->DY[j + 1] * s->DYF[j]) +
                                          TEMP2 * nj / (s->DY[j] * s->DYF[j]);
                            MR(U, i, j) = MR(U, i, j) - TEMP2 * nq / (s->DY[j + 1] * s->DYF[j]);
                        }
                if (kind == SOLVE_U1)
                    bc_u13(s, L, D, U, V, s->p.u_bc_ymin, s->p.u_bc_ymin_c1, s->p.u_bc_ymax,
                           s->p.u_bc_ymax_c1);
                else
                    bc_u13(s, L, D, U, V, s->p.w_bc_ymin, s->p.w_bc_ymin_c1, s->p.w_bc_ymax,
                           s->p.w_bc_ymax_c1);
                jc0 = jlo - 1; jc1 = jhi + 1;
            }
            thomas_real_mpi(L, D, U, V, NY, NX);
            for (int j = jc0; j <= jc1; ++j)
                for (int i = 0; i <= s->NXM; ++i) PH(field, i, k, j) = MR(V, i, j);
        }
        free(L); free(D); free(U); free(V);
    }
}
#undef MR

/* ------------------------------------------------------------------------ */
/* LES, constant-Smagorinsky model (LES_MODEL_TYPE = 1).                      */
/* ------------------------------------------------------------------------ */

/* APPLY_BC_LES (les.f:805-865): Neumann walls copy the last interior row of
 * CU1 / CU3 into the ghost rows (the upper wall rewrites row NY too). */
static void apply_bc_les(orc_state* s) {
    const int NY = s->NY, NXP = s->NXP, TNKZ = s->TNKZ;
    const diablo_params* p = &s->p;
    double* CU[2] = {s->U1, s->U3};
    const int top[2] = {p->u_bc_ymax, p->w_bc_ymax}, bot[2] = {p->u_bc_ymin, p->w_bc_ymin};
    for (int c = 0; c < 2; ++c) {
        double* C = CU[c];
        if (top[c] == 1)
            for (int k = 0; k <= TNKZ; ++k)
                for (int i = 0; i <= NXP - 1; ++i) {
                    CX(C, i, k, NY) = CX(C, i, k, NY - 1);
                    CX(C, i, k, NY + 1) = CX(C, i, k, NY);
                }
    }
    for (int c = 0; c < 2; ++c) {
        double* C = CU[c];
        if (bot[c] == 1)
            for (int k = 0; k <= TNKZ; ++k)
                for (int i = 0; i <= NXP - 1; ++i) {
                    CX(C, i, k, 1) = CX(C, i, k, 2);
                    CX(C, i, k, 0) = CX(C, i, k, 1);
                }
    }
}

/* APPLY_BC_VEL_PHYS_LOWER / _UPPER (channel.f:2495-2660) on U1..U3 in
 * physical space.  V_BC = 2 stops the reference there, so it never gets here. */
static void apply_bc_vel_phys(orc_state* s) {
    const int NY = s->NY, NZP = s->NZP, NXM = s->NXM;
    const diablo_params* p = &s->p;
    const double* DY = s->DY;
    const double* DYF = s->DYF;
    double *U1 = s->U1, *U2 = s->U2, *U3 = s->U3;
    for (int k = 0; k <= NZP - 1; ++k)
        for (int i = 0; i <= NXM; ++i) {
            /* lower wall */
            if (p->u_bc_ymin == 0) {
                PH(U1, i, k, 0) = p->u_bc_ymin_c1; PH(U1, i, k, 1) = p->u_bc_ymin_c1;
            } else {
                PH(U1, i, k, 1) = PH(U1, i, k, 2) - DY[2] * p->u_bc_ymin_c1;
                PH(U1, i, k, 0) = PH(U1, i, k, 1) - DY[1] * p->u_bc_ymin_c1;
            }
            if (p->w_bc_ymin == 0) {
                PH(U3, i, k, 0) = p->w_bc_ymin_c1; PH(U3, i, k, 1) = p->w_bc_ymin_c1;
            } else {
                PH(U3, i, k, 1) = PH(U3, i, k, 2) - DY[2] * p->w_bc_ymin_c1;
                PH(U3, i, k, 0) = PH(U3, i, k, 1) - DY[1] * p->w_bc_ymin_c1;
            }
            if (p->v_bc_ymin == 0) {
                PH(U2, i, k, 1) = 2.0 * p->v_bc_ymin_c1 - PH(U2, i, k, 2);
                PH(U2, i, k, 0) = PH(U2, i, k, 1);
            } else {
                PH(U2, i, k, 1) = PH(U2, i, k, 2) - DYF[1] * p->v_bc_ymin_c1;
                PH(U2, i, k, 0) = PH(U2, i, k, 1) - DYF[1] * p->v_bc_ymin_c1;
            }
            /* upper wall */
            if (p->u_bc_ymax == 0) {
                PH(U1, i, k, NY) = p->u_bc_ymax_c1; PH(U1, i, k, NY + 1) = p->u_bc_ymax_c1;
            } else {
                PH(U1, i, k, NY) = PH(U1, i, k, NY - 1) + DY[NY] * p->u_bc_ymax_c1;
                PH(U1, i, k, NY + 1) = PH(U1, i, k, NY) + DY[NY] * p->u_bc_ymax_c1;
            }
            if (p->w_bc_ymax == 0) {
                PH(U3, i, k, NY) = p->w_bc_ymax_c1; PH(U3, i, k, NY + 1) = p->w_bc_ymax_c1;
            } else {
                PH(U3, i, k, NY) = PH(U3, i, k, NY - 1) + DY[NY] * p->w_bc_ymax_c1;
                PH(U3, i, k, NY + 1) = PH(U3, i, k, NY) + DY[NY] * p->w_bc_ymax_c1;
            }
            if (p->v_bc_ymax == 0)
                PH(U2, i, k, NY + 1) = 2.0 * p->v_bc_ymax_c1 - PH(U2, i, k, NY);
            else
                PH(U2, i, k, NY + 1) = PH(U2, i, k, NY) + DY[NY] * p->v_bc_ymax_c1;
        }
}

/* Filter widths with -2 C_s^2 absorbed, C_s = 0.13, beta_sgs = 1
 * (les.f:196-217): at GYF (dyf = DYF) or GY (dyf = DY) points. */
static double smag_width(orc_state* s, double dyj) {
    const double C_SMAG = 0.13, beta_sgs = 1.0;
    return -2.0 * (C_SMAG * C_SMAG) * pow(s->DX * beta_sgs * dyj * 2.0 * s->DZ * beta_sgs, 2.0 / 3.0);
}

/* The 5-point test filter of les_filter_chan (les.f:572-712) on one x-z
 * plane of nq quantities q[nq][NZ][NX], periodic in x, then in z; tmp has
 * the same size. */
static void test_filter_plane(orc_state* s, double* q, double* tmp, int nq) {
    const double Wm2 = 1.0 / 8.0, Wm1 = 1.0 / 4.0, W0 = 1.0 / 4.0, W1 = 1.0 / 4.0, W2 = 1.0 / 8.0;
    const int NX = s->NX, NZ = s->NZ;
    for (int f = 0; f < nq; ++f) {
        double* A = q + (size_t)f * NZ * NX;
        double* B = tmp + (size_t)f * NZ * NX;
        for (int k = 0; k < NZ; ++k)
            for (int i = 0; i < NX; ++i) {
                const double* r = A + (size_t)k * NX;
                B[(size_t)k * NX + i] = Wm2 * r[(i - 2 + NX) % NX] + Wm1 * r[(i - 1 + NX) % NX] + W0 * r[i] +
                                        W1 * r[(i + 1) % NX] + W2 * r[(i + 2) % NX];
            }
        for (int k = 0; k < NZ; ++k)
            for (int i = 0; i < NX; ++i)
                A[(size_t)k * NX + i] = Wm2 * B[(size_t)((k - 2 + NZ) % NZ) * NX + i] +
                                        Wm1 * B[(size_t)((k - 1 + NZ) % NZ) * NX + i] + W0 * B[(size_t)k * NX + i] +
                                        W1 * B[(size_t)((k + 1) % NZ) * NX + i] + W2 * B[(size_t)((k + 2) % NZ) * NX + i];
    }
}

/* Dynamic Smagorinsky coefficient, LES_MODEL_TYPE = 2.  The reference stops
 * for this model type (les.f:269-272); this model is written for this
 * library: the Germano identity with Lilly's least squares over each x-z
 * plane, at GYF points J = 2..NY, with U2 and the GY strains S_12, S_23
 * averaged to GYF:
 *   L_ij = (u_i u_j)^ - u^_i u^_j
 *   M_ij = R |S^| S^_ij - (|S| S_ij)^,   R = (Delta^/Delta)^2 = 9^(2/3)
 *   (C Delta^2)(J) = max(0, -<L_ij M_ij> / (2 <M_ij M_ij>))
 * where ^ is the test filter above, <.> the plane sum with the off-diagonal
 * pairs counted twice, and |S|, |S^| have the mean shear removed as in
 * les.f:113-137.  R reads the reference's label for this filter, alpha*beta
 * = 9 (les.f:601), as the ratio of filtered cell volumes: the test filter
 * widens x and z only.  DELTA_YF = -2 C Delta^2 at GYF points and DELTA_Y
 * its interpolation to GY points, in the place of the constant model's
 * -2 C_s^2 Delta^2 (les.f:196-217).  S1 holds |S| at GYF. */
static void dynamic_widths(orc_state* s, const double* U1_bar, const double* U3_bar, double* DELTA_YF,
                           double* DELTA_Y) {
    const int NY = s->NY, NX = s->NX, NZ = s->NZ;
    const double* DY = s->DY;
    const double* DYF = s->DYF;
    const double R = pow(9.0, 2.0 / 3.0);
    double* CD = (double*)calloc(NY + 2, sizeof(double));
    const size_t pl = (size_t)NX * NZ;
#pragma omp parallel num_threads(nthreads())
    {
        double* q = (double*)malloc(sizeof(double) * 21 * pl);
        double* tmp = (double*)malloc(sizeof(double) * 21 * pl);
#pragma omp for schedule(dynamic)
        for (int j = 2; j <= NY; ++j) {
            for (int k = 0; k < NZ; ++k)
                for (int i = 0; i < NX; ++i) {
                    const double u1 = PH(s->U1, i, k, j), u3 = PH(s->U3, i, k, j);
                    const double u2 = 0.5 * (PH(s->U2, i, k, j) + PH(s->U2, i, k, j + 1));
                    const double s11 = PH(s->SIJ[0], i, k, j), s22 = PH(s->SIJ[1], i, k, j);
                    const double s33 = PH(s->SIJ[2], i, k, j), s13 = PH(s->SIJ[4], i, k, j);
                    const double s12 = 0.5 * (PH(s->SIJ[3], i, k, j) + PH(s->SIJ[3], i, k, j + 1));
                    const double s23 = 0.5 * (PH(s->SIJ[5], i, k, j) + PH(s->SIJ[5], i, k, j + 1));
                    const double sm = PH(s->S1, i, k, j);
                    const double v[21] = {u1, u2, u3, u1 * u1, u2 * u2, u3 * u3, u1 * u2, u1 * u3, u2 * u3,
                                          s11, s22, s33, s12, s13, s23,
                                          sm * s11, sm * s22, sm * s33, sm * s12, sm * s13, sm * s23};
                    for (int f = 0; f < 21; ++f) q[(size_t)f * pl + (size_t)k * NX + i] = v[f];
                }
            test_filter_plane(s, q, tmp, 21);
            const double m1 = 0.5 * (U1_bar[j] - U1_bar[j - 1]) / DY[j] + 0.5 * (U1_bar[j + 1] - U1_bar[j]) / DY[j + 1];
            const double m3 = 0.5 * (U3_bar[j] - U3_bar[j - 1]) / DY[j] + 0.5 * (U3_bar[j + 1] - U3_bar[j]) / DY[j + 1];
            double num = 0.0, den = 0.0;
            for (size_t e = 0; e < pl; ++e) {
                double h[21];
                for (int f = 0; f < 21; ++f) h[f] = q[(size_t)f * pl + e];
                const double a12 = h[12] - 0.5 * m1, a23 = h[14] - 0.5 * m3;
                const double sh = sqrt(2.0 * (h[9] * h[9]) + 4.0 * (a12 * a12) + 4.0 * (h[13] * h[13]) +
                                       2.0 * (h[10] * h[10]) + 4.0 * (a23 * a23) + 2.0 * (h[11] * h[11]));
                const double L11 = h[3] - h[0] * h[0], L22 = h[4] - h[1] * h[1], L33 = h[5] - h[2] * h[2];
                const double L12 = h[6] - h[0] * h[1], L13 = h[7] - h[0] * h[2], L23 = h[8] - h[1] * h[2];
                const double M11 = R * sh * h[9] - h[15], M22 = R * sh * h[10] - h[16], M33 = R * sh * h[11] - h[17];
                const double M12 = R * sh * h[12] - h[18], M13 = R * sh * h[13] - h[19], M23 = R * sh * h[14] - h[20];
                num += L11 * M11 + L22 * M22 + L33 * M33 + 2.0 * (L12 * M12 + L13 * M13 + L23 * M23);
                den += M11 * M11 + M22 * M22 + M33 * M33 + 2.0 * (M12 * M12 + M13 * M13 + M23 * M23);
            }
            const double c = den > 0.0 ? -0.5 * num / den : 0.0;
            CD[j] = c > 0.0 ? c : 0.0;
        }
        free(q);
        free(tmp);
    }
    for (int j = 1; j <= NY + 1; ++j) {
        const int jf = j < 2 ? 2 : j > NY ? NY : j;
        DELTA_YF[j] = -2.0 * CD[jf];
    }
    for (int j = 2; j <= NY + 1; ++j) {
        const double cg = (j >= 3 && j <= NY) ? (CD[j] * DYF[j - 1] + CD[j - 1] * DYF[j]) / (2.0 * DY[j])
                        : CD[j <= 2 ? 2 : NY];
        DELTA_Y[j] = -2.0 * cg;
    }
    free(CD);
}

/* The learned closure (LES_MODEL_TYPE 4), which the reference does not
 * have: the features of the resolved field at GYF rows J = 2..NY-1 (the
 * velocity gradients by centred differences, U2 averaged to GYF, divided by
 * their norm G; y+ and the grid filter width Delta), the MLP of the GPU
 * library, whose outputs times Delta^2 G^2 are the stresses, with its weights,
 * normalised inputs and hidden activations rounded to bfloat16 as its
 * tensor cores see them, tau_12 and tau_23 interpolated to GY points, and
 * CF_i -= d tau_ij / dx_j, all explicit. */
#define MLP_NIN 11
#define MLP_NH 64
#define MLP_NOUT 6
static float bf16r(double v) {
    float f = (float)v;
    uint32_t u;
    memcpy(&u, &f, 4);
    u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
    memcpy(&f, &u, 4);
    return f;
}

void orc_set_mlp(orc_state* s, const float* params) {
    const size_t n = (size_t)MLP_NH * MLP_NIN + MLP_NH + 2 * ((size_t)MLP_NH * MLP_NH + MLP_NH) +
                     (size_t)MLP_NOUT * MLP_NH + MLP_NOUT + 2 * MLP_NIN + MLP_NOUT;
    free(s->MLP);
    s->MLP = NULL;
    if (!params) return;
    s->MLP = (float*)malloc(sizeof(float) * n);
    memcpy(s->MLP, params, sizeof(float) * n);
}

/* GELU in its tanh form, as the GPU library evaluates it */
static double mlp_gelu(double z) {
    return 0.5 * z * (1.0 + tanh(sqrt(2.0 / (4.0 * atan(1.0))) * (z + 0.044715 * z * z * z)));
}

static void mlp_forward(const float* P, const float* xf, float* y) {
    const float* W1 = P;
    const float* b1 = W1 + MLP_NH * MLP_NIN;
    const float* W2 = b1 + MLP_NH;
    const float* b2 = W2 + MLP_NH * MLP_NH;
    const float* W3 = b2 + MLP_NH;
    const float* b3 = W3 + MLP_NH * MLP_NH;
    const float* W4 = b3 + MLP_NH;
    const float* b4 = W4 + MLP_NOUT * MLP_NH;
    const float* mean = b4 + MLP_NOUT;
    const float* scale = mean + MLP_NIN;
    const float* osc = scale + MLP_NIN;
    double h[MLP_NH], g[MLP_NH], x[MLP_NIN];
    for (int k = 0; k < MLP_NIN; ++k) x[k] = bf16r((xf[k] - mean[k]) / scale[k]);
    for (int o = 0; o < MLP_NH; ++o) {
        double z = b1[o];
        for (int k = 0; k < MLP_NIN; ++k) z += (double)bf16r(W1[o * MLP_NIN + k]) * x[k];
        h[o] = bf16r((float)mlp_gelu(z));
    }
    const float* Ws[2] = {W2, W3};
    const float* bs[2] = {b2, b3};
    for (int l = 0; l < 2; ++l) {
        for (int o = 0; o < MLP_NH; ++o) {
            double z = bs[l][o];
            for (int k = 0; k < MLP_NH; ++k) z += (double)bf16r(Ws[l][o * MLP_NH + k]) * h[k];
            g[o] = bf16r((float)mlp_gelu(z));
        }
        memcpy(h, g, sizeof(h));
    }
    for (int o = 0; o < MLP_NOUT; ++o) {
        double z = b4[o];
        for (int k = 0; k < MLP_NH; ++k) z += (double)bf16r(W4[o * MLP_NH + k]) * h[k];
        y[o] = (float)z * osc[o];
    }
}

static void les_mlp(orc_state* s) {
    const int NY = s->NY, NX = s->NX, NZ = s->NZ, NXP = s->NXP, TNKZ = s->TNKZ;
    const double* DY = s->DY;
    const double* DYF = s->DYF;
    const double* GYF = s->GYF;
    double *U1 = s->U1, *U2 = s->U2, *U3 = s->U3;
    double *CF1 = s->F1, *CF2 = s->F2, *CF3 = s->F3;
    const cplx CI = I;
    orc_apply_bc_vel(s);
    apply_bc_les(s);
    orc_fft_xz_to_physical(s, U1, U1, 0, NY + 1);
    orc_fft_xz_to_physical(s, U2, U2, 0, NY + 1);
    orc_fft_xz_to_physical(s, U3, U3, 0, NY + 1);
    double* T[6];
    for (int q = 0; q < 6; ++q) {
        T[q] = s->SIJ[q];
        memset(T[q], 0, sizeof(double) * s->nreal);
    }
    const size_t pl = (size_t)NX * NZ;
    float* tau = (float*)calloc((size_t)(NY + 2) * pl * 6, sizeof(float));
#pragma omp parallel for num_threads(nthreads())
    for (int j = 2; j <= NY - 1; ++j)
        for (int k = 0; k < NZ; ++k)
            for (int i = 0; i < NX; ++i) {
                const int ip = (i + 1) % NX, im = (i - 1 + NX) % NX, kp = (k + 1) % NZ, km = (k - 1 + NZ) % NZ;
                double x[MLP_NIN];
                const double* Us[3] = {U1, U2, U3};
                const double hy = GYF[j + 1] - GYF[j - 1];
                for (int c = 0; c < 3; ++c) {
                    const double* u = Us[c];
#define UU(ii, kk, jj) (c == 1 ? 0.5 * (PH(u, ii, kk, jj) + PH(u, ii, kk, (jj) + 1)) : PH(u, ii, kk, jj))
                    x[3 * c + 0] = (UU(ip, k, j) - UU(im, k, j)) / (2.0 * s->DX);
                    x[3 * c + 1] = (UU(i, k, j + 1) - UU(i, k, j - 1)) / hy;
                    x[3 * c + 2] = (UU(i, kp, j) - UU(i, km, j)) / (2.0 * s->DZ);
#undef UU
                }
                double g2 = 0.0;
                for (int q = 0; q < 9; ++q) g2 += x[q] * x[q];
                const double G = sqrt(g2), ig = G > 0.0 ? 1.0 / G : 0.0;
                for (int q = 0; q < 9; ++q) x[q] *= ig;
                x[9] = fmin(GYF[j] - GYF[1], GYF[NY] - GYF[j]) / s->p.nu;
                x[10] = cbrt(s->DX * DYF[j] * s->DZ);
                const float sc = (float)(x[10] * x[10] * g2);
                float xf[MLP_NIN];
                for (int q = 0; q < MLP_NIN; ++q) xf[q] = (float)x[q];
                float* y = tau + (((size_t)j * NZ + k) * NX + i) * 6;
                mlp_forward(s->MLP, xf, y);
                for (int q = 0; q < 6; ++q) y[q] = y[q] * sc;
            }
    /* 11, 22, 33, 13 at GYF rows 2..NY-1; 12, 23 at GY rows 3..NY-1 */
#define TAU(q, i, k, j) ((double)tau[(((size_t)(j) * NZ + (k)) * NX + (i)) * 6 + (q)])
    for (int j = 2; j <= NY - 1; ++j)
        for (int k = 0; k < NZ; ++k)
            for (int i = 0; i < NX; ++i) {
                PH(T[0], i, k, j) = TAU(0, i, k, j);
                PH(T[1], i, k, j) = TAU(1, i, k, j);
                PH(T[2], i, k, j) = TAU(2, i, k, j);
                PH(T[3], i, k, j) = TAU(4, i, k, j);
                if (j >= 3) {
                    PH(T[4], i, k, j) = (TAU(3, i, k, j) * DYF[j - 1] + TAU(3, i, k, j - 1) * DYF[j]) / (2.0 * DY[j]);
                    PH(T[5], i, k, j) = (TAU(5, i, k, j) * DYF[j - 1] + TAU(5, i, k, j - 1) * DYF[j]) / (2.0 * DY[j]);
                }
            }
#undef TAU
    free(tau);
    for (int q = 0; q < 6; ++q) orc_fft_xz_to_fourier(s, T[q], T[q], 0, NY + 1);
#pragma omp parallel for num_threads(nthreads())
    for (int j = 2; j <= NY; ++j)
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) {
                if (j <= NY - 1) {
                    CX(CF1, i, k, j) = CX(CF1, i, k, j) - CI * s->KX[i] * CX(T[0], i, k, j) -
                                       (CX(T[4], i, k, j + 1) - CX(T[4], i, k, j)) / DYF[j] -
                                       CI * s->KZ[k] * CX(T[3], i, k, j);
                    CX(CF3, i, k, j) = CX(CF3, i, k, j) - CI * s->KX[i] * CX(T[3], i, k, j) -
                                       (CX(T[5], i, k, j + 1) - CX(T[5], i, k, j)) / DYF[j] -
                                       CI * s->KZ[k] * CX(T[2], i, k, j);
                }
                CX(CF2, i, k, j) = CX(CF2, i, k, j) - CI * s->KX[i] * CX(T[4], i, k, j) -
                                   (CX(T[1], i, k, j) - CX(T[1], i, k, j - 1)) / DY[j] -
                                   CI * s->KZ[k] * CX(T[5], i, k, j);
            }
}

/* les_chan (les.f:1-267, 280-336), LES_MODEL_TYPE = 1 (and 2, the dynamic
 * coefficient above in place of C_s), NPROCY = NPROCZ = 1.
 * On exit U1..U3 are in physical space, NU_T is set and CF1..CF3 hold the
 * subgrid-stress divergence and the explicit cross terms. */
static void les_chan(orc_state* s) {
    const int NY = s->NY, NXP = s->NXP, TNKZ = s->TNKZ, NZP = s->NZP, NXM = s->NXM;
    const int JSTART = s->JSTART, JEND = s->JEND;
    const double* DY = s->DY;
    const double* DYF = s->DYF;
    double *CU1 = s->U1, *CU2 = s->U2, *CU3 = s->U3;
    double *U1 = s->U1, *U3 = s->U3;
    double *CF1 = s->F1, *CF2 = s->F2, *CF3 = s->F3;
    double *S1 = s->S1, *TEMP = s->TEMP, *NU_T = s->NU_T;
    double *Sij1 = s->SIJ[0], *Sij2 = s->SIJ[1], *Sij3 = s->SIJ[2];
    double *Sij4 = s->SIJ[3], *Sij5 = s->SIJ[4], *Sij6 = s->SIJ[5];
    const cplx CI = I;
    if (s->p.les_model_type == 4 && s->MLP) {
        les_mlp(s);
        return;
    }
    /* ghost cells (les.f:64-77): APPLY_BC_VEL_MPI, then APPLY_BC_LES */
    orc_apply_bc_vel(s);
    apply_bc_les(s);
    /* compute_strain_chan (les.f:526-569) */
#pragma omp parallel for num_threads(nthreads())
    for (int j = 1; j <= NY; ++j)
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) {
                CX(Sij1, i, k, j) = CI * s->KX[i] * CX(CU1, i, k, j);
                CX(Sij2, i, k, j) = (CX(CU2, i, k, j + 1) - CX(CU2, i, k, j)) / DYF[j];
                CX(Sij3, i, k, j) = CI * s->KZ[k] * CX(CU3, i, k, j);
                CX(Sij5, i, k, j) = 0.5 * (CI * s->KZ[k] * CX(CU1, i, k, j) + CI * s->KX[i] * CX(CU3, i, k, j));
            }
#pragma omp parallel for num_threads(nthreads())
    for (int j = 1; j <= NY + 1; ++j)
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) {
                CX(Sij4, i, k, j) =
                    0.5 * ((CX(CU1, i, k, j) - CX(CU1, i, k, j - 1)) / DY[j] + CI * s->KX[i] * CX(CU2, i, k, j));
                CX(Sij6, i, k, j) =
                    0.5 * (CI * s->KZ[k] * CX(CU2, i, k, j) + (CX(CU3, i, k, j) - CX(CU3, i, k, j - 1)) / DY[j]);
            }
    for (int q = 0; q < 6; ++q) orc_fft_xz_to_physical(s, s->SIJ[q], s->SIJ[q], 0, NY + 1);
    /* mean profiles (les.f:87-92) */
    double* U1_bar = (double*)malloc(sizeof(double) * (NY + 2));
    double* U3_bar = (double*)malloc(sizeof(double) * (NY + 2));
    for (int j = 0; j <= NY + 1; ++j) {
        U1_bar[j] = creal(CX(CU1, 0, 0, j));
        U3_bar[j] = creal(CX(CU3, 0, 0, j));
    }
    orc_fft_xz_to_physical(s, CU1, U1, 0, NY + 1);
    orc_fft_xz_to_physical(s, CU2, s->U2, 0, NY + 1);
    orc_fft_xz_to_physical(s, CU3, U3, 0, NY + 1);
    /* |S| at GYF points with the mean shear removed (les.f:113-137) */
#pragma omp parallel for num_threads(nthreads())
    for (int j = JSTART; j <= JEND; ++j)
        for (int k = 0; k <= NZP - 1; ++k)
            for (int i = 0; i <= NXM; ++i) {
                const double a4 = 0.5 * (PH(Sij4, i, k, j + 1) + PH(Sij4, i, k, j) -
                                         0.5 * (U1_bar[j] - U1_bar[j - 1]) / DY[j] -
                                         0.5 * (U1_bar[j + 1] - U1_bar[j]) / DY[j + 1]);
                const double a6 = 0.5 * (PH(Sij6, i, k, j + 1) + PH(Sij6, i, k, j) -
                                         0.5 * (U3_bar[j] - U3_bar[j - 1]) / DY[j] -
                                         0.5 * (U3_bar[j + 1] - U3_bar[j]) / DY[j + 1]);
                const double s1 = PH(Sij1, i, k, j), s2 = PH(Sij2, i, k, j), s3 = PH(Sij3, i, k, j);
                const double s5 = PH(Sij5, i, k, j);
                PH(S1, i, k, j) = sqrt(2.0 * (s1 * s1) + 4.0 * (a4 * a4) + 4.0 * (s5 * s5) + 2.0 * (s2 * s2) +
                                       4.0 * (a6 * a6) + 2.0 * (s3 * s3));
            }
    /* |S| at GY points (les.f:140-160) */
#pragma omp parallel for num_threads(nthreads())
    for (int j = 2; j <= NY + 1; ++j)
        for (int k = 0; k <= NZP - 1; ++k)
            for (int i = 0; i <= NXM; ++i) {
                const double g1 = (PH(Sij1, i, k, j) * DYF[j - 1] + PH(Sij1, i, k, j - 1) * DYF[j]) / (2.0 * DY[j]);
                const double g5 = (PH(Sij5, i, k, j) * DYF[j - 1] + PH(Sij5, i, k, j - 1) * DYF[j]) / (2.0 * DY[j]);
                const double g2 = (PH(Sij2, i, k, j) * DYF[j - 1] + PH(Sij2, i, k, j - 1) * DYF[j]) / (2.0 * DY[j]);
                const double g3 = (PH(Sij3, i, k, j) * DYF[j - 1] + PH(Sij3, i, k, j - 1) * DYF[j]) / (2.0 * DY[j]);
                const double b4 = PH(Sij4, i, k, j) - 0.5 * (U1_bar[j] - U1_bar[j - 1]) / DY[j];
                const double b6 = PH(Sij6, i, k, j) - 0.5 * (U3_bar[j] - U3_bar[j - 1]) / DY[j];
                PH(TEMP, i, k, j) = sqrt(2.0 * (g1 * g1) + 4.0 * (b4 * b4) + 4.0 * (g5 * g5) + 2.0 * (g2 * g2) +
                                         4.0 * (b6 * b6) + 2.0 * (g3 * g3));
            }
    /* filter widths with -2 C^2 absorbed: constant (les.f:196-217) or
     * dynamic (model type 2) */
    double* DELTA_YF = (double*)calloc(NY + 2, sizeof(double));
    double* DELTA_Y = (double*)calloc(NY + 2, sizeof(double));
    if (s->p.les_model_type == 2 || s->p.les_model_type == 4) {   /* 4 without a network: dynamic */
        dynamic_widths(s, U1_bar, U3_bar, DELTA_YF, DELTA_Y);
    } else {
        for (int j = 1; j <= NY + 1; ++j) {
            DELTA_YF[j] = smag_width(s, DYF[j]);
            DELTA_Y[j] = smag_width(s, DY[j]);
        }
    }
    free(U1_bar);
    free(U3_bar);
    /* |S| S_ij: GYF components (les.f:165-177), Sij2 left to the implicit
     * eddy viscosity; GY components without the implicit dU/dy part
     * (les.f:181-194) */
#pragma omp parallel for num_threads(nthreads())
    for (int j = JSTART; j <= JEND; ++j)
        for (int k = 0; k <= NZP - 1; ++k)
            for (int i = 0; i <= NXM; ++i) {
                PH(Sij1, i, k, j) = PH(S1, i, k, j) * PH(Sij1, i, k, j);
                PH(Sij5, i, k, j) = PH(S1, i, k, j) * PH(Sij5, i, k, j);
                PH(Sij2, i, k, j) = 0.0;
                PH(Sij3, i, k, j) = PH(S1, i, k, j) * PH(Sij3, i, k, j);
            }
#pragma omp parallel for num_threads(nthreads())
    for (int j = 2; j <= NY + 1; ++j)
        for (int k = 0; k <= NZP - 1; ++k)
            for (int i = 0; i <= NXM; ++i) {
                PH(Sij4, i, k, j) = PH(TEMP, i, k, j) * (PH(Sij4, i, k, j) - 0.5 * (PH(U1, i, k, j) - PH(U1, i, k, j - 1)) / DY[j]);
                PH(Sij6, i, k, j) = PH(TEMP, i, k, j) * (PH(Sij6, i, k, j) - 0.5 * (PH(U3, i, k, j) - PH(U3, i, k, j - 1)) / DY[j]);
            }
    /* NU_T = C_s^2 Delta^2 |S| at GY points (les.f:219-227); GHOST_LES_MPI
     * zeroes rows 1, 2, NY and NY+1 (mpi.f:494-507) */
#pragma omp parallel for num_threads(nthreads())
    for (int j = 2; j <= NY; ++j)
        for (int k = 0; k <= NZP - 1; ++k)
            for (int i = 0; i <= NXM; ++i) PH(NU_T, i, k, j) = -0.5 * DELTA_Y[j] * PH(TEMP, i, k, j);
    for (int k = 0; k <= NZP - 1; ++k)
        for (int i = 0; i <= NXM; ++i) {
            PH(NU_T, i, k, 1) = 0.0; PH(NU_T, i, k, 2) = 0.0;
            PH(NU_T, i, k, NY) = 0.0; PH(NU_T, i, k, NY + 1) = 0.0;
        }
    /* tau_ij in Fourier space (les.f:235-262) */
    orc_fft_xz_to_fourier(s, Sij1, Sij1, 0, NY + 1);
    orc_fft_xz_to_fourier(s, Sij3, Sij3, 0, NY + 1);
    orc_fft_xz_to_fourier(s, Sij4, Sij4, 0, NY + 1);
    orc_fft_xz_to_fourier(s, Sij5, Sij5, 0, NY + 1);
    orc_fft_xz_to_fourier(s, Sij6, Sij6, 0, NY + 1);
#pragma omp parallel for num_threads(nthreads())
    for (int j = 1; j <= NY + 1; ++j)
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) {
                CX(Sij1, i, k, j) = DELTA_YF[j] * CX(Sij1, i, k, j);
                CX(Sij5, i, k, j) = DELTA_YF[j] * CX(Sij5, i, k, j);
                CX(Sij3, i, k, j) = DELTA_YF[j] * CX(Sij3, i, k, j);
            }
#pragma omp parallel for num_threads(nthreads())
    for (int j = 2; j <= NY + 1; ++j)
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) {
                CX(Sij4, i, k, j) = DELTA_Y[j] * CX(Sij4, i, k, j);
                CX(Sij6, i, k, j) = DELTA_Y[j] * CX(Sij6, i, k, j);
            }
    free(DELTA_YF);
    free(DELTA_Y);
    /* CF_i -= d tau_ij / dx_j (les.f:280-304); J1 = JSTART, J2 = NY-1 on the
     * rank at the upper wall, which NPROCY = 1 makes the only one (les.f:46-59) */
#pragma omp parallel for num_threads(nthreads())
    for (int j = JSTART; j <= NY - 1; ++j)
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) {
                CX(CF1, i, k, j) = CX(CF1, i, k, j) - CI * s->KX[i] * CX(Sij1, i, k, j) -
                                   (CX(Sij4, i, k, j + 1) - CX(Sij4, i, k, j)) / DYF[j] -
                                   CI * s->KZ[k] * CX(Sij5, i, k, j);
                CX(CF3, i, k, j) = CX(CF3, i, k, j) - CI * s->KX[i] * CX(Sij5, i, k, j) -
                                   (CX(Sij6, i, k, j + 1) - CX(Sij6, i, k, j)) / DYF[j] -
                                   CI * s->KZ[k] * CX(Sij3, i, k, j);
            }
#pragma omp parallel for num_threads(nthreads())
    for (int j = 2; j <= NY; ++j)
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i)
                CX(CF2, i, k, j) = CX(CF2, i, k, j) - CI * s->KX[i] * CX(Sij4, i, k, j) -
                                   CI * s->KZ[k] * CX(Sij6, i, k, j);
    /* explicit cross terms (les.f:307-336) */
    for (int c = 0; c < 2; ++c) {
        const double* U = c == 0 ? U1 : U3;
#pragma omp parallel for num_threads(nthreads())
        for (int j = 2; j <= NY; ++j)
            for (int k = 0; k <= NZP - 1; ++k)
                for (int i = 0; i <= NXM; ++i)
                    PH(TEMP, i, k, j) = PH(NU_T, i, k, j) * (PH(U, i, k, j) - PH(U, i, k, j - 1)) / DY[j];
        orc_fft_xz_to_fourier(s, TEMP, TEMP, 2, NY);
#pragma omp parallel for num_threads(nthreads())
        for (int j = 2; j <= NY; ++j)
            for (int k = 0; k <= TNKZ; ++k)
                for (int i = 0; i <= NXP - 1; ++i)
                    CX(CF2, i, k, j) = CX(CF2, i, k, j) + CI * (c == 0 ? s->KX[i] : s->KZ[k]) * CX(TEMP, i, k, j);
    }
}

/* ------------------------------------------------------------------------ */
/* RK_CHAN_1 (channel.f:62-1073).                                             */
/* ------------------------------------------------------------------------ */
void orc_rk_chan_1(orc_state* s, int rk_step) {
    const int NY = s->NY, NXP = s->NXP, TNKZ = s->TNKZ, NZP = s->NZP, NXM = s->NXM;
    const int JSTART = s->JSTART, JEND = s->JEND;
    const diablo_params* p = &s->p;
    s->RK_STEP = rk_step;
    const int r = rk_step - 1;
    const double TEMP1 = p->nu * s->H_BAR[r] / 2.0;
    const double TEMP2 = s->H_BAR[r] / 2.0;
    const double TEMP3 = s->ZETA_BAR[r] * s->H_BAR[r];
    const double TEMP4 = s->H_BAR[r];
    const double TEMP5 = s->BETA_BAR[r] * s->H_BAR[r];
    double *CU1 = s->U1, *CU2 = s->U2, *CU3 = s->U3, *CP = s->P;
    double *CR1 = s->R1, *CR2 = s->R2, *CR3 = s->R3;
    double *CF1 = s->F1, *CF2 = s->F2, *CF3 = s->F3, *CS1 = s->S1;
    double *U1 = s->U1, *U2 = s->U2, *U3 = s->U3;
    double *R1 = s->R1, *R2 = s->R2, *R3 = s->R3, *S1 = s->S1;
    const cplx CI = I;

    /* CR <- CU (channel.f:88-103) */
#pragma omp parallel for num_threads(nthreads())
    for (int j = JSTART; j <= JEND; ++j)
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) {
                CX(CR1, i, k, j) = CX(CU1, i, k, j);
                CX(CR3, i, k, j) = CX(CU3, i, k, j);
            }
#pragma omp parallel for num_threads(nthreads())
    for (int j = 2; j <= NY; ++j)
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) CX(CR2, i, k, j) = CX(CU2, i, k, j);
    /* + zeta h CF (channel.f:106-121) */
    if (rk_step > 1) {
#pragma omp parallel for num_threads(nthreads())
        for (int j = JSTART; j <= JEND; ++j)
            for (int k = 0; k <= TNKZ; ++k)
                for (int i = 0; i <= NXP - 1; ++i) {
                    CX(CR1, i, k, j) = CX(CR1, i, k, j) + TEMP3 * CX(CF1, i, k, j);
                    CX(CR3, i, k, j) = CX(CR3, i, k, j) + TEMP3 * CX(CF3, i, k, j);
                }
#pragma omp parallel for num_threads(nthreads())
        for (int j = 2; j <= NY; ++j)
            for (int k = 0; k <= TNKZ; ++k)
                for (int i = 0; i <= NXP - 1; ++i)
                    CX(CR2, i, k, j) = CX(CR2, i, k, j) + TEMP3 * CX(CF2, i, k, j);
    }
    /* pressure gradient (channel.f:124-148) */
#pragma omp parallel for num_threads(nthreads())
    for (int j = 2; j <= NY; ++j)
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i)
                CX(CS1, i, k, j) = (CX(CP, i, k, j) - CX(CP, i, k, j - 1)) / s->DY[j];
#pragma omp parallel for num_threads(nthreads())
    for (int j = JSTART; j <= JEND; ++j)
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) {
                CX(CR1, i, k, j) = CX(CR1, i, k, j) - TEMP4 * (CI * s->KX[i] * CX(CP, i, k, j));
                CX(CR3, i, k, j) = CX(CR3, i, k, j) - TEMP4 * (CI * s->KZ[k] * CX(CP, i, k, j));
            }
#pragma omp parallel for num_threads(nthreads())
    for (int j = 2; j <= NY; ++j)
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i)
                CX(CR2, i, k, j) = CX(CR2, i, k, j) - TEMP4 * CX(CS1, i, k, j);
    /* forcing (channel.f:155-167) */
    if (p->f_type == 1) {
        for (int j = JSTART; j <= JEND; ++j) CX(CR1, 0, 0, j) = CX(CR1, 0, 0, j) - TEMP4 * p->px0;
    } else if (p->f_type == 2) {
        for (int j = JSTART; j <= JEND; ++j)
            CX(CR1, 0, 0, j) =
                CX(CR1, 0, 0, j) - TEMP4 * (p->px0 + p->amp_omega0 * cos(p->omega0 * s->TIME));
    }
    /* horizontal viscous terms (channel.f:175-189) */
#pragma omp parallel for num_threads(nthreads())
    for (int j = JSTART; j <= JEND; ++j)
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) {
                const double kk = pow(s->KX2[i] + s->KZ2[k], p->beta);
                CX(CF1, i, k, j) = -p->nu * kk * CX(CU1, i, k, j);
                CX(CF3, i, k, j) = -p->nu * kk * CX(CU3, i, k, j);
            }
#pragma omp parallel for num_threads(nthreads())
    for (int j = 2; j <= NY; ++j)
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i)
                CX(CF2, i, k, j) = -p->nu * pow(s->KX2[i] + s->KZ2[k], p->beta) * CX(CU2, i, k, j);
    /* Coriolis (channel.f:193-200) */
#pragma omp parallel for num_threads(nthreads())
    for (int k = 0; k <= TNKZ; ++k)
        for (int i = 0; i <= NXP - 1; ++i)
            for (int j = JSTART; j <= JEND; ++j) {
                CX(CF1, i, k, j) = CX(CF1, i, k, j) + p->i_ro * CX(CU3, i, k, j);
                CX(CF3, i, k, j) = CX(CF3, i, k, j) - p->i_ro * CX(CU1, i, k, j);
            }
    for (int n = 0; n < s->NTH; ++n) {
        double* CTHn = s->CTH + (size_t)n * s->nreal;
        double* CRTHn = s->CRTH + (size_t)n * s->nreal;
        double* CFTHn = s->CFTH + (size_t)n * s->nreal;
        /* buoyancy into CF2, (0,0) mode skipped (channel.f:209-227) */
#pragma omp parallel for num_threads(nthreads())
        for (int j = 2; j <= NY; ++j) {
            for (int k = 1; k <= TNKZ; ++k)
                for (int i = 0; i <= NXP - 1; ++i)
                    CX(CF2, i, k, j) = CX(CF2, i, k, j) +
                        p->ri[n] * p->grav_y *
                            (CX(CTHn, i, k, j) * s->DYF[j - 1] + CX(CTHn, i, k, j - 1) * s->DYF[j]) /
                            (2.0 * s->DY[j]);
            for (int i = 1; i <= NXP - 1; ++i)
                CX(CF2, i, 0, j) = CX(CF2, i, 0, j) +
                    p->ri[n] * p->grav_y *
                        (CX(CTHn, i, 0, j) * s->DYF[j - 1] + CX(CTHn, i, 0, j - 1) * s->DYF[j]) /
                        (2.0 * s->DY[j]);
        }
#pragma omp parallel for num_threads(nthreads())
        for (int j = JSTART; j <= JEND; ++j)
            for (int k = 0; k <= TNKZ; ++k)
                for (int i = 0; i <= NXP - 1; ++i) {
                    CX(CF1, i, k, j) = CX(CF1, i, k, j) + p->ri[n] * p->grav_x * CX(CTHn, i, k, j);
                }
#pragma omp parallel for num_threads(nthreads())
        for (int j = JSTART; j <= JEND; ++j)
            for (int k = 0; k <= TNKZ; ++k)
                for (int i = 0; i <= NXP - 1; ++i)
                    CX(CF3, i, k, j) = CX(CF3, i, k, j) + p->ri[n] * p->grav_z * CX(CTHn, i, k, j);
        /* scalar RHS (channel.f:254-290) */
        const int j0 = s->JSTART_TH[n], j1 = s->JEND_TH[n];
#pragma omp parallel for num_threads(nthreads())
        for (int j = j0; j <= j1; ++j)
            for (int k = 0; k <= TNKZ; ++k)
                for (int i = 0; i <= NXP - 1; ++i) CX(CRTHn, i, k, j) = CX(CTHn, i, k, j);
        if (rk_step > 1) {
#pragma omp parallel for num_threads(nthreads())
            for (int j = j0; j <= j1; ++j)
                for (int k = 0; k <= TNKZ; ++k)
                    for (int i = 0; i <= NXP - 1; ++i)
                        CX(CRTHn, i, k, j) = CX(CRTHn, i, k, j) + TEMP3 * CX(CFTHn, i, k, j);
        }
#pragma omp parallel for num_threads(nthreads())
        for (int j = j0; j <= j1; ++j)
            for (int k = 0; k <= TNKZ; ++k)
                for (int i = 0; i <= NXP - 1; ++i)
                    CX(CFTHn, i, k, j) = -(p->nu / p->pr[n]) * pow(s->KX2[i] + s->KZ2[k], p->beta) *
                                         CX(CTHn, i, k, j);
#pragma omp parallel for num_threads(nthreads())
        for (int j = j0; j <= j1; ++j)
            for (int k = 0; k <= TNKZ; ++k)
                for (int i = 0; i <= NXP - 1; ++i)
                    CX(CFTHn, i, k, j) = CX(CFTHn, i, k, j) - CX(CU1, i, k, j) * p->drhodx[n] -
                                         CX(CU3, i, k, j) * p->drhodz[n];
    }
    /* USER_RHS_CHAN_FOURIER (user_rhs.f:77-121): CU in Fourier space, CF the
     * Fourier right-hand sides so far */
    if (s->user_fn[0]) s->user_fn[0](s->user_data[0]);
    if (p->les && (!p->create_new_flow || s->TIME_STEP > 100)) {
        /* LES branch (channel.f:303-384): subgrid stress into CF, U to
         * physical space, physical BCs re-applied, then the explicit
         * horizontal eddy diffusivity of every scalar with KAPPA_T = NU_T */
        les_chan(s);
        apply_bc_vel_phys(s);
        for (int n = 0; n < s->NTH; ++n) {
            const double* CTHn = s->CTH + (size_t)n * s->nreal;
            double* CFTHn = s->CFTH + (size_t)n * s->nreal;
            for (int c = 0; c < 2; ++c) {
#pragma omp parallel for num_threads(nthreads())
                for (int j = 1; j <= NY + 1; ++j)
                    for (int k = 0; k <= TNKZ; ++k)
                        for (int i = 0; i <= NXP - 1; ++i)
                            CX(CS1, i, k, j) = CI * (c == 0 ? s->KX[i] : s->KZ[k]) * CX(CTHn, i, k, j);
                orc_fft_xz_to_physical(s, CS1, S1, 0, NY + 1);
#pragma omp parallel for num_threads(nthreads())
                for (int j = 1; j <= NY + 1; ++j)
                    for (int k = 0; k <= NZP - 1; ++k)
                        for (int i = 0; i <= NXM; ++i) PH(S1, i, k, j) = PH(s->NU_T, i, k, j) * PH(S1, i, k, j);
                orc_fft_xz_to_fourier(s, S1, CS1, 0, NY + 1);
#pragma omp parallel for num_threads(nthreads())
                for (int j = s->JSTART_TH[n]; j <= s->JEND_TH[n]; ++j)
                    for (int k = 0; k <= TNKZ; ++k)
                        for (int i = 0; i <= NXP - 1; ++i)
                            CX(CFTHn, i, k, j) =
                                CX(CFTHn, i, k, j) + CI * (c == 0 ? s->KX[i] : s->KZ[k]) * CX(CS1, i, k, j);
            }
        }
    } else {
        /* non-LES branch: transforms to physical space (channel.f:389-391) */
        orc_fft_xz_to_physical(s, CU1, U1, 0, NY + 1);
        orc_fft_xz_to_physical(s, CU2, U2, 0, NY + 1);
        orc_fft_xz_to_physical(s, CU3, U3, 0, NY + 1);
    }
    /* scalars to physical space (channel.f:380-384, 394-398) */
    for (int n = 0; n < s->NTH; ++n) {
        memcpy(CS1, s->CTH + (size_t)n * s->nreal, sizeof(double) * s->nreal);
        orc_fft_xz_to_physical(s, CS1, S1, 0, NY + 1);
        memcpy(s->TH + (size_t)n * s->nreal, S1, sizeof(double) * s->nreal);
    }

    /* nonlinear terms, one product at a time (channel.f:410-571) */
#define PRODUCT(J0, J1, EXPR)                                                  \
    do {                                                                       \
        _Pragma("omp parallel for num_threads(nthreads())")                    \
        for (int j = (J0); j <= (J1); ++j)                                     \
            for (int k = 0; k <= NZP - 1; ++k)                                 \
                for (int i = 0; i <= NXM; ++i) PH(S1, i, k, j) = (EXPR);       \
        orc_fft_xz_to_fourier(s, S1, CS1, 0, NY + 1);                          \
    } while (0)
#define ACCUM(J0, J1, STMT)                                                    \
    do {                                                                       \
        _Pragma("omp parallel for num_threads(nthreads())")                    \
        for (int j = (J0); j <= (J1); ++j)                                     \
            for (int k = 0; k <= TNKZ; ++k)                                    \
                for (int i = 0; i <= NXP - 1; ++i) { STMT; }                   \
    } while (0)
    const double* DY = s->DY;
    const double* DYF = s->DYF;
    /* U1*U3 */
    PRODUCT(JSTART, JEND, PH(U3, i, k, j) * PH(U1, i, k, j));
    ACCUM(JSTART, JEND,
          CX(CF1, i, k, j) = CX(CF1, i, k, j) - CI * s->KZ[k] * CX(CS1, i, k, j);
          CX(CF3, i, k, j) = CX(CF3, i, k, j) - CI * s->KX[i] * CX(CS1, i, k, j));
    /* U1*U1 */
    PRODUCT(JSTART, JEND, PH(U1, i, k, j) * PH(U1, i, k, j));
    ACCUM(JSTART, JEND, CX(CF1, i, k, j) = CX(CF1, i, k, j) - CI * s->KX[i] * CX(CS1, i, k, j));
    /* U3*U3 */
    PRODUCT(JSTART, JEND, PH(U3, i, k, j) * PH(U3, i, k, j));
    ACCUM(JSTART, JEND, CX(CF3, i, k, j) = CX(CF3, i, k, j) - CI * s->KZ[k] * CX(CS1, i, k, j));
    /* U1*U2 (U1 interpolated to GY) */
    PRODUCT(2, NY, ((DYF[j] * PH(U1, i, k, j) + DYF[j - 1] * PH(U1, i, k, j - 1)) / (2. * DY[j])) *
                       PH(U2, i, k, j));
    ACCUM(2, NY, CX(CF2, i, k, j) = CX(CF2, i, k, j) - CI * s->KX[i] * CX(CS1, i, k, j));
    /* U3*U2 */
    PRODUCT(2, NY, ((DYF[j] * PH(U3, i, k, j) + DYF[j - 1] * PH(U3, i, k, j - 1)) / (2. * DY[j])) *
                       PH(U2, i, k, j));
    ACCUM(2, NY, CX(CF2, i, k, j) = CX(CF2, i, k, j) - CI * s->KZ[k] * CX(CS1, i, k, j));
    /* d/dy(U1 U2) */
    PRODUCT(JSTART, JEND,
            (PH(U1, i, k, j + 1) * PH(U2, i, k, j + 1) + PH(U1, i, k, j) * PH(U2, i, k, j + 1) -
             PH(U1, i, k, j) * PH(U2, i, k, j) - PH(U1, i, k, j - 1) * PH(U2, i, k, j)) /
                (2.0 * DYF[j]));
    ACCUM(JSTART, JEND, CX(CF1, i, k, j) = CX(CF1, i, k, j) - CX(CS1, i, k, j));
    /* d/dy(U3 U2) */
    PRODUCT(JSTART, JEND,
            (PH(U3, i, k, j + 1) * PH(U2, i, k, j + 1) + PH(U3, i, k, j) * PH(U2, i, k, j + 1) -
             PH(U3, i, k, j) * PH(U2, i, k, j) - PH(U3, i, k, j - 1) * PH(U2, i, k, j)) /
                (2.0 * DYF[j]));
    ACCUM(JSTART, JEND, CX(CF3, i, k, j) = CX(CF3, i, k, j) - CX(CS1, i, k, j));
    /* d/dy(U2 U2) */
    PRODUCT(2, NY,
            (0.25 * pow(PH(U2, i, k, j) + PH(U2, i, k, j + 1), 2.0) -
             0.25 * pow(PH(U2, i, k, j) + PH(U2, i, k, j - 1), 2.0)) /
                DY[j]);
    ACCUM(2, NY, CX(CF2, i, k, j) = CX(CF2, i, k, j) - CX(CS1, i, k, j));
    /* USER_RHS_CHAN_PHYSICAL (user_rhs.f:1-74): U1..U3, TH in physical space,
     * CF in Fourier space */
    if (s->user_fn[1]) s->user_fn[1](s->user_data[1]);

    /* CR += beta h CF (channel.f:581-595) */
#pragma omp parallel for num_threads(nthreads())
    for (int j = JSTART; j <= JEND; ++j)
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) {
                CX(CR1, i, k, j) = CX(CR1, i, k, j) + TEMP5 * CX(CF1, i, k, j);
                CX(CR3, i, k, j) = CX(CR3, i, k, j) + TEMP5 * CX(CF3, i, k, j);
            }
#pragma omp parallel for num_threads(nthreads())
    for (int j = 2; j <= NY; ++j)
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i)
                CX(CR2, i, k, j) = CX(CR2, i, k, j) + TEMP5 * CX(CF2, i, k, j);
    orc_fft_xz_to_physical(s, CR1, R1, 0, NY + 1);
    orc_fft_xz_to_physical(s, CR2, R2, 2, NY);
    orc_fft_xz_to_physical(s, CR3, R3, 0, NY + 1);
    /* explicit half of CN in y (channel.f:606-626) */
    const double nuv = p->nu_v_scale;
#pragma omp parallel for num_threads(nthreads())
    for (int j = JSTART; j <= JEND; ++j)
        for (int k = 0; k <= NZP - 1; ++k)
            for (int i = 0; i <= NXM; ++i) {
                PH(R1, i, k, j) = PH(R1, i, k, j) + TEMP1 * nuv *
                    (((PH(U1, i, k, j + 1) - PH(U1, i, k, j)) / DY[j + 1] -
                      (PH(U1, i, k, j) - PH(U1, i, k, j - 1)) / DY[j]) / DYF[j]);
                PH(R3, i, k, j) = PH(R3, i, k, j) + TEMP1 * nuv *
                    (((PH(U3, i, k, j + 1) - PH(U3, i, k, j)) / DY[j + 1] -
                      (PH(U3, i, k, j) - PH(U3, i, k, j - 1)) / DY[j]) / DYF[j]);
            }
#pragma omp parallel for num_threads(nthreads())
    for (int j = 2; j <= NY; ++j)
        for (int k = 0; k <= NZP - 1; ++k)
            for (int i = 0; i <= NXM; ++i)
                PH(R2, i, k, j) = PH(R2, i, k, j) + TEMP1 * nuv *
                    (((PH(U2, i, k, j + 1) - PH(U2, i, k, j)) / DYF[j] -
                      (PH(U2, i, k, j) - PH(U2, i, k, j - 1)) / DYF[j - 1]) / DY[j]);
    if (p->les) {
        /* eddy-viscosity part of the explicit CN half, NU_T at GY points
         * (channel.f:631-660) */
        const double* NU_T = s->NU_T;
#pragma omp parallel for num_threads(nthreads())
        for (int j = JSTART; j <= JEND; ++j)
            for (int k = 0; k <= NZP - 1; ++k)
                for (int i = 0; i <= NXM; ++i) {
                    PH(R1, i, k, j) = PH(R1, i, k, j) + TEMP2 *
                        ((PH(NU_T, i, k, j + 1) * (PH(U1, i, k, j + 1) - PH(U1, i, k, j)) / DY[j + 1] -
                          PH(NU_T, i, k, j) * (PH(U1, i, k, j) - PH(U1, i, k, j - 1)) / DY[j]) / DYF[j]);
                    PH(R3, i, k, j) = PH(R3, i, k, j) + TEMP2 *
                        ((PH(NU_T, i, k, j + 1) * (PH(U3, i, k, j + 1) - PH(U3, i, k, j)) / DY[j + 1] -
                          PH(NU_T, i, k, j) * (PH(U3, i, k, j) - PH(U3, i, k, j - 1)) / DY[j]) / DYF[j]);
                }
#pragma omp parallel for num_threads(nthreads())
        for (int j = 2; j <= NY; ++j)
            for (int k = 0; k <= NZP - 1; ++k)
                for (int i = 0; i <= NXM; ++i)
                    PH(R2, i, k, j) = PH(R2, i, k, j) + TEMP2 *
                        ((0.5 * (PH(NU_T, i, k, j) + PH(NU_T, i, k, j + 1)) * (PH(U2, i, k, j + 1) - PH(U2, i, k, j)) /
                              DYF[j] -
                          0.5 * (PH(NU_T, i, k, j) + PH(NU_T, i, k, j - 1)) * (PH(U2, i, k, j) - PH(U2, i, k, j - 1)) /
                              DYF[j - 1]) / DY[j]);
    }

    /* scalars (channel.f:666-840) */
    for (int n = 0; n < s->NTH; ++n) {
        double* THn = s->TH + (size_t)n * s->nreal;
        double* CFTHn = s->CFTH + (size_t)n * s->nreal;
        double* CRTHn = s->CRTH + (size_t)n * s->nreal;
        double* RTHn = s->RTH + (size_t)n * s->nreal;
        const int j0 = s->JSTART_TH[n], j1 = s->JEND_TH[n];
        PRODUCT(j0, j1, PH(THn, i, k, j) * PH(U1, i, k, j));
        ACCUM(j0, j1, CX(CFTHn, i, k, j) = CX(CFTHn, i, k, j) - CI * s->KX[i] * CX(CS1, i, k, j));
        PRODUCT(j0, j1, PH(THn, i, k, j) * PH(U3, i, k, j));
        ACCUM(j0, j1, CX(CFTHn, i, k, j) = CX(CFTHn, i, k, j) - CI * s->KZ[k] * CX(CS1, i, k, j));
        PRODUCT(j0, j1,
                (PH(THn, i, k, j + 1) * PH(U2, i, k, j + 1) + PH(THn, i, k, j) * PH(U2, i, k, j + 1) -
                 PH(THn, i, k, j) * PH(U2, i, k, j) - PH(THn, i, k, j - 1) * PH(U2, i, k, j)) /
                    (2.0 * DYF[j]));
        ACCUM(j0, j1, CX(CFTHn, i, k, j) = CX(CFTHn, i, k, j) - CX(CS1, i, k, j));
        ACCUM(j0, j1, CX(CRTHn, i, k, j) = CX(CRTHn, i, k, j) + TEMP5 * CX(CFTHn, i, k, j));
        memcpy(CS1, CRTHn, sizeof(double) * s->nreal);
        orc_fft_xz_to_physical(s, CS1, S1, 0, NY + 1);
        memcpy(RTHn, S1, sizeof(double) * s->nreal);
        const double c = (TEMP1 / p->pr[n]) * nuv;
#pragma omp parallel for num_threads(nthreads())
        for (int j = j0; j <= j1; ++j)
            for (int k = 0; k <= NZP - 1; ++k)
                for (int i = 0; i <= NXM; ++i)
                    PH(RTHn, i, k, j) = PH(RTHn, i, k, j) + c *
                        (((PH(THn, i, k, j + 1) - PH(THn, i, k, j)) / DY[j + 1] -
                          (PH(THn, i, k, j) - PH(THn, i, k, j - 1)) / DY[j]) / DYF[j]);
        if (p->les) {
            /* eddy diffusivity KAPPA_T = NU_T (channel.f:748-760) */
            const double* K = s->NU_T;
#pragma omp parallel for num_threads(nthreads())
            for (int j = j0; j <= j1; ++j)
                for (int k = 0; k <= NZP - 1; ++k)
                    for (int i = 0; i <= NXM; ++i)
                        PH(RTHn, i, k, j) = PH(RTHn, i, k, j) + TEMP2 *
                            ((PH(K, i, k, j + 1) * (PH(THn, i, k, j + 1) - PH(THn, i, k, j)) / DY[j + 1] -
                              PH(K, i, k, j) * (PH(THn, i, k, j) - PH(THn, i, k, j - 1)) / DY[j]) / DYF[j]);
        }
        cn_solve(s, SOLVE_TH, n, TEMP1, TEMP2);
    }
#undef PRODUCT
#undef ACCUM
    /* velocity solves: U2, U1, U3 (channel.f:842-1029) */
    cn_solve(s, SOLVE_U2, 0, TEMP1, TEMP2);
    cn_solve(s, SOLVE_U1, 0, TEMP1, TEMP2);
    cn_solve(s, SOLVE_U3, 0, TEMP1, TEMP2);
    /* CFL (channel.f:1037-1040) */
    if (p->variable_dt && rk_step == 3 && (s->TIME_STEP % p->update_dt) == 0) orc_courant(s);
    /* back to Fourier space (channel.f:1043-1050) */
    orc_fft_xz_to_fourier(s, U1, CU1, 0, NY + 1);
    orc_fft_xz_to_fourier(s, U2, CU2, 0, NY + 1);
    orc_fft_xz_to_fourier(s, U3, CU3, 0, NY + 1);
    for (int n = 0; n < s->NTH; ++n) {
        memcpy(S1, s->TH + (size_t)n * s->nreal, sizeof(double) * s->nreal);
        orc_fft_xz_to_fourier(s, S1, CS1, 0, NY + 1);
        memcpy(s->CTH + (size_t)n * s->nreal, CS1, sizeof(double) * s->nreal);
    }
    orc_rem_div_chan(s);
    /* pressure update with phi in CR1 (channel.f:1059-1065) */
#pragma omp parallel for num_threads(nthreads())
    for (int j = JSTART; j <= JEND; ++j)
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i)
                CX(CP, i, k, j) = CX(CP, i, k, j) + CX(CR1, i, k, j) / TEMP4;
    /* GHOST_CHAN_MPI: no-op for NPROCY = 1 */
}

/* ------------------------------------------------------------------------ */
/* REM_DIV_CHAN (channel.f:1103-1214) with APPLY_BC_REM_DIV_MPI               */
/* (mpi.f:1239-1278) and the complex MPI Thomas.  phi -> CR1 (J = 1..NY).     */
/* ------------------------------------------------------------------------ */
void orc_rem_div_chan(orc_state* s) {
    const int NY = s->NY, NXP = s->NXP, TNKZ = s->TNKZ;
    double *CU1 = s->U1, *CU2 = s->U2, *CU3 = s->U3, *CR1 = s->R1;
    const int ld = NXP + 1;
    const size_t msz = (size_t)ld * (NY + 2);
#define MC(a, i, j) (a)[(size_t)(i) + (size_t)ld * (size_t)(j)]
#pragma omp parallel num_threads(nthreads())
    {
        double* A = (double*)malloc(sizeof(double) * msz);
        double* B = (double*)malloc(sizeof(double) * msz);
        double* C = (double*)malloc(sizeof(double) * msz);
        cplx* G = (cplx*)malloc(sizeof(cplx) * msz);
        /* Column I = NXP is never initialised by the reference (local array,
         * loops to NXP-1) yet is swept by the MPI Thomas; its result is never
         * copied out.  Zero/identity here keeps it inert. */
        for (size_t q = 0; q < msz; ++q) { A[q] = 0.0; B[q] = 1.0; C[q] = 0.0; G[q] = 0.0; }
#pragma omp for schedule(static)
        for (int k = 0; k <= TNKZ; ++k) {
            for (int j = 1; j <= NY; ++j)
                for (int i = 0; i <= NXP - 1; ++i) {
                    MC(A, i, j) = 1. / (s->DY[j] * s->DYF[j]);
                    MC(B, i, j) = -s->KX2[i] - s->KZ2[k] - 1. / (s->DY[j + 1] * s->DYF[j]) -
                                  1. / (s->DY[j] * s->DYF[j]);
                    MC(C, i, j) = 1. / (s->DY[j + 1] * s->DYF[j]);
                }
            for (int j = 1; j <= NY; ++j)
                for (int i = 0; i <= NXP - 1; ++i)
                    MC(G, i, j) = I * s->KX[i] * CX(CU1, i, k, j) +
                                  (CX(CU2, i, k, j + 1) - CX(CU2, i, k, j)) / s->DYF[j] +
                                  I * s->KZ[k] * CX(CU3, i, k, j);
            for (int i = 0; i <= NXP - 1; ++i) {
                if (k == 0 && i == 0) {
                    MC(A, i, 1) = 0.; MC(B, i, 1) = 1.; MC(C, i, 1) = 0.; MC(G, i, 1) = 0.;
                } else {
                    MC(A, i, 1) = 0.; MC(B, i, 1) = 1.; MC(C, i, 1) = -1.; MC(G, i, 1) = 0.;
                }
                MC(A, i, NY) = 1.; MC(B, i, NY) = -1.; MC(C, i, NY) = 0.; MC(G, i, NY) = 0.;
            }
            thomas_complex_mpi(A, B, C, G, NY, NXP);
            for (int j = 1; j <= NY; ++j)
                for (int i = 0; i <= NXP - 1; ++i) CX(CR1, i, k, j) = MC(G, i, j);
        }
        free(A); free(B); free(C); free(G);
    }
#undef MC
#pragma omp parallel for num_threads(nthreads())
    for (int j = 1; j <= NY; ++j)
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) {
                CX(CU1, i, k, j) = CX(CU1, i, k, j) - I * s->KX[i] * CX(CR1, i, k, j);
                CX(CU3, i, k, j) = CX(CU3, i, k, j) - I * s->KZ[k] * CX(CR1, i, k, j);
            }
#pragma omp parallel for num_threads(nthreads())
    for (int j = 2; j <= NY; ++j)
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i)
                CX(CU2, i, k, j) = CX(CU2, i, k, j) - (CX(CR1, i, k, j) - CX(CR1, i, k, j - 1)) / s->DY[j];
}

/* ------------------------------------------------------------------------ */
/* POISSON_P_CHAN (channel.f:1217-1453) with APPLY_BC_POISSON_MPI             */
/* (mpi.f:1280-1315).                                                         */
/* ------------------------------------------------------------------------ */
void orc_poisson_p_chan(orc_state* s) {
    const int NY = s->NY, NXP = s->NXP, TNKZ = s->TNKZ, NZP = s->NZP, NXM = s->NXM;
    double *CU1 = s->U1, *CU2 = s->U2, *CU3 = s->U3, *CP = s->P;
    double *CF1 = s->F1, *CF2 = s->F2, *CF3 = s->F3, *CS1 = s->S1;
    double *F1 = s->F1, *F2 = s->F2, *F3 = s->F3;
    const double* DYF = s->DYF;
#define LOOPF(STMT)                                                           \
    _Pragma("omp parallel for num_threads(nthreads())")                       \
    for (int j = 2; j <= NY; ++j)                                             \
        for (int k = 0; k <= TNKZ; ++k)                                       \
            for (int i = 0; i <= NXP - 1; ++i) { STMT; }
#define LOOPP(STMT)                                                           \
    _Pragma("omp parallel for num_threads(nthreads())")                       \
    for (int j = 2; j <= NY; ++j)                                             \
        for (int k = 0; k <= NZP - 1; ++k)                                    \
            for (int i = 0; i <= NXM; ++i) { STMT; }
    LOOPF(CX(CF1, i, k, j) = I * s->KX[i] * CX(CU1, i, k, j);
          CX(CF2, i, k, j) = (CX(CU2, i, k, j + 1) - CX(CU2, i, k, j)) / DYF[j];
          CX(CF3, i, k, j) = I * s->KZ[k] * CX(CU3, i, k, j));
    orc_fft_xz_to_physical(s, CF1, F1, 0, NY + 1);
    orc_fft_xz_to_physical(s, CF2, F2, 0, NY + 1);
    orc_fft_xz_to_physical(s, CF3, F3, 0, NY + 1);
    LOOPP(PH(F1, i, k, j) = pow(PH(F1, i, k, j), 2.); PH(F2, i, k, j) = pow(PH(F2, i, k, j), 2.);
          PH(F3, i, k, j) = pow(PH(F3, i, k, j), 2.));
    orc_fft_xz_to_fourier(s, F1, CF1, 0, NY + 1);
    orc_fft_xz_to_fourier(s, F2, CF2, 0, NY + 1);
    orc_fft_xz_to_fourier(s, F3, CF3, 0, NY + 1);
    LOOPF(CX(CS1, i, k, j) = CX(CF1, i, k, j) + CX(CF2, i, k, j) + CX(CF3, i, k, j));
    LOOPF(CX(CF1, i, k, j) = (CX(CU1, i, k, j + 1) - CX(CU1, i, k, j - 1)) / (2. * DYF[j]);
          CX(CF2, i, k, j) = I * s->KX[i] * 0.5 * (CX(CU2, i, k, j) + CX(CU2, i, k, j + 1)));
    orc_fft_xz_to_physical(s, CF1, F1, 0, NY + 1);
    orc_fft_xz_to_physical(s, CF2, F2, 0, NY + 1);
    LOOPP(PH(F1, i, k, j) = 2. * PH(F1, i, k, j) * PH(F2, i, k, j));
    orc_fft_xz_to_fourier(s, F1, CF1, 0, NY + 1);
    LOOPF(CX(CS1, i, k, j) = CX(CS1, i, k, j) + CX(CF1, i, k, j));
    LOOPF(CX(CF1, i, k, j) = (CX(CU3, i, k, j + 1) - CX(CU3, i, k, j - 1)) / (2. * DYF[j]);
          CX(CF2, i, k, j) = I * s->KZ[k] * 0.5 * (CX(CU2, i, k, j) + CX(CU2, i, k, j + 1)));
    orc_fft_xz_to_physical(s, CF1, F1, 0, NY + 1);
    orc_fft_xz_to_physical(s, CF2, F2, 0, NY + 1);
    LOOPP(PH(F1, i, k, j) = 2. * PH(F1, i, k, j) * PH(F2, i, k, j));
    orc_fft_xz_to_fourier(s, F1, CF1, 0, NY + 1);
    LOOPF(CX(CS1, i, k, j) = CX(CS1, i, k, j) + CX(CF1, i, k, j));
    LOOPF(CX(CF1, i, k, j) = I * s->KZ[k] * CX(CU1, i, k, j);
          CX(CF2, i, k, j) = I * s->KX[i] * CX(CU3, i, k, j));
    orc_fft_xz_to_physical(s, CF1, F1, 0, NY + 1);
    orc_fft_xz_to_physical(s, CF2, F2, 0, NY + 1);
    LOOPP(PH(F1, i, k, j) = 2. * PH(F1, i, k, j) * PH(F2, i, k, j));
    orc_fft_xz_to_fourier(s, F1, CF1, 0, NY + 1);
    LOOPF(CX(CS1, i, k, j) = CX(CS1, i, k, j) + CX(CF1, i, k, j));
    for (int n = 0; n < s->NTH; ++n) {
        double* CTHn = s->CTH + (size_t)n * s->nreal;
        LOOPF(if (i != 0 || k != 0) CX(CS1, i, k, j) = CX(CS1, i, k, j) +
                  s->p.ri[n] * (CX(CTHn, i, k, j + 1) - CX(CTHn, i, k, j - 1)) /
                      (s->GYF[j + 1] - s->GYF[j - 1]));
    }
#undef LOOPF
#undef LOOPP
    const int ld = NXP + 1;
    const size_t msz = (size_t)ld * (NY + 2);
#define MC(a, i, j) (a)[(size_t)(i) + (size_t)ld * (size_t)(j)]
#pragma omp parallel num_threads(nthreads())
    {
        double* A = (double*)malloc(sizeof(double) * msz);
        double* B = (double*)malloc(sizeof(double) * msz);
        double* C = (double*)malloc(sizeof(double) * msz);
        cplx* G = (cplx*)malloc(sizeof(cplx) * msz);
        for (size_t q = 0; q < msz; ++q) { A[q] = 0.0; B[q] = 1.0; C[q] = 0.0; G[q] = 0.0; }
#pragma omp for schedule(static)
        for (int k = 0; k <= TNKZ; ++k) {
            for (int j = 2; j <= NY; ++j)
                for (int i = 0; i <= NXP - 1; ++i) {
                    MC(A, i, j) = 1. / (s->DY[j] * s->DYF[j]);
                    MC(B, i, j) = -s->KX2[i] - s->KZ2[k] - 1. / (s->DY[j + 1] * s->DYF[j]) -
                                  1. / (s->DY[j] * s->DYF[j]);
                    MC(C, i, j) = 1. / (s->DY[j + 1] * s->DYF[j]);
                    MC(G, i, j) = -1. * CX(CS1, i, k, j);
                }
            for (int i = 0; i <= NXP - 1; ++i) {
                if (i == 0 && k == 0) {
                    MC(B, i, 1) = 1.; MC(C, i, 1) = 0.; MC(G, i, 1) = 0.;
                } else {
                    MC(B, i, 1) = 1.; MC(C, i, 1) = -1.; MC(G, i, 1) = 0.;
                }
                MC(B, i, NY) = -1.; MC(A, i, NY) = 1.; MC(G, i, NY) = 0.;
            }
            thomas_complex_mpi(A, B, C, G, NY, NXP);
            for (int j = 1; j <= NY; ++j)
                for (int i = 0; i <= NXP - 1; ++i) CX(CP, i, k, j) = MC(G, i, j);
        }
        free(A); free(B); free(C); free(G);
    }
#undef MC
}

/* ------------------------------------------------------------------------ */
/* COURANT (courant.f:1-66) on the physical velocity.                          */
/* ------------------------------------------------------------------------ */
void orc_courant(orc_state* s) {
    const diablo_params* p = &s->p;
    double dt = 999.0;
    /* dx(1), dy(1): DX is uniform (channel.f:1566-1570) */
    dt = fmin(dt, 0.5 * pow(fmin(s->DX, s->DY[1]), 2.0) / p->nu);
    for (int n = 0; n < s->NTH; ++n) dt = fmin(dt, dt * p->nu / (p->nu / p->pr[n]));
    if (p->i_ro != 0.0) dt = fmin(dt, 2.0 * s->PI / fabs(p->i_ro) / 20.0);
    for (int n = 0; n < s->NTH; ++n)
        if (p->ri[n] != 0.0) {
            const double Nmax = sqrt(fabs(p->ri[n] * p->th_bc_ymin_c1[n]));
            /* 0.1 is a default-real (single precision) literal in courant.f:32 */
            dt = fmin(dt, (double)0.1f * 2.0 * s->PI / Nmax);
        }
    double dtv = dt;
#pragma omp parallel for reduction(min : dtv) num_threads(nthreads())
    for (int j = 1; j <= s->NY; ++j)
        for (int k = 0; k <= s->NZP - 1; ++k)
            for (int i = 0; i <= s->NXM; ++i) {
                const double dt_x = p->cfl * s->DX / fabs(PH(s->U1, i, k, j));
                const double dt_y = p->cfl * s->DY[j] / fabs(PH(s->U2, i, k, j));
                const double dt_z = p->cfl * s->DZ / fabs(PH(s->U3, i, k, j));
                dtv = fmin(dtv, fmin(dt_x, fmin(dt_y, dt_z)));
            }
    dt = dtv;
    if (dt <= 0) s->DELTA_T = 0.0001;
    else if (dt >= 999.) s->DELTA_T = 999.0;
    else s->DELTA_T = dt;
    s->H_BAR[0] = s->DELTA_T * (8.0 / 15.0);
    s->H_BAR[1] = s->DELTA_T * (2.0 / 15.0);
    s->H_BAR[2] = s->DELTA_T * (5.0 / 15.0);
}

/* ------------------------------------------------------------------------ */
/* APPLY_BC_VEL_LOWER / _UPPER (channel.f:2285-2492), Fourier space.          */
/* ------------------------------------------------------------------------ */
void orc_apply_bc_vel(orc_state* s) {
    const int NY = s->NY, NXP = s->NXP, TNKZ = s->TNKZ;
    const diablo_params* p = &s->p;
    double *CU1 = s->U1, *CU2 = s->U2, *CU3 = s->U3;
    const double* DY = s->DY;
    const double* DYF = s->DYF;
    /* lower */
    if (p->u_bc_ymin == 0) {
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) { CX(CU1, i, k, 0) = 0; CX(CU1, i, k, 1) = 0; }
        CX(CU1, 0, 0, 1) = p->u_bc_ymin_c1;
        CX(CU1, 0, 0, 0) = p->u_bc_ymin_c1;
    } else {
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) {
                CX(CU1, i, k, 1) = CX(CU1, i, k, 2);
                CX(CU1, i, k, 0) = CX(CU1, i, k, 1);
            }
        CX(CU1, 0, 0, 1) = CX(CU1, 0, 0, 2) - DY[2] * p->u_bc_ymin_c1;
        CX(CU1, 0, 0, 0) = CX(CU1, 0, 0, 1) - DY[1] * p->u_bc_ymin_c1;
    }
    if (p->w_bc_ymin == 0) {
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) { CX(CU3, i, k, 0) = 0; CX(CU3, i, k, 1) = 0; }
        CX(CU3, 0, 0, 1) = p->w_bc_ymin_c1;
        CX(CU3, 0, 0, 0) = p->w_bc_ymin_c1;
    } else {
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) {
                CX(CU3, i, k, 1) = CX(CU3, i, k, 2);
                CX(CU3, i, k, 0) = CX(CU3, i, k, 1);
            }
        CX(CU3, 0, 0, 1) = CX(CU3, 0, 0, 2) - DY[2] * p->w_bc_ymin_c1;
        CX(CU3, 0, 0, 0) = CX(CU3, 0, 0, 1) - DY[1] * p->w_bc_ymin_c1;
    }
    if (p->v_bc_ymin == 0) {
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) {
                CX(CU2, i, k, 1) = 2.0 * p->v_bc_ymin_c1 - CX(CU2, i, k, 2);
                CX(CU2, i, k, 0) = CX(CU2, i, k, 1);
            }
    } else if (p->v_bc_ymin == 1) {
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) {
                CX(CU2, i, k, 1) = CX(CU2, i, k, 2);
                CX(CU2, i, k, 0) = CX(CU2, i, k, 1);
            }
        CX(CU2, 0, 0, 1) = CX(CU2, 0, 0, 2) - DYF[1] * p->v_bc_ymin_c1;
        CX(CU2, 0, 0, 0) = CX(CU2, 0, 0, 1) - DYF[1] * p->v_bc_ymin_c1;
    } else if (p->v_bc_ymin == 2) {
        CX(CU2, 0, 0, 1) = -CX(CU2, 0, 0, 2);
    }
    /* upper */
    if (p->u_bc_ymax == 0) {
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) { CX(CU1, i, k, NY) = 0; CX(CU1, i, k, NY + 1) = 0; }
        CX(CU1, 0, 0, NY) = p->u_bc_ymax_c1;
        CX(CU1, 0, 0, NY + 1) = p->u_bc_ymax_c1;
    } else {
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) {
                CX(CU1, i, k, NY) = CX(CU1, i, k, NY - 1);
                CX(CU1, i, k, NY + 1) = CX(CU1, i, k, NY);
            }
        CX(CU1, 0, 0, NY) = CX(CU1, 0, 0, NY - 1) + DY[NY] * p->u_bc_ymax_c1;
        CX(CU1, 0, 0, NY + 1) = CX(CU1, 0, 0, NY) + DY[NY] * p->u_bc_ymax_c1;
    }
    if (p->w_bc_ymax == 0) {
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) { CX(CU3, i, k, NY) = 0; CX(CU3, i, k, NY + 1) = 0; }
        CX(CU3, 0, 0, NY) = p->w_bc_ymax_c1;
        CX(CU3, 0, 0, NY + 1) = p->w_bc_ymax_c1;
        CX(CU3, 0, 0, NY + 1) = 0.0;   /* "ghost cell not used" (channel.f:2434) */
    } else {
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) {
                CX(CU3, i, k, NY) = CX(CU3, i, k, NY - 1);
                CX(CU3, i, k, NY + 1) = CX(CU3, i, k, NY);
            }
        CX(CU3, 0, 0, NY) = CX(CU3, 0, 0, NY - 1) + DY[NY] * p->w_bc_ymax_c1;
        CX(CU3, 0, 0, NY + 1) = CX(CU3, 0, 0, NY) + DY[NY] * p->w_bc_ymax_c1;
    }
    if (p->v_bc_ymax == 0) {
        /* the reference loops over (k,i) but only ever writes the (0,0) entry
         * (channel.f:2463-2467) */
        CX(CU2, 0, 0, NY + 1) = 2.0 * p->v_bc_ymax_c1 - CX(CU2, 0, 0, NY);
    } else if (p->v_bc_ymax == 1) {
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) {
                CX(CU2, i, k, NY) = CX(CU2, i, k, NY - 1);
                CX(CU2, i, k, NY + 1) = CX(CU2, i, k, NY);
            }
        CX(CU2, 0, 0, NY + 1) = CX(CU2, 0, 0, NY) + DY[NY] * p->v_bc_ymax_c1;
    } else if (p->v_bc_ymax == 2) {
        CX(CU2, 0, 0, NY + 1) = -CX(CU2, 0, 0, NY);
    }
}

/* APPLY_BC_SCALAR_LOWER / _UPPER (channel.f:2723-2807). */
void orc_apply_bc_scalar(orc_state* s) {
    const int NY = s->NY, NXP = s->NXP, TNKZ = s->TNKZ;
    const diablo_params* p = &s->p;
    for (int n = 0; n < s->NTH; ++n) {
        double* C = s->CTH + (size_t)n * s->nreal;
        if (p->th_bc_ymin[n] == 0) {
            for (int k = 0; k <= TNKZ; ++k)
                for (int i = 0; i <= NXP - 1; ++i) { CX(C, i, k, 0) = 0; CX(C, i, k, 1) = 0; }
            CX(C, 0, 0, 1) = p->th_bc_ymin_c1[n];
            CX(C, 0, 0, 0) = p->th_bc_ymin_c1[n];
        } else {
            for (int k = 0; k <= TNKZ; ++k)
                for (int i = 0; i <= NXP - 1; ++i) {
                    CX(C, i, k, 1) = CX(C, i, k, 2);
                    CX(C, i, k, 0) = CX(C, i, k, 1);
                }
            CX(C, 0, 0, 1) = CX(C, 0, 0, 2) - s->DY[2] * p->th_bc_ymin_c1[n];
            CX(C, 0, 0, 0) = CX(C, 0, 0, 1) - s->DY[1] * p->th_bc_ymin_c1[n];
        }
        if (p->th_bc_ymax[n] == 0) {
            for (int k = 0; k <= TNKZ; ++k)
                for (int i = 0; i <= NXP - 1; ++i) { CX(C, i, k, NY) = 0; CX(C, i, k, NY + 1) = 0; }
            CX(C, 0, 0, NY) = p->th_bc_ymax_c1[n];
            CX(C, 0, 0, NY + 1) = p->th_bc_ymax_c1[n];
        } else {
            for (int k = 0; k <= TNKZ; ++k)
                for (int i = 0; i <= NXP - 1; ++i) {
                    CX(C, i, k, NY) = CX(C, i, k, NY - 1);
                    CX(C, i, k, NY + 1) = CX(C, i, k, NY);
                }
            CX(C, 0, 0, NY) = CX(C, 0, 0, NY - 1) + s->DY[NY] * p->th_bc_ymax_c1[n];
            CX(C, 0, 0, NY + 1) = CX(C, 0, 0, NY) + s->DY[NY] * p->th_bc_ymax_c1[n];
        }
    }
}

/* The time loop body of diablo.f:70-110 without statistics or I/O. */
void orc_step(orc_state* s) {
    s->TIME_STEP += 1;
    for (int rk = 1; rk <= 3; ++rk) orc_rk_chan_1(s, rk);
    s->TIME += s->DELTA_T;
}

/* ------------------------------------------------------------------------ */
/* SAVE_STATS_CHAN profiles (save_stats.f:104-347, 452-536).  Computed from   */
/* copies after APPLY_BC_VEL (save_stats.f:28-36), which is the only state    */
/* change kept; the reference's FFT round trips only add round-off.           */
/* ------------------------------------------------------------------------ */
void orc_stats(orc_state* s, double* out) {
    const int NY = s->NY, NX = s->NX, NZ = s->NZ, NZP = s->NZP, NXM = s->NXM;
    const size_t ny2 = (size_t)NY + 2;
    memset(out, 0, sizeof(double) * DIABLO_NSTATS * ny2);
    orc_apply_bc_vel(s);
    double* u[3];
    for (int c = 0; c < 3; ++c) {
        u[c] = (double*)malloc(sizeof(double) * s->nreal);
        memcpy(u[c], c == 0 ? s->U1 : c == 1 ? s->U2 : s->U3, sizeof(double) * s->nreal);
    }
    double *ume = out + DIABLO_STAT_UME * ny2, *vme = out + DIABLO_STAT_VME * ny2,
           *wme = out + DIABLO_STAT_WME * ny2;
    for (size_t j = 0; j < ny2; ++j) {
        ume[j] = creal(CX(s->U1, 0, 0, j));
        vme[j] = creal(CX(s->U2, 0, 0, j));
        wme[j] = creal(CX(s->U3, 0, 0, j));
        out[DIABLO_STAT_CP * ny2 + j] = creal(CX(s->P, 0, 0, j));
    }
    for (int c = 0; c < 3; ++c) orc_fft_xz_to_physical(s, u[c], u[c], 0, NY + 1);
    double* U1 = u[0]; double* U2 = u[1]; double* U3 = u[2];
    const double nn = (double)((float)NZ * (float)NX);
    for (int j = 1; j <= NY; ++j) {
        double ur = 0, vr = 0, wr = 0, uv = 0, wv = 0, uw = 0, sh = 0;
        for (int k = 0; k <= NZP - 1; ++k)
            for (int i = 0; i <= NXM; ++i) {
                ur += pow(PH(U1, i, k, j) - ume[j], 2.);
                vr += 0.5 * (pow(PH(U2, i, k, j) - vme[j], 2.) + pow(PH(U2, i, k, j + 1) - vme[j + 1], 2.));
                wr += pow(PH(U3, i, k, j) - wme[j], 2.);
                uv += (s->DYF[j - 1] * (PH(U1, i, k, j) - ume[j]) + s->DYF[j] * (PH(U1, i, k, j - 1) - ume[j - 1])) /
                      (2.0 * s->DY[j]) * (PH(U2, i, k, j) - vme[j]);
                wv += (s->DYF[j - 1] * (PH(U3, i, k, j) - wme[j]) + s->DYF[j] * (PH(U3, i, k, j - 1) - wme[j - 1])) /
                      (2.0 * s->DY[j]) * (PH(U2, i, k, j) - vme[j]);
                uw += (PH(U1, i, k, j) - ume[j]) * (PH(U3, i, k, j) - wme[j]);
                sh += pow((PH(U1, i, k, j + 1) - PH(U1, i, k, j - 1)) / (2.0 * s->DYF[j]), 2.0) +
                      pow((PH(U3, i, k, j + 1) - PH(U3, i, k, j - 1)) / (2.0 * s->DYF[j]), 2.0);
            }
        out[DIABLO_STAT_URMS * ny2 + j] = sqrt(ur / nn);
        out[DIABLO_STAT_VRMS * ny2 + j] = sqrt(vr / nn);
        out[DIABLO_STAT_WRMS * ny2 + j] = sqrt(wr / nn);
        out[DIABLO_STAT_UV * ny2 + j] = uv / nn;
        out[DIABLO_STAT_UW * ny2 + j] = uw / nn;
        out[DIABLO_STAT_WV * ny2 + j] = wv / nn;
        out[DIABLO_STAT_DUDY * ny2 + j] = (ume[j] - ume[j - 1]) / (s->GYF[j] - s->GYF[j - 1]);
        out[DIABLO_STAT_DWDY * ny2 + j] = (wme[j] - wme[j - 1]) / (s->GYF[j] - s->GYF[j - 1]);
        out[DIABLO_STAT_SHEAR * ny2 + j] = sh / (double)(NX * NZ);
    }
    if (s->NTH > 0) {
        double* th = (double*)malloc(sizeof(double) * s->nreal);
        memcpy(th, s->CTH, sizeof(double) * s->nreal);
        double* thme = out + DIABLO_STAT_THME * ny2;
        for (size_t j = 0; j < ny2; ++j) thme[j] = creal(CX(s->CTH, 0, 0, j));
        orc_fft_xz_to_physical(s, th, th, 0, NY + 1);
        for (int j = 1; j <= NY; ++j) {
            double a = 0, b = 0;
            for (int k = 0; k <= NZP - 1; ++k)
                for (int i = 0; i <= NXM; ++i) {
                    a += pow(fabs(PH(th, i, k, j) - thme[j]), 2.);
                    b += (PH(th, i, k, j) - thme[j]) *
                         (0.5 * (PH(U2, i, k, j) + PH(U2, i, k, j + 1)) - 0.5 * (vme[j] + vme[j + 1]));
                }
            out[DIABLO_STAT_THRMS * ny2 + j] = sqrt(a / nn);
            out[DIABLO_STAT_THV * ny2 + j] = b / nn;
            out[DIABLO_STAT_DTHDY * ny2 + j] = (thme[j] - thme[j - 1]) / (s->GYF[j] - s->GYF[j - 1]);
        }
        free(th);
    }
    for (int c = 0; c < 3; ++c) free(u[c]);
}

/* ------------------------------------------------------------------------ */
/* The remaining profiles of SAVE_STATS_CHAN's mean.h5 and tke.h5, after      */
/* orc_stats (which applies APPLY_BC_VEL):                                    */
/*  - rms vorticity (save_stats.f:270-347): each component formed from CR =   */
/*    CU on rows 1..NY, transformed, sqrt(sum S1^2 / (DBLE(NX) DBLE(NZ)));    */
/*  - per scalar (save_stats.f:452-536): thme, dthdy, thrms, thv and pe_diss, */
/*    the plane sum of |grad TH|^2 over DBLE(NX*NZ);                          */
/*  - epsilon of tkebudget_chan (save_stats.f:937-1135) on rows 2..NY-1, its  */
/*    nine terms in the reference's order.  Rows 1 and NY stay 0: there the   */
/*    reference reads rows of S1 / CS1 that earlier code left behind.         */
/* ------------------------------------------------------------------------ */
static void stats_field(orc_state* s, int kind, const double* C, double* out) {
    const int NY = s->NY, NXP = s->NXP, TNKZ = s->TNKZ;
    const cplx CI = I;
    memset(out, 0, sizeof(double) * s->nreal);
    for (int j = 1; j <= NY; ++j)
        for (int k = 0; k <= TNKZ; ++k)
            for (int i = 0; i <= NXP - 1; ++i) {
                const cplx ikx = CI * s->KX[i], ikz = CI * s->KZ[k];
                const double d2 = 2.0 * s->DYF[j];
                cplx v;
                switch (kind) {
                    case 0: v = (CX(s->U3, i, k, j + 1) - CX(s->U3, i, k, j - 1)) / d2 -
                                ikz * 0.5 * (CX(s->U2, i, k, j + 1) + CX(s->U2, i, k, j)); break;
                    case 1: v = ikz * CX(s->U1, i, k, j) - ikx * CX(s->U3, i, k, j); break;
                    case 2: v = ikx * 0.5 * (CX(s->U2, i, k, j + 1) + CX(s->U2, i, k, j)) -
                                (CX(s->U1, i, k, j + 1) - CX(s->U1, i, k, j - 1)) / d2; break;
                    case 3: v = ikx * CX(s->U1, i, k, j); break;
                    case 4: v = ikx * CX(s->U2, i, k, j); break;
                    case 5: v = ikx * CX(s->U3, i, k, j); break;
                    case 6: v = ikz * CX(s->U1, i, k, j); break;
                    case 7: v = ikz * CX(s->U2, i, k, j); break;
                    case 8: v = ikz * CX(s->U3, i, k, j); break;
                    case 9: v = ikx * CX(C, i, k, j); break;
                    case 10: v = (CX(C, i, k, j + 1) - CX(C, i, k, j - 1)) / (s->GYF[j + 1] - s->GYF[j - 1]); break;
                    default: v = ikz * CX(C, i, k, j); break;
                }
                CX(out, i, k, j) = v;
            }
    orc_fft_xz_to_physical(s, out, out, 0, NY + 1);
}

void orc_mean_stats(orc_state* s, double* chan, double* scal, double* eps) {
    const int NY = s->NY, NX = s->NX, NZ = s->NZ, NZP = s->NZP, NXM = s->NXM;
    const size_t ny2 = (size_t)NY + 2;
    double* base = (double*)malloc(sizeof(double) * DIABLO_NSTATS * ny2);
    orc_stats(s, base);
    memset(chan, 0, sizeof(double) * DIABLO_NMEAN * ny2);
    memcpy(chan, base, sizeof(double) * DIABLO_STAT_THME * ny2);
    const double* ume = base + DIABLO_STAT_UME * ny2;
    const double* vme = base + DIABLO_STAT_VME * ny2;
    const double* wme = base + DIABLO_STAT_WME * ny2;
    double* S1 = (double*)malloc(sizeof(double) * s->nreal);
    for (int c = 0; c < 3; ++c) {
        stats_field(s, c, NULL, S1);
        for (int j = 1; j <= NY; ++j) {
            double a = 0.0;
            for (int k = 0; k <= NZP - 1; ++k)
                for (int i = 0; i <= NXM; ++i) a += pow(PH(S1, i, k, j), 2.0);
            chan[(DIABLO_MEAN_OMEGA_X + c) * ny2 + j] = sqrt(a / ((double)NX * (double)NZ));
        }
    }
    double* u[3];
    for (int c = 0; c < 3; ++c) {
        u[c] = (double*)malloc(sizeof(double) * s->nreal);
        memcpy(u[c], c == 0 ? s->U1 : c == 1 ? s->U2 : s->U3, sizeof(double) * s->nreal);
        orc_fft_xz_to_physical(s, u[c], u[c], 0, NY + 1);
    }
    double *U1 = u[0], *U2 = u[1], *U3 = u[2];
    if (eps) {
        memset(eps, 0, sizeof(double) * ny2);
        double* e = (double*)calloc(ny2, sizeof(double));
        /* mode 0: S1(j)^2, 1: GYF values interpolated to GY */
        #define EPS_ADD(mode)                                                                          \
            for (int j = 2; j <= NY - 1; ++j)                                                          \
                for (int k = 0; k <= NZP - 1; ++k)                                                     \
                    for (int i = 0; i <= NXM; ++i)                                                     \
                        e[j] += (mode) ? (s->DYF[j - 1] * pow(PH(S1, i, k, j), 2.0) +                  \
                                          s->DYF[j] * pow(PH(S1, i, k, j - 1), 2.0)) / (2.0 * s->DY[j]) \
                                       : pow(PH(S1, i, k, j), 2.0);
        stats_field(s, 3, NULL, S1); EPS_ADD(1)                         /* du/dx */
        stats_field(s, 4, NULL, S1); EPS_ADD(0)                         /* dv/dx */
        for (int j = 2; j <= NY - 1; ++j)                               /* du/dy */
            for (int k = 0; k <= NZP - 1; ++k)
                for (int i = 0; i <= NXM; ++i)
                    e[j] += pow(((PH(U1, i, k, j) - ume[j]) - (PH(U1, i, k, j - 1) - ume[j - 1])) / s->DY[j], 2.0);
        stats_field(s, 5, NULL, S1); EPS_ADD(1)                         /* dw/dx */
        stats_field(s, 6, NULL, S1); EPS_ADD(1)                         /* du/dz */
        for (int j = 2; j <= NY - 1; ++j)                               /* dv/dy */
            for (int k = 0; k <= NZP - 1; ++k)
                for (int i = 0; i <= NXM; ++i)
                    e[j] += pow(((PH(U2, i, k, j + 1) - vme[j]) - (PH(U2, i, k, j - 1) - vme[j - 1])) /
                                    (s->GY[j + 1] - s->GY[j - 1]), 2.0);
        for (int j = 2; j <= NY - 1; ++j)                               /* dw/dy */
            for (int k = 0; k <= NZP - 1; ++k)
                for (int i = 0; i <= NXM; ++i)
                    e[j] += pow(((PH(U3, i, k, j) - wme[j]) - (PH(U3, i, k, j - 1) - wme[j - 1])) / s->DY[j], 2.0);
        stats_field(s, 7, NULL, S1); EPS_ADD(0)                         /* dv/dz */
        stats_field(s, 8, NULL, S1); EPS_ADD(1)                         /* dw/dz */
        #undef EPS_ADD
        for (int j = 2; j <= NY - 1; ++j) eps[j] = s->p.nu * e[j] / (double)(NX * NZ);
        free(e);
    }
    const double nn = (double)((float)NZ * (float)NX);
    double* th = (double*)malloc(sizeof(double) * s->nreal);
    double* R[3];
    for (int c = 0; c < 3; ++c) R[c] = (double*)malloc(sizeof(double) * s->nreal);
    for (int n = 0; n < s->NTH; ++n) {
        const double* C = s->CTH + (size_t)n * s->nreal;
        double* o = scal + (size_t)n * DIABLO_NSCAL * ny2;
        memset(o, 0, sizeof(double) * DIABLO_NSCAL * ny2);
        double* thme = o + DIABLO_SCAL_THME * ny2;
        for (size_t j = 0; j < ny2; ++j) thme[j] = creal(CX(C, 0, 0, j));
        for (int c = 0; c < 3; ++c) stats_field(s, 9 + c, C, R[c]);
        memcpy(th, C, sizeof(double) * s->nreal);
        orc_fft_xz_to_physical(s, th, th, 0, NY + 1);
        for (int j = 1; j <= NY; ++j) {
            double a = 0, b = 0, g = 0;
            for (int k = 0; k <= NZP - 1; ++k)
                for (int i = 0; i <= NXM; ++i) {
                    a += pow(fabs(PH(th, i, k, j) - thme[j]), 2.);
                    b += (PH(th, i, k, j) - thme[j]) *
                         (0.5 * (PH(U2, i, k, j) + PH(U2, i, k, j + 1)) - 0.5 * (vme[j] + vme[j + 1]));
                    g += pow(PH(R[0], i, k, j), 2.0) + pow(PH(R[1], i, k, j), 2.0) + pow(PH(R[2], i, k, j), 2.0);
                }
            o[DIABLO_SCAL_THRMS * ny2 + j] = sqrt(a / nn);
            o[DIABLO_SCAL_THV * ny2 + j] = b / nn;
            o[DIABLO_SCAL_DTHDY * ny2 + j] = (thme[j] - thme[j - 1]) / (s->GYF[j] - s->GYF[j - 1]);
            o[DIABLO_SCAL_PE_DISS * ny2 + j] = g / (double)(NX * NZ);
        }
    }
    for (int c = 0; c < 3; ++c) { free(R[c]); free(u[c]); }
    free(th); free(S1); free(base);
}

/* ------------------------------------------------------------------------ */
/* filter_chan(n) (filter.f:1-98) on scalar n (1..N_TH): a sharpened raised   */
/* cosine in the horizontal on every mode and rows J = 0..NY, then, for       */
/* I = 1..NKX and K = 1..TNKZ, the vertical compact filter with alpha = 0,    */
/* i.e. the explicit stencil of VEC_C on rows J = 2..NY-1 (rows 1 and NY keep  */
/* their values; the identity tridiagonal system returns VEC_C).  Row J = 0    */
/* keeps its horizontally filtered value: the reference copies an element of  */
/* VEC_C that it never sets there.                                            */
/* ------------------------------------------------------------------------ */
/* tkebudget_chan_les (save_stats.f:859-900): the plane sums, J = 1..NY, of
 * U_i times the implicit vertical eddy-viscosity term of U_i, on the
 * physical velocity after APPLY_BC_VEL (orc_stats applies it) and NU_T of
 * the last LES substage.  out: NY+2 values, rows 1..NY.  Row 1 is finite
 * where the reference's is NaN (FLUX below). */
/* tkebudget_chan's 3-D dissipation field F1 (save_stats.f:957-1131): NU times
 * the nine squared gradient terms at each point, GYF quantities
 * interpolated to GY, on rows 2..NY-1 (0 elsewhere: rows 1 and NY read rows
 * of S1 that earlier code left behind).  F1 in the physical layout. */
void orc_epsilon_field(orc_state* s, double* F1) {
    const int NY = s->NY, NZP = s->NZP, NXM = s->NXM;
    memset(F1, 0, sizeof(double) * s->nreal);
    double* base = (double*)malloc(sizeof(double) * DIABLO_NSTATS * (NY + 2));
    orc_stats(s, base);                         /* APPLY_BC_VEL on the state */
    const double* ume = base + DIABLO_STAT_UME * (NY + 2);
    const double* vme = base + DIABLO_STAT_VME * (NY + 2);
    const double* wme = base + DIABLO_STAT_WME * (NY + 2);
    double* u[3];
    for (int c = 0; c < 3; ++c) {
        u[c] = (double*)malloc(sizeof(double) * s->nreal);
        memcpy(u[c], c == 0 ? s->U1 : c == 1 ? s->U2 : s->U3, sizeof(double) * s->nreal);
        orc_fft_xz_to_physical(s, u[c], u[c], 0, NY + 1);
    }
    double* S1 = (double*)malloc(sizeof(double) * s->nreal);
    const int order[9] = {3, 4, -1, 5, 6, -2, -3, 7, 8};   /* tkebudget_chan's order of terms */
    for (int t = 0; t < 9; ++t) {
        const int kind = order[t];
        if (kind >= 0) stats_field(s, kind, NULL, S1);
        const int interp = kind == 3 || kind == 5 || kind == 6 || kind == 8;
        for (int j = 2; j <= NY - 1; ++j)
            for (int k = 0; k <= NZP - 1; ++k)
                for (int i = 0; i <= NXM; ++i) {
                    double v;
                    if (kind >= 0 && interp)
                        v = (s->DYF[j - 1] * pow(PH(S1, i, k, j), 2.0) + s->DYF[j] * pow(PH(S1, i, k, j - 1), 2.0)) /
                            (2.0 * s->DY[j]);
                    else if (kind >= 0)
                        v = pow(PH(S1, i, k, j), 2.0);
                    else if (kind == -1)
                        v = pow(((PH(u[0], i, k, j) - ume[j]) - (PH(u[0], i, k, j - 1) - ume[j - 1])) / s->DY[j], 2.0);
                    else if (kind == -2)
                        v = pow(((PH(u[1], i, k, j + 1) - vme[j]) - (PH(u[1], i, k, j - 1) - vme[j - 1])) /
                                    (s->GY[j + 1] - s->GY[j - 1]), 2.0);
                    else
                        v = pow(((PH(u[2], i, k, j) - wme[j]) - (PH(u[2], i, k, j - 1) - wme[j - 1])) / s->DY[j], 2.0);
                    PH(F1, i, k, j) += v;
                }
    }
    for (int j = 2; j <= NY - 1; ++j)
        for (int k = 0; k <= NZP - 1; ++k)
            for (int i = 0; i <= NXM; ++i) PH(F1, i, k, j) *= s->p.nu;
    for (int c = 0; c < 3; ++c) free(u[c]);
    free(S1);
    free(base);
}

/* a zero eddy viscosity carries no flux: at J = 1 the reference divides 0 by
 * DYF(0), which it never sets (0), and gets NaN */
#define FLUX(coef, du, h) ((coef) == 0.0 ? 0.0 : (coef) * (du) / (h))
void orc_epsilon_sgs(orc_state* s, double* out) {
    const int NY = s->NY, NZP = s->NZP, NXM = s->NXM;
    memset(out, 0, sizeof(double) * (NY + 2));
    if (!s->p.les) return;
    double* base = (double*)malloc(sizeof(double) * DIABLO_NSTATS * (NY + 2));
    orc_stats(s, base);                         /* APPLY_BC_VEL on the state */
    free(base);
    double* u[3];
    for (int c = 0; c < 3; ++c) {
        u[c] = (double*)malloc(sizeof(double) * s->nreal);
        memcpy(u[c], c == 0 ? s->U1 : c == 1 ? s->U2 : s->U3, sizeof(double) * s->nreal);
        orc_fft_xz_to_physical(s, u[c], u[c], 0, NY + 1);
    }
    const double *U1 = u[0], *U2 = u[1], *U3 = u[2], *NT = s->NU_T, *DY = s->DY, *DYF = s->DYF;
    for (int j = 1; j <= NY; ++j) {
        double e = 0.0;
        for (int i = 0; i <= NXM; ++i)
            for (int k = 0; k <= NZP - 1; ++k) {
                const double t =
                    PH(U1, i, k, j) * ((PH(NT, i, k, j + 1) * (PH(U1, i, k, j + 1) - PH(U1, i, k, j)) / DY[j + 1] -
                                        PH(NT, i, k, j) * (PH(U1, i, k, j) - PH(U1, i, k, j - 1)) / DY[j]) / DYF[j]) +
                    PH(U3, i, k, j) * ((PH(NT, i, k, j + 1) * (PH(U3, i, k, j + 1) - PH(U3, i, k, j)) / DY[j + 1] -
                                        PH(NT, i, k, j) * (PH(U3, i, k, j) - PH(U3, i, k, j - 1)) / DY[j]) / DYF[j]) +
                    PH(U2, i, k, j) * ((FLUX(0.5 * (PH(NT, i, k, j) + PH(NT, i, k, j + 1)),
                                             PH(U2, i, k, j + 1) - PH(U2, i, k, j), DYF[j]) -
                                        FLUX(0.5 * (PH(NT, i, k, j) + PH(NT, i, k, j - 1)),
                                             PH(U2, i, k, j) - PH(U2, i, k, j - 1), DYF[j - 1])) / DY[j]);
                e += t;
            }
        out[j] = e;
    }
    for (int c = 0; c < 3; ++c) free(u[c]);
}
#undef FLUX

void orc_set_user_rhs(orc_state* s, int kind, void (*fn)(void*), void* user) {
    if (kind < 0 || kind > 1) return;
    s->user_fn[kind] = fn;
    s->user_data[kind] = user;
}

void orc_filter_chan(orc_state* s, int n) {
    if (n < 1 || n > s->NTH) return;
    const int NY = s->NY, NKX = s->NKX, TNKZ = s->TNKZ;
    double* C = s->CTH + (size_t)(n - 1) * s->nreal;
    const double alpha = 0.0;
    const double f_a = (1.0 / 8.0) * (5.0 + 6.0 * alpha), f_b = 0.5 * (1.0 + 2.0 * alpha),
                 f_c = (-1.0 / 8.0) * (1.0 - 2.0 * alpha);
    for (int k = 0; k <= TNKZ; ++k)
        for (int i = 0; i <= NKX; ++i) {
            const double a1 = s->KX[i] * s->p.lx * 1.0 / (double)(float)s->NX;
            const double a2 = s->KZ[k] * s->p.lz * 1.0 / (double)(float)s->NZ;
            const double sigma0 = 0.5 * (1.0 + cos(sqrt(pow(a1, 2.0) + pow(a2, 2.0))));
            const double sigma = pow(sigma0, 4.0) * (35.0 - 84.0 * sigma0 + 70.0 * pow(sigma0, 2.0) -
                                                     20.0 * pow(sigma0, 3.0));
            for (int j = 0; j <= NY; ++j) CX(C, i, k, j) = CX(C, i, k, j) * sigma;
        }
    cplx* vec = (cplx*)malloc(sizeof(cplx) * (size_t)(NY + 2));
    for (int k = 1; k <= TNKZ; ++k)
        for (int i = 1; i <= NKX; ++i) {
            for (int j = 2; j <= NY - 1; ++j)
                vec[j] = f_a * CX(C, i, k, j) + (f_b / 2.0) * (CX(C, i, k, j + 1) + CX(C, i, k, j - 1)) +
                         (f_c / 2.0) * (CX(C, i, k, j + 2) + CX(C, i, k, j - 2));
            for (int j = 2; j <= NY - 1; ++j) CX(C, i, k, j) = vec[j];
        }
    free(vec);
}
