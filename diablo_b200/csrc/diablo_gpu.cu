// diablo_gpu.cu -- the C ABI (include/diablo_gpu.h): handle, device state,
// host <-> device layout conversion and the RK_CHAN_1 substage pipeline.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/diablo_gpu.h"
#include "fft.cuh"
#include "kernels.cuh"
#include "launch.h"

using namespace dgpu;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define CK(call)                                                                            \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail(DIABLO_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

struct Handle {
    diablo_params p;
    Dims d;
    int nxp;
    int jstart, jend, jstart_th[DIABLO_MAX_TH], jend_th[DIABLO_MAX_TH];
    int jlo_prod;
    double dx, dz, pi;
    std::vector<double> gy, gyf, dy, dyf;
    bool fp32;
    bool pb;          // CF pair-blocked (spec_at): the Fourier-space path without LES
    cudaStream_t st = nullptr;
    size_t s_plane, s_field;      // elements
    size_t x_plane, x_field;      // elements
    // device memory
    double *d_dy = nullptr, *d_dyf = nullptr, *d_kx = nullptr, *d_kz = nullptr;
    double2 *cu = nullptr, *cf = nullptr, *cp = nullptr, *phi = nullptr, *api_s = nullptr;
    void *nl = nullptr, *xb = nullptr, *yb = nullptr;
    double* bsc = nullptr;
    double2* gsc = nullptr;
    double* phys = nullptr;
    double* d_gyf = nullptr;
    double* pw = nullptr;         // 4 physical fields (POISSON_P_CHAN, statistics), allocated on first use
    double* d_me = nullptr;       // [4][nyp] mean profiles for the statistics
    double* d_sums = nullptr;     // [9][nyp] plane sums of the statistics
    double* d_msums = nullptr;    // [4 + 3 N_TH][nyp] plane sums of the mean.h5 / tke.h5 profiles, then [nyp] 1/(GY(j+1)-GY(j-1))
    double* bcv = nullptr;        // [3][nf][nyp] BC-row values of the (0,0) mode, per RK substage
    double* d_tabs = nullptr;     // [3][nf][part_table_doubles] CN partition factors, per RK substage
    // The CN rows depend on the grid, the parameters and TEMP1 = NU*H_BAR/2
    // only: the factors of substage r stay valid while TEMP1 is tab_temp1[r].
    bool tab_ok[3] = {false, false, false};
    double tab_temp1[3] = {0.0, 0.0, 0.0};
    double* d_phitab = nullptr;   // [column][phi_table_doubles/column] phi partition factors
    int* d_nan = nullptr;         // set by the kernels that write CU when a value is not finite
    // user right-hand-side hooks (USER_RHS_CHAN_FOURIER / _PHYSICAL), their
    // Fourier-space addend (nf fields, S) and, for the physical hook, the
    // physical fields and their addend (2 nf fields, P); allocated on first use
    diablo_user_rhs_fn urhs_fn[2] = {nullptr, nullptr};
    void* urhs_user[2] = {nullptr, nullptr};
    double2* ufa = nullptr;
    double* uphys = nullptr;
    signed char* kind = nullptr;
    double* dtmin = nullptr;
    double* d_k2 = nullptr;       // (KX^2+KZ^2)**BETA per padded column
    double* d_rows = nullptr;     // [RT_COUNT][nyp] reciprocal grid metrics
    // LES branch (allocated when p.les): NU_T at GY points, physical fields
    // (lu: U1..U3, TH; la, lb: work fields), spectral work (ls: 7 fields, lr:
    // the nf right-hand sides), the x-spectrum work lx and the filter widths
    // Delta_YF, Delta_Y ([2][nyp])
    double *nut = nullptr, *lu = nullptr, *la = nullptr, *lb = nullptr, *d_delta = nullptr;
    double* d_dyn = nullptr;      // dynamic model: [2][nyp] plane sums, [2][nyp] widths
    void* mlp = nullptr;          // learned closure (LES_MODEL_TYPE 4), owned by the caller
    float *mlp_x = nullptr, *mlp_t = nullptr, *mlp_s = nullptr;   // its features [n][11], outputs [n][6], scales [n]
    double2 *ls = nullptr, *lr = nullptr;
    void* lx = nullptr;
    bool nut_set = false;         // NU_T has been computed at least once
    FftPlan pm, pz;   // NX/2-point complex plan (real x transforms), NZ-point plan
    void *twn_d = nullptr, *twm_d = nullptr, *twz_d = nullptr;   // exp(-2 pi i k/n), n = NX, NX/2, NZ
    void *twn_f = nullptr, *twm_f = nullptr, *twz_f = nullptr;
    int bc_type[2 * MAXF];
    double bc_c1[2 * MAXF];
    long long launches = 0;
    // launch shapes (diablo_gpu_autotune): planes per products block chunk, planes per z-forward block
    int prod_chunk = 32, zf_planes = 8;
    // optional per-kernel event timing
    bool profiling = false;
    struct Rec { int kind; cudaEvent_t a, b; };
    std::vector<Rec> recs;
    // one RK3 step as a CUDA graph (diablo_gpu_step_graph) and what it was
    // captured with: H_BAR, BETA_BAR, ZETA_BAR, the launch shapes, the network
    cudaGraph_t sg_graph = nullptr;
    cudaGraphExec_t sg_exec = nullptr;
    double sg_coef[9] = {};
    int sg_prod = 0, sg_zf = 0;
    void* sg_mlp = nullptr;
    long long sg_launches = 0;    // kernel launches of one captured step
};

// Bracket a launch with events when profiling (kinds: DIABLO_KERNEL_*).
struct ProfScope {
    Handle* h;
    int kind;
    cudaEvent_t a = nullptr;
    ProfScope(Handle* hh, int k) : h(hh), kind(k) {
        if (h->profiling && cudaEventCreate(&a) == cudaSuccess) cudaEventRecord(a, h->st);
        else a = nullptr;
    }
    ~ProfScope() {
        if (!a) return;
        cudaEvent_t b;
        if (cudaEventCreate(&b) == cudaSuccess) {
            cudaEventRecord(b, h->st);
            h->recs.push_back({kind, a, b});
        } else {
            cudaEventDestroy(a);
        }
    }
};

bool is_235(int n) {
    if (n < 2) return false;
    for (int r : {2, 3, 5})
        while (n % r == 0) n /= r;
    return n == 1;
}

template <typename T>
void* make_twiddles(int n, cudaStream_t st, cudaError_t* err) {
    std::vector<T> h(2 * (size_t)n);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < n; ++k) {
        // angle reduced to the first octant for an accurate table
        const long double a = -2.0L * pi * (long double)k / (long double)n;
        h[2 * k] = (T)cosl(a);
        h[2 * k + 1] = (T)sinl(a);
    }
    void* d = nullptr;
    *err = cudaMalloc(&d, sizeof(T) * h.size());
    // stream-ordered with the handle's kernels; a pageable source is consumed before the call returns
    if (*err == cudaSuccess) *err = cudaMemcpyAsync(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, st);
    return d;
}

void free_handle(Handle* h) {
    if (!h) return;
    if (h->sg_exec) cudaGraphExecDestroy(h->sg_exec);
    if (h->sg_graph) cudaGraphDestroy(h->sg_graph);
    for (auto& r : h->recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    void* ptrs[] = {h->d_dy, h->d_dyf, h->d_kx, h->d_kz, h->cu, h->cf, h->cp, h->phi, h->api_s,
                    h->nl, h->xb, h->yb, h->bsc, h->gsc, h->phys, h->d_gyf, h->pw, h->d_me, h->d_sums, h->d_msums, h->d_nan, h->ufa, h->uphys, h->d_tabs, h->d_phitab,
                    h->bcv, h->kind, h->dtmin, h->d_k2, h->d_rows, h->twn_d, h->twm_d, h->twz_d, h->twn_f, h->twm_f,
                    h->twz_f, h->nut, h->lu, h->la, h->lb, h->d_delta, h->ls, h->lr, h->lx, h->d_dyn,
                    h->mlp_x, h->mlp_t, h->mlp_s};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
}

// After a stream synchronisation: DIABLO_ENAN, once, if a kernel that writes
// CU (the column kernel, the projection) met a value that is not finite
// since the last check; the flag is cleared.
static int take_nan(Handle* h) {
    int v = 0;
    CK(cudaMemcpyAsync(&v, h->d_nan, sizeof(int), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    if (!v) return DIABLO_OK;
    CK(cudaMemsetAsync(h->d_nan, 0, sizeof(int), h->st));
    return fail(DIABLO_ENAN, "a non-finite value appeared in the state (CU) during a step");
}

// Host Fortran complex array (0:NXP,0:NZ+1,0:NY+1) <-> device spectral field.
cudaError_t copy_fourier(Handle* h, double2* dev, const double* host_in, double* host_out, int j0,
                         int nplanes) {
    const Dims& d = h->d;
    cudaMemcpy3DParms c = {};
    const size_t hpitch = sizeof(double2) * (size_t)(h->nxp + 1);
    const size_t dpitch = sizeof(double2) * (size_t)d.ldx;
    cudaPitchedPtr hp = make_cudaPitchedPtr((void*)(host_in ? host_in : host_out), hpitch,
                                            (size_t)(h->nxp + 1), (size_t)(d.nz + 2));
    cudaPitchedPtr dp = make_cudaPitchedPtr((void*)dev, dpitch, (size_t)d.ldx, (size_t)d.nkzp);
    c.extent = make_cudaExtent(sizeof(double2) * (size_t)d.nkxp, (size_t)d.nkzt, (size_t)nplanes);
    if (host_in) {
        c.srcPtr = hp; c.dstPtr = dp;
        c.srcPos = make_cudaPos(0, 0, j0); c.dstPos = make_cudaPos(0, 0, j0);
        c.kind = cudaMemcpyHostToDevice;
    } else {
        c.srcPtr = dp; c.dstPtr = hp;
        c.srcPos = make_cudaPos(0, 0, j0); c.dstPos = make_cudaPos(0, 0, j0);
        c.kind = cudaMemcpyDeviceToHost;
    }
    return cudaMemcpy3DAsync(&c, h->st);
}

// Host Fortran physical array (0:NX+1,0:NZ+1,0:NY+1) <-> device P[J][z][x].
cudaError_t copy_physical(Handle* h, double* dev, const double* host_in, double* host_out, int j0,
                          int nplanes) {
    const Dims& d = h->d;
    cudaMemcpy3DParms c = {};
    cudaPitchedPtr hp = make_cudaPitchedPtr((void*)(host_in ? host_in : host_out),
                                            sizeof(double) * (size_t)(d.nx + 2), (size_t)(d.nx + 2),
                                            (size_t)(d.nz + 2));
    cudaPitchedPtr dp = make_cudaPitchedPtr((void*)dev, sizeof(double) * (size_t)d.nx, (size_t)d.nx,
                                            (size_t)d.nz);
    c.extent = make_cudaExtent(sizeof(double) * (size_t)d.nx, (size_t)d.nz, (size_t)nplanes);
    c.srcPos = make_cudaPos(0, 0, j0);
    c.dstPos = make_cudaPos(0, 0, j0);
    if (host_in) { c.srcPtr = hp; c.dstPtr = dp; c.kind = cudaMemcpyHostToDevice; }
    else { c.srcPtr = dp; c.dstPtr = hp; c.kind = cudaMemcpyDeviceToHost; }
    return cudaMemcpy3DAsync(&c, h->st);
}

// dst += src over n complex elements (the user right-hand side added to NL or CF).
template <typename T>
__global__ void k_add_user(cpx<T>* __restrict__ dst, const double2* __restrict__ src, size_t n) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const double2 v = src[e];
        dst[e] = dst[e] + mk(T(v.x), T(v.y));
    }
}

// One spectral field between the S layout and the pair-blocked one.
__global__ void k_to_pair_blocked(Dims d, const double2* __restrict__ src, double2* __restrict__ dst) {
    const size_t ps = d.splane(), n = ps * d.nyp;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
        dst[spec_at(d, true, (int)(e / ps), e % ps)] = src[e];
}
__global__ void k_from_pair_blocked(Dims d, const double2* __restrict__ src, double2* __restrict__ dst) {
    const size_t ps = d.splane(), n = ps * d.nyp;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
        dst[e] = src[spec_at(d, true, (int)(e / ps), e % ps)];
}

// CF of field f <-> the host array; CF is pair-blocked on the Fourier-space
// path (h->pb) and passes through the API scratch field.  host == nullptr on
// upload zeroes the field.
cudaError_t cf_upload(Handle* h, int f, const double* host) {
    double2* dev = h->cf + (size_t)f * h->s_field;
    if (!host) return cudaMemsetAsync(dev, 0, sizeof(double2) * h->s_field, h->st);
    if (!h->pb) return copy_fourier(h, dev, host, nullptr, 0, h->d.nyp);
    cudaError_t e = cudaMemsetAsync(h->api_s, 0, sizeof(double2) * h->s_field, h->st);
    if (e == cudaSuccess) e = copy_fourier(h, h->api_s, host, nullptr, 0, h->d.nyp);
    if (e != cudaSuccess) return e;
    k_to_pair_blocked<<<1184, 256, 0, h->st>>>(h->d, h->api_s, dev);
    return cudaGetLastError();
}

cudaError_t cf_download(Handle* h, int f, double* host) {
    const double2* dev = h->cf + (size_t)f * h->s_field;
    if (!h->pb) return copy_fourier(h, const_cast<double2*>(dev), nullptr, host, 0, h->d.nyp);
    k_from_pair_blocked<<<1184, 256, 0, h->st>>>(h->d, dev, h->api_s);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = copy_fourier(h, h->api_s, nullptr, host, 0, h->d.nyp);
    return e;
}


// APPLY_BC_VEL_LOWER / _UPPER (channel.f:2285-2492) on the device state.
__global__ void k_apply_bc_vel(Dims d, double2* cu, const double* dy, const double* dyf, diablo_params p) {
    const int kx = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = blockIdx.y;
    if (kx >= d.nkxp || m >= d.nkzt) return;
    const size_t ps = d.splane(), fs = ps * d.nyp, col = (size_t)m * d.ldx + kx;
    const bool z0 = (kx == 0 && m == 0);
    const int ny = d.ny;
    double2* u1 = cu + col;
    double2* u2 = cu + fs + col;
    double2* u3 = cu + 2 * fs + col;
    const double2 zero = make_double2(0, 0);
    auto at = [&](double2* f, int j) -> double2& { return f[(size_t)j * ps]; };
    // lower wall
    if (p.u_bc_ymin == 0) {
        at(u1, 0) = zero; at(u1, 1) = zero;
        if (z0) { at(u1, 1) = make_double2(p.u_bc_ymin_c1, 0); at(u1, 0) = make_double2(p.u_bc_ymin_c1, 0); }
    } else {
        at(u1, 1) = at(u1, 2); at(u1, 0) = at(u1, 1);
        if (z0) {
            at(u1, 1).x = at(u1, 2).x - dy[2] * p.u_bc_ymin_c1;
            at(u1, 0).x = at(u1, 1).x - dy[1] * p.u_bc_ymin_c1;
        }
    }
    if (p.w_bc_ymin == 0) {
        at(u3, 0) = zero; at(u3, 1) = zero;
        if (z0) { at(u3, 1) = make_double2(p.w_bc_ymin_c1, 0); at(u3, 0) = make_double2(p.w_bc_ymin_c1, 0); }
    } else {
        at(u3, 1) = at(u3, 2); at(u3, 0) = at(u3, 1);
        if (z0) {
            at(u3, 1).x = at(u3, 2).x - dy[2] * p.w_bc_ymin_c1;
            at(u3, 0).x = at(u3, 1).x - dy[1] * p.w_bc_ymin_c1;
        }
    }
    if (p.v_bc_ymin == 0) {
        const double2 v2 = at(u2, 2);
        at(u2, 1) = make_double2(2.0 * p.v_bc_ymin_c1 - v2.x, -v2.y);
        at(u2, 0) = at(u2, 1);
    } else if (p.v_bc_ymin == 1) {
        at(u2, 1) = at(u2, 2); at(u2, 0) = at(u2, 1);
        if (z0) {
            at(u2, 1).x = at(u2, 2).x - dyf[1] * p.v_bc_ymin_c1;
            at(u2, 0).x = at(u2, 1).x - dyf[1] * p.v_bc_ymin_c1;
        }
    }
    // upper wall
    if (p.u_bc_ymax == 0) {
        at(u1, ny) = zero; at(u1, ny + 1) = zero;
        if (z0) { at(u1, ny) = make_double2(p.u_bc_ymax_c1, 0); at(u1, ny + 1) = make_double2(p.u_bc_ymax_c1, 0); }
    } else {
        at(u1, ny) = at(u1, ny - 1); at(u1, ny + 1) = at(u1, ny);
        if (z0) {
            at(u1, ny).x = at(u1, ny - 1).x + dy[ny] * p.u_bc_ymax_c1;
            at(u1, ny + 1).x = at(u1, ny).x + dy[ny] * p.u_bc_ymax_c1;
        }
    }
    if (p.w_bc_ymax == 0) {
        at(u3, ny) = zero; at(u3, ny + 1) = zero;
        if (z0) { at(u3, ny) = make_double2(p.w_bc_ymax_c1, 0); at(u3, ny + 1) = zero; }
    } else {
        at(u3, ny) = at(u3, ny - 1); at(u3, ny + 1) = at(u3, ny);
        if (z0) {
            at(u3, ny).x = at(u3, ny - 1).x + dy[ny] * p.w_bc_ymax_c1;
            at(u3, ny + 1).x = at(u3, ny).x + dy[ny] * p.w_bc_ymax_c1;
        }
    }
    if (p.v_bc_ymax == 0) {
        // only the (0,0) entry is written by the reference (channel.f:2463-2467)
        if (z0) {
            const double2 v = at(u2, ny);
            at(u2, ny + 1) = make_double2(2.0 * p.v_bc_ymax_c1 - v.x, -v.y);
        }
    } else if (p.v_bc_ymax == 1) {
        at(u2, ny) = at(u2, ny - 1); at(u2, ny + 1) = at(u2, ny);
        if (z0) at(u2, ny + 1).x = at(u2, ny).x + dy[ny] * p.v_bc_ymax_c1;
    }
}

int validate(const diablo_params* p) {
    if (!p) return fail(DIABLO_EINVAL, "null params");
    if (p->nx < 8 || p->nz < 8 || (p->nx % 2)) return fail(DIABLO_EINVAL, "NX and NZ must be >= 8, NX even");
    if (!is_235(p->nx) || !is_235(p->nz)) return fail(DIABLO_ERADIX, "NX and NZ must be products of 2, 3 and 5");
    if (p->nx > 1536 || p->nz > 512) return fail(DIABLO_EINVAL, "NX <= 1536 and NZ <= 512 are supported");
    if (p->ny < 4) return fail(DIABLO_EINVAL, "NY must be >= 4");
    if (p->n_th < 0 || p->n_th > DIABLO_MAX_TH) return fail(DIABLO_EINVAL, "N_TH must be in 0..4");
    if (p->les) {
        // 1: constant Smagorinsky (les.f); 2: this library's dynamic model; the
        // reference stops for 2 and 3 (les.f:269-272)
        if (p->les_model_type != 1 && p->les_model_type != 2 && p->les_model_type != 4)
            return fail(DIABLO_ENOTSUP, "LES_MODEL_TYPE must be 1 (constant), 2 (dynamic) or 4 (learned closure)");
        if (p->precision != DIABLO_PREC_FP64) return fail(DIABLO_ENOTSUP, "the LES branch runs in FP64 only");
    }
    auto bc01 = [](int t) { return t == 0 || t == 1; };
    if (!bc01(p->u_bc_ymin) || !bc01(p->u_bc_ymax) || !bc01(p->w_bc_ymin) || !bc01(p->w_bc_ymax) ||
        !bc01(p->v_bc_ymin) || !bc01(p->v_bc_ymax))
        return fail(DIABLO_EINVAL, "velocity BC types must be 0 (Dirichlet) or 1 (Neumann)");
    for (int n = 0; n < p->n_th; ++n) {
        if (!bc01(p->th_bc_ymin[n]) || !bc01(p->th_bc_ymax[n]))
            return fail(DIABLO_EINVAL, "scalar BC types must be 0 or 1");
        if (p->pr[n] == 0.0) return fail(DIABLO_EINVAL, "PR must be non-zero");
    }
    if (p->precision != DIABLO_PREC_FP64 && p->precision != DIABLO_PREC_FP32SPLIT)
        return fail(DIABLO_EINVAL, "precision must be DIABLO_PREC_FP64 or DIABLO_PREC_FP32SPLIT");
    if (p->variable_dt && p->update_dt <= 0) return fail(DIABLO_EINVAL, "UPDATE_DT must be > 0");
    return DIABLO_OK;
}

int smem_limits(const Handle* h) {
    // shared-memory budget of the products kernel (FP64 is the larger case)
    const Dims& d = h->d;
    const int group = products_group(d.nx);
    const int m = d.nx / 2;
    const int rows = group < d.nf + d.np ? group : d.nf + d.np;
    const size_t smem = sizeof(double) * (size_t)4 * d.nf * d.nx + 16 * (size_t)rows * (m + m / 16 + 1) + 16 * 3 * (size_t)m +
                        16 * 2 * (size_t)d.nf * d.ldx + 16;
    if (group < 1 || smem > 227 * 1024) return fail(DIABLO_EINVAL, "NX too large for the number of fields");
    // the column kernel holds whole columns: NY+2 <= 528 rows
    if (part_rows(d.nyp) == 0) return fail(DIABLO_EINVAL, "NY too large (at most 526)");
    if (colpart_smem<cpx<double>>(d) > 227 * 1024) return fail(DIABLO_EINVAL, "NY too large for the number of fields");
    return DIABLO_OK;
}

template <typename T>
int run_transforms(Handle* h) {
    const Dims& d = h->d;
    const bool f = std::is_same<T, float>::value;
    const void* twn = f ? h->twn_f : h->twn_d;
    const void* twm = f ? h->twm_f : h->twm_d;
    const void* twz = f ? h->twz_f : h->twz_d;
    // FP32 transforms carry each field's fluctuation about its plane mean; the
    // means (the (0,0) mode, O(1) in a shear layer or channel) stay FP64
    { ProfScope ps(h, DIABLO_KERNEL_ZINV);
      CK(launch_zinv<T>(d, h->cu, h->s_field, h->xb, h->x_field, d.nf, 0, d.nyp, h->pz, twz, h->st, f ? 1 : 0)); }
    { ProfScope ps(h, DIABLO_KERNEL_PRODUCTS);
      if (f && products_hw_supported(d))
          CK(launch_products_hw(d, h->xb, h->yb, h->jlo_prod, d.ny, h->prod_chunk, h->d_dy, h->d_dyf, h->d_kx, twm, twn,
                                h->st, h->cu, h->s_field));
      else
          CK(launch_products<T>(d, h->xb, h->yb, h->jlo_prod, d.ny, h->prod_chunk, h->d_dy, h->d_dyf, h->d_kx, h->pm, twm,
                                twn, h->st, f ? h->cu : nullptr, h->s_field)); }
    { ProfScope ps(h, DIABLO_KERNEL_ZFWD_NL);
      CK(launch_zfwd_nl<T>(d, h->yb, h->nl, h->jlo_prod, d.ny, h->zf_planes, h->d_kx, h->d_kz, h->pz, twz, h->st)); }
    h->launches += 3;
    return DIABLO_OK;
}


}  // namespace

int dgpu::set_error(int code, const std::string& msg) { return fail(code, msg); }

extern "C" {

const char* diablo_gpu_last_error(void) { return g_err.c_str(); }

int diablo_gpu_create(const diablo_params* p, const double* gy, const double* gyf, const double* dy,
                      const double* dyf, void** handle) {
    if (!handle || !gy || !gyf || !dy || !dyf) return fail(DIABLO_EINVAL, "null pointer argument");
    *handle = nullptr;
    int rc = validate(p);
    if (rc) return rc;
    Handle* h = new Handle();
    h->p = *p;
    Dims& d = h->d;
    d.nx = p->nx; d.ny = p->ny; d.nz = p->nz; d.nth = p->n_th;
    d.nf = 3 + p->n_th;
    d.np = 8 + 3 * p->n_th;
    d.nkx = p->nx / 3; d.nkz = p->nz / 3; d.tnkz = 2 * d.nkz;
    d.nkxp = d.nkx + 1; d.nkzt = d.tnkz + 1;
    d.nkzp = (d.nkzt + 1) / 2 * 2;
    d.ldx = (d.nkxp + 15) / 16 * 16;
    d.nyp = p->ny + 2;
    h->nxp = p->nx / 2;
    h->fp32 = p->precision == DIABLO_PREC_FP32SPLIT;
    h->pb = !p->les;      // the LES branch's kernels take CF in the S layout
    h->pi = 4.0 * std::atan(1.0);
    h->dx = p->lx / p->nx;
    h->dz = p->lz / p->nz;
    h->gy.assign(gy, gy + d.nyp);
    h->gyf.assign(gyf, gyf + d.nyp);
    h->dy.assign(dy, dy + d.nyp);
    h->dyf.assign(dyf, dyf + d.nyp);
    // INIT_CHAN_MPI, RANKY = 0 branch (mpi.f:1024-1044)
    h->jstart = 2;
    h->jend = p->ny;
    h->jlo_prod = 2;
    for (int n = 0; n < p->n_th; ++n) {
        h->jend_th[n] = p->ny;
        h->jstart_th[n] = p->th_bc_ymin[n] == 1 ? 1 : 2;
        if (h->jstart_th[n] < h->jlo_prod) h->jlo_prod = h->jstart_th[n];
    }
    if ((rc = smem_limits(h))) { delete h; return rc; }
    if (!make_plan(d.nx / 2, &h->pm) || !make_plan(d.nz, &h->pz)) { delete h; return fail(DIABLO_ERADIX, "bad radix"); }
    // BC table: [field][lower, upper]
    for (int f = 0; f < 2 * MAXF; ++f) { h->bc_type[f] = 0; h->bc_c1[f] = 0.0; }
    h->bc_type[0] = p->u_bc_ymin; h->bc_type[1] = p->u_bc_ymax;
    h->bc_c1[0] = p->u_bc_ymin_c1; h->bc_c1[1] = p->u_bc_ymax_c1;
    h->bc_type[2] = p->v_bc_ymin; h->bc_type[3] = p->v_bc_ymax;
    h->bc_c1[2] = p->v_bc_ymin_c1; h->bc_c1[3] = p->v_bc_ymax_c1;
    h->bc_type[4] = p->w_bc_ymin; h->bc_type[5] = p->w_bc_ymax;
    h->bc_c1[4] = p->w_bc_ymin_c1; h->bc_c1[5] = p->w_bc_ymax_c1;
    for (int n = 0; n < p->n_th; ++n) {
        h->bc_type[2 * (3 + n)] = p->th_bc_ymin[n]; h->bc_type[2 * (3 + n) + 1] = p->th_bc_ymax[n];
        h->bc_c1[2 * (3 + n)] = p->th_bc_ymin_c1[n]; h->bc_c1[2 * (3 + n) + 1] = p->th_bc_ymax_c1[n];
    }

    h->s_plane = d.splane();
    h->s_field = h->s_plane * d.nyp;
    h->x_plane = (size_t)d.nz * d.ldx;
    h->x_field = h->x_plane * d.nyp;
    // Every set-up memset and copy goes on the handle's non-blocking stream: work on the legacy
    // default stream would not be ordered before the kernels that read these buffers.
    cudaError_t e = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking);
    auto dmalloc = [&](void** ptr, size_t bytes) -> cudaError_t {
        cudaError_t e = cudaMalloc(ptr, bytes);
        if (e == cudaSuccess) e = cudaMemsetAsync(*ptr, 0, bytes, h->st);
        return e;
    };
    const size_t sb = sizeof(double2) * h->s_field;
    const size_t nyp = (size_t)d.nyp;
    if (e == cudaSuccess) e = dmalloc((void**)&h->d_dy, sizeof(double) * nyp);
    if (e == cudaSuccess) e = dmalloc((void**)&h->d_dyf, sizeof(double) * nyp);
    if (e == cudaSuccess) e = dmalloc((void**)&h->d_gyf, sizeof(double) * nyp);
    if (e == cudaSuccess) e = dmalloc((void**)&h->d_kx, sizeof(double) * d.ldx);
    if (e == cudaSuccess) e = dmalloc((void**)&h->d_kz, sizeof(double) * d.nkzp);
    if (e == cudaSuccess) e = dmalloc((void**)&h->cu, sb * d.nf);
    if (e == cudaSuccess) e = dmalloc((void**)&h->cf, sb * d.nf);
    if (e == cudaSuccess) e = dmalloc((void**)&h->cp, sb);
    if (e == cudaSuccess) e = dmalloc((void**)&h->phi, sb);
    if (e == cudaSuccess) e = dmalloc((void**)&h->api_s, sb);
    if (e == cudaSuccess) e = dmalloc(&h->nl, sb * d.nf);
    if (e == cudaSuccess) e = dmalloc((void**)&h->bsc, sizeof(double) * h->s_field);
    if (e == cudaSuccess) e = dmalloc((void**)&h->gsc, sb);
    if (e == cudaSuccess) e = dmalloc(&h->xb, sizeof(double2) * h->x_field * d.nf);
    if (e == cudaSuccess) e = dmalloc(&h->yb, sizeof(double2) * h->x_field * d.np);
    if (e == cudaSuccess) e = dmalloc((void**)&h->d_tabs, sizeof(double) * part_table_doubles(d.nyp) * d.nf * 3);
    if (e == cudaSuccess) e = dmalloc((void**)&h->d_phitab, sizeof(double) * phi_table_doubles(d));
    if (e == cudaSuccess) e = dmalloc((void**)&h->d_nan, sizeof(int));
    if (e == cudaSuccess) e = dmalloc((void**)&h->bcv, sizeof(double) * nyp * d.nf * 3);
    if (e == cudaSuccess) e = dmalloc((void**)&h->kind, nyp * d.nf * 3);
    if (e == cudaSuccess) e = dmalloc((void**)&h->dtmin, sizeof(double));
    if (e == cudaSuccess) e = dmalloc((void**)&h->d_k2, sizeof(double) * d.splane());
    if (e == cudaSuccess) e = dmalloc((void**)&h->d_rows, sizeof(double) * RT_COUNT * nyp);
    if (p->les) {
        const size_t pf = sizeof(double) * nyp * d.nz * d.nx;
        const int nw = d.nf > 7 ? d.nf : 7;
        if (e == cudaSuccess) e = dmalloc((void**)&h->nut, pf);
        if (e == cudaSuccess) e = dmalloc((void**)&h->lu, pf * d.nf);
        if (e == cudaSuccess) e = dmalloc((void**)&h->la, pf * nw);
        if (e == cudaSuccess) e = dmalloc((void**)&h->lb, pf * 7);
        if (e == cudaSuccess) e = dmalloc((void**)&h->ls, sb * 7);
        if (e == cudaSuccess) e = dmalloc((void**)&h->lr, sb * d.nf);
        if (e == cudaSuccess) e = dmalloc(&h->lx, sizeof(double2) * h->x_field * nw);
        if (e == cudaSuccess) e = dmalloc((void**)&h->d_delta, sizeof(double) * 2 * nyp);
        if (e == cudaSuccess) e = dmalloc((void**)&h->d_dyn, sizeof(double) * 4 * nyp);
    }
    if (e != cudaSuccess) {
        free_handle(h);
        return fail(e == cudaErrorMemoryAllocation ? DIABLO_ENOMEM : DIABLO_ECUDA,
                    std::string("device set-up: ") + cudaGetErrorString(e));
    }
    // wavenumbers (fft.f:77-100)
    std::vector<double> kx(d.ldx, 0.0), kz(d.nkzp, 0.0);
    for (int i = 0; i <= d.nkx; ++i) kx[i] = (double)i * (2.0 * h->pi) / p->lx;
    for (int k = 0; k <= d.nkz; ++k) kz[k] = (double)k * (2.0 * h->pi) / p->lz;
    for (int k = 1; k <= d.nkz; ++k) kz[d.tnkz + 1 - k] = -(double)k * (2.0 * h->pi) / p->lz;
    // (KX2+KZ2)**BETA of the horizontal viscous term (channel.f:178)
    std::vector<double> k2(d.splane(), 0.0);
    for (int m = 0; m < d.nkzp; ++m)
        for (int i = 0; i < d.ldx; ++i) k2[(size_t)m * d.ldx + i] = std::pow(kx[i] * kx[i] + kz[m] * kz[m], p->beta);
    e = cudaMemcpyAsync(h->d_k2, k2.data(), sizeof(double) * k2.size(), cudaMemcpyHostToDevice, h->st);
    {
        std::vector<double> rows((size_t)RT_COUNT * nyp, 0.0);
        auto R = [&](int t, int j) -> double& { return rows[(size_t)t * nyp + j]; };
        for (int j = 0; j < (int)nyp; ++j) {
            const double DYj = dy[j], DYFj = dyf[j];
            const double DYj1 = j + 1 < (int)nyp ? dy[j + 1] : 0.0, DYFjm = j > 0 ? dyf[j - 1] : 0.0;
            auto inv = [](double v) { return v != 0.0 ? 1.0 / v : 0.0; };
            R(RT_RDY, j) = inv(DYj);
            R(RT_RDYF, j) = inv(DYFj);
            R(RT_E1P, j) = inv(DYj1 * DYFj);
            R(RT_E1M, j) = inv(DYj * DYFj);
            R(RT_E2P, j) = inv(DYFj * DYj);
            R(RT_E2M, j) = inv(DYFjm * DYj);
            R(RT_BY0, j) = DYj != 0.0 ? DYFjm / (2.0 * DYj) : 0.0;
            R(RT_BY1, j) = DYj != 0.0 ? DYFj / (2.0 * DYj) : 0.0;
        }
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(h->d_rows, rows.data(), sizeof(double) * rows.size(), cudaMemcpyHostToDevice, h->st);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->d_kx, kx.data(), sizeof(double) * d.ldx, cudaMemcpyHostToDevice, h->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->d_kz, kz.data(), sizeof(double) * d.nkzp, cudaMemcpyHostToDevice, h->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->d_dy, dy, sizeof(double) * nyp, cudaMemcpyHostToDevice, h->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->d_dyf, dyf, sizeof(double) * nyp, cudaMemcpyHostToDevice, h->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->d_gyf, gyf, sizeof(double) * nyp, cudaMemcpyHostToDevice, h->st);
    if (e == cudaSuccess && p->les) {
        // filter widths with -2 C_s^2 absorbed, C_s = 0.13, beta_sgs = 1
        // (les.f:196-217), Delta_YF at GYF and Delta_Y at GY points, J = 1..NY+1
        std::vector<double> w(2 * nyp, 0.0);
        const double C_SMAG = 0.13, beta_sgs = 1.0;
        for (size_t j = 1; j < nyp; ++j) {
            w[j] = -2.0 * (C_SMAG * C_SMAG) * std::pow(h->dx * beta_sgs * dyf[j] * 2.0 * h->dz * beta_sgs, 2.0 / 3.0);
            w[nyp + j] = -2.0 * (C_SMAG * C_SMAG) * std::pow(h->dx * beta_sgs * dy[j] * 2.0 * h->dz * beta_sgs, 2.0 / 3.0);
        }
        e = cudaMemcpyAsync(h->d_delta, w.data(), sizeof(double) * w.size(), cudaMemcpyHostToDevice, h->st);
    }
    if (e == cudaSuccess) h->twn_d = make_twiddles<double>(d.nx, h->st, &e);
    if (e == cudaSuccess) h->twm_d = make_twiddles<double>(d.nx / 2, h->st, &e);
    if (e == cudaSuccess) h->twz_d = make_twiddles<double>(d.nz, h->st, &e);
    if (e == cudaSuccess) h->twn_f = make_twiddles<float>(d.nx, h->st, &e);
    if (e == cudaSuccess) h->twm_f = make_twiddles<float>(d.nx / 2, h->st, &e);
    if (e == cudaSuccess) h->twz_f = make_twiddles<float>(d.nz, h->st, &e);
    if (e == cudaSuccess) e = launch_phi_part(d, h->d_rows, h->d_kx, h->d_kz, h->d_phitab, h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
    if (e != cudaSuccess) {
        free_handle(h);
        return fail(DIABLO_ECUDA, std::string("device set-up: ") + cudaGetErrorString(e));
    }
    *handle = h;
    return DIABLO_OK;
}

int diablo_gpu_destroy(void* handle) {
    Handle* h = (Handle*)handle;
    if (!h) return fail(DIABLO_EINVAL, "null handle");
    cudaStreamSynchronize(h->st);
    free_handle(h);
    return DIABLO_OK;
}

int diablo_gpu_upload_state(void* handle, const double* cu1, const double* cu2, const double* cu3,
                            const double* cp, const double* cth, const double* cf1, const double* cf2,
                            const double* cf3, const double* cfth) {
    Handle* h = (Handle*)handle;
    if (!h || !cu1 || !cu2 || !cu3 || !cp || (h->d.nth > 0 && !cth))
        return fail(DIABLO_EINVAL, "null pointer argument");
    const Dims& d = h->d;
    const size_t fstride = (size_t)(h->nxp + 1) * (d.nz + 2) * d.nyp * 2;   // doubles per host field
    const double* cus[3] = {cu1, cu2, cu3};
    for (int f = 0; f < 3; ++f) CK(copy_fourier(h, h->cu + f * h->s_field, cus[f], nullptr, 0, d.nyp));
    for (int n = 0; n < d.nth; ++n)
        CK(copy_fourier(h, h->cu + (3 + n) * h->s_field, cth + n * fstride, nullptr, 0, d.nyp));
    CK(copy_fourier(h, h->cp, cp, nullptr, 0, d.nyp));
    const double* cfs[3] = {cf1, cf2, cf3};
    for (int f = 0; f < 3; ++f) CK(cf_upload(h, f, cfs[f]));
    for (int n = 0; n < d.nth; ++n) CK(cf_upload(h, 3 + n, cfth ? cfth + n * fstride : nullptr));
    CK(cudaStreamSynchronize(h->st));
    return DIABLO_OK;
}

int diablo_gpu_download_state(void* handle, double* cu1, double* cu2, double* cu3, double* cp, double* cth,
                              double* cf1, double* cf2, double* cf3, double* cfth) {
    Handle* h = (Handle*)handle;
    if (!h) return fail(DIABLO_EINVAL, "null handle");
    const Dims& d = h->d;
    const size_t fstride = (size_t)(h->nxp + 1) * (d.nz + 2) * d.nyp * 2;
    double* cus[3] = {cu1, cu2, cu3};
    double* cfs[3] = {cf1, cf2, cf3};
    for (int f = 0; f < 3; ++f) {
        if (cus[f]) CK(copy_fourier(h, h->cu + f * h->s_field, nullptr, cus[f], 0, d.nyp));
        if (cfs[f]) CK(cf_download(h, f, cfs[f]));
    }
    for (int n = 0; n < d.nth; ++n) {
        if (cth) CK(copy_fourier(h, h->cu + (3 + n) * h->s_field, nullptr, cth + n * fstride, 0, d.nyp));
        if (cfth) CK(cf_download(h, 3 + n, cfth + n * fstride));
    }
    if (cp) CK(copy_fourier(h, h->cp, nullptr, cp, 0, d.nyp));
    CK(cudaStreamSynchronize(h->st));
    return take_nan(h);
}

int diablo_gpu_download_phi(void* handle, double* phi) {
    Handle* h = (Handle*)handle;
    if (!h || !phi) return fail(DIABLO_EINVAL, "null pointer argument");
    CK(copy_fourier(h, h->phi, nullptr, phi, 0, h->d.nyp));
    CK(cudaStreamSynchronize(h->st));
    return DIABLO_OK;
}

static int rem_div(Handle* h, int update_cp, double inv_h) {
    RemDivArgs a;
    a.d = h->d;
    a.cu = h->cu;
    a.cp = h->cp;
    a.phi = h->phi;
    a.rows = h->d_rows;
    a.phitab = h->d_phitab;
    a.kx = h->d_kx;
    a.kz = h->d_kz;
    a.dy = h->d_dy;
    a.dyf = h->d_dyf;
    a.inv_h = inv_h;
    a.update_cp = update_cp;
    a.nan_flag = h->d_nan;
    { ProfScope ps(h, DIABLO_KERNEL_REMDIV); CK(launch_remdiv(a, h->st)); }
    h->launches += 1;
    return DIABLO_OK;
}

// COURANT (courant.f:1-66): the a-priori limits on the host, the velocity
// minimum on the device from the state's current CU1..CU3, or from physical
// fields U1..U3 when phys is given (the LES branch's solved velocity).
static int courant(Handle* h, double* delta_t, double* h_bar, const double* phys = nullptr) {
    const diablo_params& p = h->p;
    const Dims& d = h->d;
    double dt = 999.0;
    dt = std::fmin(dt, 0.5 * std::pow(std::fmin(h->dx, h->dy[1]), 2.0) / p.nu);
    for (int n = 0; n < d.nth; ++n) dt = std::fmin(dt, dt * p.nu / (p.nu / p.pr[n]));
    if (p.i_ro != 0.0) dt = std::fmin(dt, 2.0 * h->pi / std::fabs(p.i_ro) / 20.0);
    for (int n = 0; n < d.nth; ++n)
        if (p.ri[n] != 0.0) {
            const double Nmax = std::sqrt(std::fabs(p.ri[n] * p.th_bc_ymin_c1[n]));
            dt = std::fmin(dt, (double)0.1f * 2.0 * h->pi / Nmax);   // single-precision 0.1 (courant.f:32)
        }
    const double inf = HUGE_VAL;
    CK(cudaMemcpyAsync(h->dtmin, &inf, sizeof(double), cudaMemcpyHostToDevice, h->st));
    if (phys) {
        ProfScope ps(h, DIABLO_KERNEL_CFL);
        CK(launch_les_cfl(d, phys, h->d_dy, p.cfl, h->dx, h->dz, h->dtmin, h->st));
        h->launches += 1;
    } else {
        ProfScope ps(h, DIABLO_KERNEL_CFL);
        CK(launch_zinv<double>(d, h->cu, h->s_field, h->xb, h->x_field, 3, 0, d.nyp, h->pz, h->twz_d, h->st));
        CK(launch_cfl(d, h->xb, h->x_field, h->pm, h->twm_d, h->twn_d, h->d_dy, p.cfl, h->dx, h->dz, h->dtmin, h->st));
        h->launches += 2;
    }
    double vmin = inf;
    CK(cudaMemcpyAsync(&vmin, h->dtmin, sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    if (int rc = take_nan(h)) return rc;   // DELTA_T and H_BAR keep their values
    dt = std::fmin(dt, vmin);
    double DELTA_T;
    if (dt <= 0) DELTA_T = 0.0001;
    else if (dt >= 999.) DELTA_T = 999.0;
    else DELTA_T = dt;
    *delta_t = DELTA_T;
    h_bar[0] = DELTA_T * (8.0 / 15.0);
    h_bar[1] = DELTA_T * (2.0 / 15.0);
    h_bar[2] = DELTA_T * (5.0 / 15.0);
    return DIABLO_OK;
}

// The constants and row ranges of RK_CHAN_1 (channel.f:77-81, INIT_CHAN_MPI
// for NPROCY = 1) as the LES kernels take them.
static CnArgs substage_args(Handle* h, int rk_step, double time, const double* h_bar, const double* beta_bar,
                            const double* zeta_bar) {
    const diablo_params& p = h->p;
    const Dims& d = h->d;
    const int r = rk_step - 1;
    const double TEMP4 = h_bar[r];
    CnArgs a;
    a.d = d;
    a.cu = h->cu;
    a.cf = h->cf;
    a.cp = h->cp;
    a.kx = h->d_kx;
    a.kz = h->d_kz;
    a.dy = h->d_dy;
    a.dyf = h->d_dyf;
    a.bcv = h->bcv;
    a.kind = h->kind;
    for (int f = 0; f < MAXF; ++f) { a.cf_lo[f] = 2; a.cf_hi[f] = d.ny; a.cb_lo[f] = 1; }
    for (int n = 0; n < d.nth; ++n) {
        a.cf_lo[3 + n] = h->jstart_th[n];
        a.cf_hi[3 + n] = h->jend_th[n];
        a.cb_lo[3 + n] = h->jstart_th[n] - 1;
    }
    a.temp1 = p.nu * h_bar[r] / 2.0;
    a.temp3 = zeta_bar[r] * h_bar[r];
    a.temp4 = TEMP4;
    a.temp5 = beta_bar[r] * h_bar[r];
    a.nu = p.nu; a.beta = p.beta; a.nu_v_scale = p.nu_v_scale; a.i_ro = p.i_ro;
    a.grav_x = p.grav_x; a.grav_y = p.grav_y; a.grav_z = p.grav_z;
    for (int n = 0; n < 4; ++n) {
        a.ri[n] = n < d.nth ? p.ri[n] : 0.0;
        a.pr[n] = n < d.nth ? p.pr[n] : 1.0;
        a.drhodx[n] = n < d.nth ? p.drhodx[n] : 0.0;
        a.drhodz[n] = n < d.nth ? p.drhodz[n] : 0.0;
    }
    a.forcing = 0.0;
    if (p.f_type == 1) a.forcing = TEMP4 * p.px0;
    else if (p.f_type == 2) a.forcing = TEMP4 * (p.px0 + p.amp_omega0 * std::cos(p.omega0 * time));
    a.rk_step = rk_step;
    a.store_cf = 1;
    return a;
}

// The column kernel's arguments of one Fourier-space substage (no LES); with
// cfl the projection waits until COURANT has run.
static ColArgs dns_col_args(Handle* h, const CnArgs& a, bool cfl) {
    ColArgs ca;
    ca.cn = a;
    ca.k2 = h->d_k2;
    ca.rows = h->d_rows;
    ca.phitab = h->d_phitab;
    ca.phi = h->phi;
    ca.inv_h = 1.0 / a.temp4;
    ca.project = cfl ? 0 : 1;     // COURANT sees the velocity before the projection
    ca.update_cp = 1;
    ca.store_phi = 0;             // phi stays where REM_DIV_CHAN alone puts it
    ca.nan_flag = h->d_nan;
    ca.pair_blocked = h->pb ? 1 : 0;
    ca.mean_split = h->fp32 ? 1 : 0;
    ca.jlo_prod = h->jlo_prod;
    return ca;
}

// CN rows and partition factors of substage r (k_cn_part) into that
// substage's slot, unless the slot already holds them for this TEMP1; points
// a.bcv / a.kind at the slot and returns the factor tables in *tabs.
static int ensure_cn_tables(Handle* h, CnArgs& a, int r, const double** tabs) {
    const Dims& d = h->d;
    const size_t tsz = part_table_doubles(d.nyp) * d.nf, rsz = (size_t)d.nyp * d.nf;
    double* t = h->d_tabs + (size_t)r * tsz;
    a.bcv = h->bcv + (size_t)r * rsz;
    a.kind = h->kind + (size_t)r * rsz;
    *tabs = t;
    if (h->tab_ok[r] && h->tab_temp1[r] == a.temp1) return DIABLO_OK;
    {
        ProfScope ps(h, DIABLO_KERNEL_CN_COEF);
        CK(launch_cn_part(d, a, t, const_cast<double*>(a.bcv), const_cast<signed char*>(a.kind), h->bc_type, h->bc_c1,
                          h->st));
    }
    h->launches += 1;
    h->tab_ok[r] = true;
    h->tab_temp1[r] = a.temp1;
    return DIABLO_OK;
}

// Spectral fields [0,nfld) of S (stride s_field) -> physical fields of P
// (stride pf), planes j0..j0+np-1, FP64.
static cudaError_t les_to_phys(Handle* h, const double2* S, int nfld, double* P, int j0, int np) {
    const Dims& d = h->d;
    const size_t pf = (size_t)d.nyp * d.nz * d.nx;
    cudaError_t e = launch_zinv<double>(d, S, h->s_field, h->lx, h->x_field, nfld, j0, np, h->pz, h->twz_d, h->st);
    for (int f = 0; f < nfld && e == cudaSuccess; ++f)
        e = launch_xinv(d, (const double2*)h->lx + (size_t)f * h->x_field, P + (size_t)f * pf, j0, np, h->pm, h->twm_d,
                        h->twn_d, h->st);
    h->launches += 1 + nfld;
    return e;
}

// Physical fields -> spectral fields (FFT_XZ_TO_FOURIER), planes j0..j0+np-1.
static cudaError_t les_to_fourier(Handle* h, const double* P, int nfld, double2* S, int j0, int np) {
    const Dims& d = h->d;
    const size_t pf = (size_t)d.nyp * d.nz * d.nx;
    cudaError_t e = cudaSuccess;
    for (int f = 0; f < nfld && e == cudaSuccess; ++f) {
        double2* X = (double2*)h->lx + (size_t)f * h->x_field;
        e = launch_xfwd(d, P + (size_t)f * pf, X, j0, np, h->pm, h->twm_d, h->twn_d, h->st);
        if (e == cudaSuccess) e = launch_zfwd_pack(d, X, S + (size_t)f * h->s_field, j0, np, h->pz, h->twz_d, h->st);
    }
    h->launches += 2 * nfld;
    return e;
}

// USER_RHS_CHAN_FOURIER / USER_RHS_CHAN_PHYSICAL (user_rhs.f:1-122): run the
// callbacks that are set and leave the sum of their Fourier-space terms in
// h->ufa (*any = true).  U (P layout, nf fields) is the physical state when
// the caller already has it (the LES branch); otherwise, and only for the
// physical hook, it is made here from CU with the FP64 transforms.  Uses xb
// and api_s as scratch: call before the substage's own transforms.
static int user_rhs(Handle* h, int rk_step, int time_step, double time, const double* U, bool* any) {
    *any = false;
    if (!h->urhs_fn[0] && !h->urhs_fn[1]) return DIABLO_OK;
    const Dims& d = h->d;
    const size_t pf = (size_t)d.nyp * d.nz * d.nx;
    if (!h->ufa) {
        cudaError_t e = cudaMalloc((void**)&h->ufa, sizeof(double2) * h->s_field * d.nf);
        if (e != cudaSuccess) { h->ufa = nullptr; return fail(DIABLO_ENOMEM, "user right-hand side buffer"); }
    }
    CK(cudaMemsetAsync(h->ufa, 0, sizeof(double2) * h->s_field * d.nf, h->st));
    diablo_user_rhs_args a;
    std::memset(&a, 0, sizeof(a));
    a.rk_step = rk_step; a.time_step = time_step; a.time = time;
    a.nx = d.nx; a.ny = d.ny; a.nz = d.nz; a.n_th = d.nth; a.nkx = d.nkx; a.tnkz = d.tnkz;
    a.s_field = (long long)h->s_field; a.s_plane = (long long)h->s_plane; a.s_row = d.ldx;
    a.p_field = (long long)pf; a.p_plane = (long long)d.nz * d.nx;
    a.cu = reinterpret_cast<const double*>(h->cu);
    a.cf_add = reinterpret_cast<double*>(h->ufa);
    a.stream = (void*)h->st;
    if (h->urhs_fn[DIABLO_USER_RHS_FOURIER]) {
        h->urhs_fn[DIABLO_USER_RHS_FOURIER](h->urhs_user[DIABLO_USER_RHS_FOURIER], &a);
        CK(cudaGetLastError());
    }
    if (h->urhs_fn[DIABLO_USER_RHS_PHYSICAL]) {
        if (!h->uphys) {
            cudaError_t e = cudaMalloc((void**)&h->uphys, sizeof(double) * pf * 2 * d.nf);
            if (e != cudaSuccess) { h->uphys = nullptr; return fail(DIABLO_ENOMEM, "user right-hand side fields"); }
        }
        double* fadd = h->uphys + pf * d.nf;
        if (!U) {
            CK(launch_zinv<double>(d, h->cu, h->s_field, h->xb, h->x_field, d.nf, 0, d.nyp, h->pz, h->twz_d, h->st));
            for (int f = 0; f < d.nf; ++f)
                CK(launch_xinv(d, (const double2*)h->xb + (size_t)f * h->x_field, h->uphys + (size_t)f * pf, 0, d.nyp,
                               h->pm, h->twm_d, h->twn_d, h->st));
            h->launches += 1 + d.nf;
            U = h->uphys;
        }
        CK(cudaMemsetAsync(fadd, 0, sizeof(double) * pf * d.nf, h->st));
        a.u = U;
        a.f_add = fadd;
        h->urhs_fn[DIABLO_USER_RHS_PHYSICAL](h->urhs_user[DIABLO_USER_RHS_PHYSICAL], &a);
        CK(cudaGetLastError());
        for (int f = 0; f < d.nf; ++f) {       // FFT_XZ_TO_FOURIER(S1,CS1,0,NY+1), then CF += CS1
            CK(launch_xfwd(d, fadd + (size_t)f * pf, h->xb, 0, d.nyp, h->pm, h->twm_d, h->twn_d, h->st));
            CK(launch_zfwd_pack(d, h->xb, h->api_s, 0, d.nyp, h->pz, h->twz_d, h->st));
            k_add_user<double><<<1184, 256, 0, h->st>>>(reinterpret_cast<cpx<double>*>(h->ufa + (size_t)f * h->s_field),
                                                        h->api_s, h->s_field);
            CK(cudaGetLastError());
        }
        h->launches += 3 * d.nf;
    }
    *any = true;
    return DIABLO_OK;
}

// RK_CHAN_1 with LES set (channel.f:62-1073 with the LES branches), in the
// reference's order: Fourier right-hand sides; when the subgrid model runs
// (sgs), les_chan (strain rates, |S|, NU_T, tau_ij and the cross terms into
// CF), the physical velocity BCs and the scalars' horizontal eddy
// diffusivity; the nonlinear terms from the physical fields; CR to physical
// space, the explicit CN half with the eddy-viscosity terms; one tridiagonal
// solve per physical column and field; COURANT at the last substage on the
// solved physical velocity; the fields back to Fourier space, the projection
// and the pressure update.
static int les_substage(Handle* h, int rk_step, int time_step, double time, double* delta_t, double* h_bar,
                        const double* beta_bar, const double* zeta_bar, bool sgs) {
    const diablo_params& p = h->p;
    const Dims& d = h->d;
    const int r = rk_step - 1;
    const size_t pf = (size_t)d.nyp * d.nz * d.nx;
    const int nyp = d.nyp;
    // LES_MODEL_TYPE 4 runs the learned closure when one is attached and
    // falls back to the dynamic model otherwise
    const bool use_mlp = p.les_model_type == 4 && h->mlp;
    const bool dyn = p.les_model_type == 2 || (p.les_model_type == 4 && !h->mlp);
    // filter widths with -2 C^2 absorbed: the constant model's, or the
    // dynamic model's of this substage
    const double* delta_yf = dyn ? h->d_dyn + 2 * nyp : h->d_delta;
    const double* delta_y = delta_yf + nyp;
    CnArgs a = substage_args(h, rk_step, time, h_bar, beta_bar, zeta_bar);
    ProfScope ps(h, DIABLO_KERNEL_OTHER);
    CK(launch_les_pre(a, h->d_k2, h->lr, h->st));
    h->launches += 1;
    if (sgs && use_mlp) {
        // the learned closure: ghost cells as les_chan sets them, features of
        // the resolved field at GYF rows 2..NY-1, the network's stresses, and
        // their divergence into CF (explicit; NU_T stays zero)
        dim3 grid((d.nkxp + 127) / 128, d.nkzt);
        k_apply_bc_vel<<<grid, 128, 0, h->st>>>(d, h->cu, h->d_dy, h->d_dyf, p);
        CK(cudaGetLastError());
        CK(launch_les_bc(d, h->cu, p, h->st));
        CK(les_to_phys(h, h->cu, 3, h->lu, 0, nyp));
        const long long n = (long long)(d.ny - 2) * d.nz * d.nx;
        CK(launch_sgs_samples(d, h->lu, h->d_gyf, h->d_dyf, h->dx, h->dz, p.nu, 1, 1, h->mlp_x, nullptr, h->mlp_s,
                              h->st));
        CK(launch_mlp_forward(h->mlp, h->mlp_x, n, h->mlp_t, h->st));
        CK(launch_mlp_tau_fields(d, h->mlp_t, h->mlp_s, h->d_dy, h->d_dyf, h->lb, h->st));
        CK(launch_phys_bc_vel(d, h->lu, h->d_dy, h->d_dyf, p, h->st));
        CK(les_to_fourier(h, h->lb, 6, h->ls, 0, nyp));
        CK(launch_mlp_tau_cf(d, h->ls, h->cf, h->d_kx, h->d_kz, h->d_dy, h->d_dyf, h->st));
        h->launches += 8;
    } else if (sgs) {
        // les_chan: ghost cells (APPLY_BC_VEL_MPI, APPLY_BC_LES), strain rates
        dim3 grid((d.nkxp + 127) / 128, d.nkzt);
        k_apply_bc_vel<<<grid, 128, 0, h->st>>>(d, h->cu, h->d_dy, h->d_dyf, p);
        CK(cudaGetLastError());
        CK(launch_les_bc(d, h->cu, p, h->st));
        CK(launch_les_strain(d, h->cu, h->d_kx, h->d_kz, h->d_dy, h->d_dyf, h->ls, h->st));
        h->launches += 3;
        CK(les_to_phys(h, h->ls, 6, h->la, 0, nyp));
        CK(les_to_phys(h, h->cu, 3, h->lu, 0, nyp));
        if (dyn) {
            CK(launch_dyn_widths(d, h->la, h->lu, h->cu, h->d_dy, h->d_dyf, std::pow(9.0, 2.0 / 3.0), h->d_dyn,
                                 h->d_dyn + 2 * nyp, h->st));
            h->launches += 2;
        }
        CK(launch_les_sgs(d, h->la, h->lu, h->cu, h->d_dy, h->d_dyf, delta_y, h->lb, h->nut, h->st));
        CK(launch_phys_bc_vel(d, h->lu, h->d_dy, h->d_dyf, p, h->st));
        h->launches += 2;
        h->nut_set = true;
        CK(les_to_fourier(h, h->lb, 7, h->ls, 0, nyp));
        CK(launch_les_tau_cf(d, h->ls, h->cf, h->d_kx, h->d_kz, h->d_dyf, delta_yf, delta_y, h->st));
        h->launches += 1;
        // horizontal eddy diffusivity of each scalar, KAPPA_T = NU_T
        for (int n = 0; n < d.nth; ++n) {
            const double2* cth = h->cu + (size_t)(3 + n) * h->s_field;
            CK(launch_les_kgrad(d, cth, h->d_kx, h->d_kz, h->ls, h->st));
            CK(les_to_phys(h, h->ls, 2, h->la, 0, nyp));
            CK(launch_les_kmul(d, h->la, h->nut, h->st));
            CK(les_to_fourier(h, h->la, 2, h->ls, 0, nyp));
            CK(launch_les_kcf(d, h->ls, h->cf + (size_t)(3 + n) * h->s_field, h->d_kx, h->d_kz, h->jstart_th[n],
                              h->jend_th[n], h->st));
            h->launches += 3;
        }
    } else {
        CK(les_to_phys(h, h->cu, 3, h->lu, 0, nyp));
    }
    if (d.nth > 0) CK(les_to_phys(h, h->cu + 3 * h->s_field, d.nth, h->lu + 3 * pf, 0, nyp));
    {   // USER_RHS_CHAN_FOURIER / _PHYSICAL (channel.f:297, 578): CF += their terms
        bool any = false;
        int rc = user_rhs(h, rk_step, time_step, time, h->lu, &any);
        if (rc) return rc;
        if (any) {
            k_add_user<double><<<1184, 256, 0, h->st>>>(reinterpret_cast<cpx<double>*>(h->cf), h->ufa,
                                                        h->s_field * d.nf);
            CK(cudaGetLastError());
            h->launches += 1;
        }
    }
    // nonlinear terms from the physical fields: x spectra, then the products
    // and z-forward kernels of the Fourier-space path
    for (int f = 0; f < d.nf; ++f)
        CK(launch_xfwd(d, h->lu + (size_t)f * pf, (double2*)h->xb + (size_t)f * h->x_field, 0, nyp, h->pm, h->twm_d,
                       h->twn_d, h->st));
    CK(launch_products<double>(d, h->xb, h->yb, h->jlo_prod, d.ny, h->prod_chunk, h->d_dy, h->d_dyf, h->d_kx, h->pm,
                               h->twm_d, h->twn_d, h->st));
    CK(launch_zfwd_nl<double>(d, h->yb, h->nl, h->jlo_prod, d.ny, h->zf_planes, h->d_kx, h->d_kz, h->pz, h->twz_d,
                              h->st));
    CK(launch_les_post(a, (const double2*)h->nl, h->lr, h->st));
    h->launches += d.nf + 3;
    // CN in physical space
    CK(les_to_phys(h, h->lr, d.nf, h->la, 0, nyp));
    LesArgs la;
    la.d = d;
    la.dy = h->d_dy;
    la.dyf = h->d_dyf;
    la.rows = h->d_rows;
    la.temp1 = a.temp1;
    la.temp2 = h_bar[r] / 2.0;
    la.nu_v_scale = p.nu_v_scale;
    for (int n = 0; n < 4; ++n) la.pr[n] = a.pr[n];
    for (int f = 0; f < MAXF; ++f) {
        la.j_lo[f] = a.cf_lo[f];
        la.j_hi[f] = a.cf_hi[f];
        la.out_lo[f] = a.cb_lo[f];
        la.bc_type[f][0] = h->bc_type[2 * f];
        la.bc_type[f][1] = h->bc_type[2 * f + 1];
        la.bc_c1[f][0] = h->bc_c1[2 * f];
        la.bc_c1[f][1] = h->bc_c1[2 * f + 1];
    }
    CK(launch_les_explicit(la, h->lu, h->la, h->nut, h->st));
    CK(launch_les_solve(la, h->la, h->nut, h->lb, h->lu, h->st));
    h->launches += 2;
    const double inv_h = 1.0 / a.temp4;
    if (p.variable_dt && rk_step == 3 && (time_step % p.update_dt) == 0) {
        int rc = courant(h, delta_t, h_bar, h->lu);
        if (rc) return rc;
    }
    CK(les_to_fourier(h, h->lu, d.nf, h->cu, 0, nyp));
    return rem_div(h, 1, inv_h);
}

int diablo_gpu_rk_chan_1(void* handle, int rk_step, int time_step, double time, double* delta_t,
                         double* h_bar, const double* beta_bar, const double* zeta_bar) {
    Handle* h = (Handle*)handle;
    if (!h || !delta_t || !h_bar || !beta_bar || !zeta_bar) return fail(DIABLO_EINVAL, "null pointer argument");
    if (rk_step < 1 || rk_step > 3) return fail(DIABLO_EINVAL, "rk_step must be 1, 2 or 3");
    const diablo_params& p = h->p;
    const Dims& d = h->d;
    const int r = rk_step - 1;
    if (p.les) {
        // the subgrid model waits for the spin-up of a new flow (channel.f:303);
        // until NU_T is first computed it is zero and the LES terms add
        // nothing, so the Fourier-space path gives the same step
        const bool sgs = !p.create_new_flow || time_step > 100;
        if (sgs || h->nut_set) return les_substage(h, rk_step, time_step, time, delta_t, h_bar, beta_bar, zeta_bar, sgs);
    }
    const double TEMP4 = h_bar[r];       // channel.f:77-81; the others are formed by substage_args
    int rc;
    bool user = false;    // USER_RHS_CHAN_FOURIER / _PHYSICAL (channel.f:297, 578)
    if ((rc = user_rhs(h, rk_step, time_step, time, nullptr, &user))) return rc;
    if (h->fp32) rc = run_transforms<float>(h);
    else rc = run_transforms<double>(h);
    if (rc) return rc;
    if (user) {           // their terms join the nonlinear term, which CF takes whole
        if (h->fp32) k_add_user<float><<<1184, 256, 0, h->st>>>((cpx<float>*)h->nl, h->ufa, h->s_field * d.nf);
        else k_add_user<double><<<1184, 256, 0, h->st>>>((cpx<double>*)h->nl, h->ufa, h->s_field * d.nf);
        CK(cudaGetLastError());
        h->launches += 1;
    }
    CnArgs a = substage_args(h, rk_step, time, h_bar, beta_bar, zeta_bar);
    const double* tabs = nullptr;
    if ((rc = ensure_cn_tables(h, a, r, &tabs))) return rc;
    const bool cfl = p.variable_dt && rk_step == 3 && (time_step % p.update_dt) == 0;
    const ColArgs ca = dns_col_args(h, a, cfl);
    {
        ProfScope ps(h, DIABLO_KERNEL_COLUMN);
        if (h->fp32) CK(launch_colpart<cpx<float>>(ca, (const cpx<float>*)h->nl, tabs, h->st));
        else CK(launch_colpart<cpx<double>>(ca, (const cpx<double>*)h->nl, tabs, h->st));
    }
    h->launches += 1;
    if (!cfl) return DIABLO_OK;
    // COURANT at the last substage (channel.f:1037-1040), then REM_DIV and the
    // pressure update with the h of this substage
    if ((rc = courant(h, delta_t, h_bar))) return rc;
    return rem_div(h, 1, 1.0 / TEMP4);
}

// n RK3 steps as replays of one captured step.  The step is static when its
// launches and their arguments do not change from step to step: a fixed time
// step (COURANT reads DELTA_T back to the host), no user right-hand side (host
// callbacks), forcing that does not depend on time, and, on the LES branch,
// the subgrid model running from the first of these steps on.  The first
// call after a change of H_BAR/BETA_BAR/ZETA_BAR, of the launch shapes or of
// the attached network runs one step directly (it sets up the lazily
// allocated buffers and the cached CN factors) and captures the next.
int diablo_gpu_step_graph(void* handle, int nsteps, int time_step, const double* h_bar, const double* beta_bar,
                          const double* zeta_bar) {
    Handle* h = (Handle*)handle;
    if (!h || !h_bar || !beta_bar || !zeta_bar) return fail(DIABLO_EINVAL, "null pointer argument");
    if (nsteps < 0) return fail(DIABLO_EINVAL, "nsteps must be >= 0");
    const diablo_params& p = h->p;
    if (p.variable_dt) return fail(DIABLO_ENOTSUP, "step graph: VARIABLE_DT reads DELTA_T back every step");
    if (p.f_type == 2) return fail(DIABLO_ENOTSUP, "step graph: the forcing depends on time");
    if (h->urhs_fn[0] || h->urhs_fn[1]) return fail(DIABLO_ENOTSUP, "step graph: a user right-hand side is set");
    if (h->profiling) return fail(DIABLO_ENOTSUP, "step graph: kernel profiling is on");
    if (p.les && p.create_new_flow && time_step + 1 <= 100)
        return fail(DIABLO_ENOTSUP, "step graph: the subgrid model starts within these steps");
    if (nsteps == 0) return DIABLO_OK;
    double coef[9];
    for (int r = 0; r < 3; ++r) { coef[r] = h_bar[r]; coef[3 + r] = beta_bar[r]; coef[6 + r] = zeta_bar[r]; }
    bool same = h->sg_exec && h->sg_prod == h->prod_chunk && h->sg_zf == h->zf_planes && h->sg_mlp == h->mlp;
    for (int q = 0; q < 9 && same; ++q) same = h->sg_coef[q] == coef[q];
    double hb[3] = {h_bar[0], h_bar[1], h_bar[2]}, dt = 0.0;
    int rc;
    if (!same) {
        if (h->sg_exec) { cudaGraphExecDestroy(h->sg_exec); h->sg_exec = nullptr; }
        if (h->sg_graph) { cudaGraphDestroy(h->sg_graph); h->sg_graph = nullptr; }
        for (int r = 1; r <= 3; ++r)
            if ((rc = diablo_gpu_rk_chan_1(handle, r, time_step + 1, 0.0, &dt, hb, beta_bar, zeta_bar))) return rc;
        nsteps -= 1;
        const long long l0 = h->launches;
        CK(cudaStreamSynchronize(h->st));
        cudaError_t e = cudaStreamBeginCapture(h->st, cudaStreamCaptureModeRelaxed);
        if (e != cudaSuccess) return fail(DIABLO_ECUDA, std::string("step graph capture: ") + cudaGetErrorString(e));
        rc = DIABLO_OK;
        for (int r = 1; r <= 3 && rc == DIABLO_OK; ++r)
            rc = diablo_gpu_rk_chan_1(handle, r, time_step + 2, 0.0, &dt, hb, beta_bar, zeta_bar);
        cudaGraph_t g = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(h->st, &g);
        if (rc != DIABLO_OK || ee != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return rc != DIABLO_OK ? rc : fail(DIABLO_ECUDA, std::string("step graph end capture: ") + cudaGetErrorString(ee));
        }
        e = cudaGraphInstantiate(&h->sg_exec, g, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(g);
            h->sg_exec = nullptr;
            return fail(DIABLO_ECUDA, std::string("step graph instantiate: ") + cudaGetErrorString(e));
        }
        h->sg_graph = g;
        h->sg_launches = h->launches - l0;
        h->launches = l0;
        for (int q = 0; q < 9; ++q) h->sg_coef[q] = coef[q];
        h->sg_prod = h->prod_chunk;
        h->sg_zf = h->zf_planes;
        h->sg_mlp = h->mlp;
    }
    for (int s = 0; s < nsteps; ++s) CK(cudaGraphLaunch(h->sg_exec, h->st));
    h->launches += h->sg_launches * nsteps;
    return DIABLO_OK;
}

int diablo_gpu_download_nu_t(void* handle, double* nu_t) {
    Handle* h = (Handle*)handle;
    if (!h || !nu_t) return fail(DIABLO_EINVAL, "null pointer argument");
    if (!h->p.les) return fail(DIABLO_EINVAL, "NU_T exists only when LES is set");
    CK(copy_physical(h, h->nut, nullptr, nu_t, 0, h->d.nyp));
    CK(cudaStreamSynchronize(h->st));
    return DIABLO_OK;
}

static int ensure_work(Handle* h);

int diablo_gpu_sgs_samples(void* handle, int width, int stride, float* x, float* t, float* scale,
                           long long capacity, long long* n) {
    Handle* h = (Handle*)handle;
    if (!h || !n) return fail(DIABLO_EINVAL, "null pointer argument");
    const Dims& d = h->d;
    if (width < 1 || width % 2 == 0 || width > d.nx || width > d.nz)
        return fail(DIABLO_EINVAL, "filter width must be odd and at most NX, NZ");
    if (stride < 1) return fail(DIABLO_EINVAL, "stride must be >= 1");
    const long long ns = (long long)(d.ny - 2) * ((d.nx + stride - 1) / stride) * ((d.nz + stride - 1) / stride);
    *n = ns;
    if (!x || !t || !scale || capacity < ns) return fail(DIABLO_EINVAL, "sample arrays too small (the count is in *n)");
    int rc = ensure_work(h);
    if (rc) return rc;
    const size_t pf = (size_t)d.nyp * d.nz * d.nx;
    CK(launch_zinv<double>(d, h->cu, h->s_field, h->xb, h->x_field, 3, 0, d.nyp, h->pz, h->twz_d, h->st));
    for (int f = 0; f < 3; ++f)
        CK(launch_xinv(d, (const double2*)h->xb + (size_t)f * h->x_field, h->pw + (size_t)f * pf, 0, d.nyp, h->pm,
                       h->twm_d, h->twn_d, h->st));
    float *dx_ = nullptr, *dt_ = nullptr, *ds_ = nullptr;
    cudaError_t e = cudaMalloc((void**)&dx_, sizeof(float) * 11 * (size_t)ns);
    if (e == cudaSuccess) e = cudaMalloc((void**)&dt_, sizeof(float) * 6 * (size_t)ns);
    if (e == cudaSuccess) e = cudaMalloc((void**)&ds_, sizeof(float) * (size_t)ns);
    if (e == cudaSuccess)
        e = launch_sgs_samples(d, h->pw, h->d_gyf, h->d_dyf, h->dx, h->dz, h->p.nu, width, stride, dx_, dt_, ds_,
                               h->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(x, dx_, sizeof(float) * 11 * (size_t)ns, cudaMemcpyDeviceToHost, h->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(t, dt_, sizeof(float) * 6 * (size_t)ns, cudaMemcpyDeviceToHost, h->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(scale, ds_, sizeof(float) * (size_t)ns, cudaMemcpyDeviceToHost, h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
    cudaFree(dx_);
    cudaFree(dt_);
    cudaFree(ds_);
    h->launches += 5;
    if (e != cudaSuccess) return fail(DIABLO_ECUDA, std::string("closure samples: ") + cudaGetErrorString(e));
    return DIABLO_OK;
}

int diablo_gpu_set_user_rhs(void* handle, int kind, diablo_user_rhs_fn fn, void* user) {
    Handle* h = (Handle*)handle;
    if (!h) return fail(DIABLO_EINVAL, "null handle");
    if (kind != DIABLO_USER_RHS_FOURIER && kind != DIABLO_USER_RHS_PHYSICAL)
        return fail(DIABLO_EINVAL, "kind must be DIABLO_USER_RHS_FOURIER or DIABLO_USER_RHS_PHYSICAL");
    h->urhs_fn[kind] = fn;
    h->urhs_user[kind] = fn ? user : nullptr;
    return DIABLO_OK;
}

int diablo_gpu_set_sgs_mlp(void* handle, void* mlp) {
    Handle* h = (Handle*)handle;
    if (!h) return fail(DIABLO_EINVAL, "null handle");
    if (!h->p.les) return fail(DIABLO_EINVAL, "the closure needs an LES instance");
    if (mlp && !h->mlp_x) {
        const size_t n = (size_t)(h->d.ny - 2) * h->d.nz * h->d.nx;
        cudaError_t e = cudaMalloc((void**)&h->mlp_x, sizeof(float) * 11 * n);
        if (e == cudaSuccess) e = cudaMalloc((void**)&h->mlp_t, sizeof(float) * 6 * n);
        if (e == cudaSuccess) e = cudaMalloc((void**)&h->mlp_s, sizeof(float) * n);
        if (e != cudaSuccess) {
            cudaFree(h->mlp_x);
            cudaFree(h->mlp_t);
            cudaFree(h->mlp_s);
            h->mlp_x = h->mlp_t = h->mlp_s = nullptr;
            return fail(DIABLO_ENOMEM, std::string("closure buffers: ") + cudaGetErrorString(e));
        }
    }
    h->mlp = mlp;
    return DIABLO_OK;
}

int diablo_gpu_rk_chan_2(void* handle) {
    (void)handle;
    return fail(DIABLO_ENOTSUP, "RK_CHAN_2 is not supported (the reference stops here too)");
}

int diablo_gpu_rem_div_chan(void* handle) {
    Handle* h = (Handle*)handle;
    if (!h) return fail(DIABLO_EINVAL, "null handle");
    int rc = rem_div(h, 0, 0.0);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->st));
    return DIABLO_OK;
}

int diablo_gpu_apply_bc_vel(void* handle) {
    Handle* h = (Handle*)handle;
    if (!h) return fail(DIABLO_EINVAL, "null handle");
    dim3 grid((h->d.nkxp + 127) / 128, h->d.nkzt);
    { ProfScope ps(h, DIABLO_KERNEL_OTHER);
      k_apply_bc_vel<<<grid, 128, 0, h->st>>>(h->d, h->cu, h->d_dy, h->d_dyf, h->p); }
    CK(cudaGetLastError());
    h->launches += 1;
    CK(cudaStreamSynchronize(h->st));
    return DIABLO_OK;
}

int diablo_gpu_courant(void* handle, double* delta_t, double* h_bar) {
    Handle* h = (Handle*)handle;
    if (!h || !delta_t || !h_bar) return fail(DIABLO_EINVAL, "null pointer argument");
    return courant(h, delta_t, h_bar);
}

static int ensure_phys(Handle* h) {
    if (h->phys) return DIABLO_OK;
    const size_t bytes = sizeof(double) * (size_t)h->d.nyp * h->d.nz * h->d.nx;
    cudaError_t e = cudaMalloc((void**)&h->phys, bytes);
    if (e != cudaSuccess) return fail(DIABLO_ENOMEM, "physical buffer allocation failed");
    return DIABLO_OK;
}

int diablo_gpu_fft_xz_to_fourier(void* handle, const double* v, double* vv, int jmin, int jmax) {
    Handle* h = (Handle*)handle;
    if (!h || !v || !vv) return fail(DIABLO_EINVAL, "null pointer argument");
    const Dims& d = h->d;
    if (jmin < 0 || jmax > d.ny + 1) return fail(DIABLO_EINVAL, "plane range outside 0..NY+1");
    if (jmax < jmin) return DIABLO_OK;
    int rc = ensure_phys(h);
    if (rc) return rc;
    const int np = jmax - jmin + 1;
    CK(copy_physical(h, h->phys, v, nullptr, jmin, np));
    { ProfScope ps(h, DIABLO_KERNEL_OTHER);
      CK(launch_xfwd(d, h->phys, h->xb, jmin, np, h->pm, h->twm_d, h->twn_d, h->st));
      CK(launch_zfwd_pack(d, h->xb, h->api_s, jmin, np, h->pz, h->twz_d, h->st)); }
    h->launches += 2;
    CK(copy_fourier(h, h->api_s, nullptr, vv, jmin, np));
    CK(cudaStreamSynchronize(h->st));
    // modes NKX < I <= NXP are zero, as the reference writes them (mpi.f:1503-1517)
    const size_t cx = (size_t)h->nxp + 1, cz = (size_t)d.nz + 2;
    for (int j = jmin; j <= jmax; ++j)
        for (int k = 0; k <= d.tnkz; ++k)
            std::memset(vv + 2 * ((size_t)j * cz * cx + (size_t)k * cx + d.nkxp), 0,
                        sizeof(double) * 2 * (cx - d.nkxp));
    return DIABLO_OK;
}

int diablo_gpu_fft_xz_to_physical(void* handle, const double* vv, double* v, int jmin, int jmax) {
    Handle* h = (Handle*)handle;
    if (!h || !v || !vv) return fail(DIABLO_EINVAL, "null pointer argument");
    const Dims& d = h->d;
    if (jmin < 0 || jmax > d.ny + 1) return fail(DIABLO_EINVAL, "plane range outside 0..NY+1");
    if (jmax < jmin) return DIABLO_OK;
    int rc = ensure_phys(h);
    if (rc) return rc;
    const int np = jmax - jmin + 1;
    CK(copy_fourier(h, h->api_s, vv, nullptr, jmin, np));
    { ProfScope ps(h, DIABLO_KERNEL_OTHER);
      CK(launch_zinv<double>(d, h->api_s, h->s_field, h->xb, h->x_field, 1, jmin, np, h->pz, h->twz_d, h->st));
      CK(launch_xinv(d, h->xb, h->phys, jmin, np, h->pm, h->twm_d, h->twn_d, h->st)); }
    h->launches += 2;
    CK(copy_physical(h, h->phys, nullptr, v, jmin, np));
    CK(cudaStreamSynchronize(h->st));
    return DIABLO_OK;
}

static int ensure_work(Handle* h) {
    if (h->pw) return DIABLO_OK;
    const size_t pf = (size_t)h->d.nyp * h->d.nz * h->d.nx;
    cudaError_t e = cudaMalloc((void**)&h->pw, sizeof(double) * 4 * pf);
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->d_me, sizeof(double) * 4 * h->d.nyp);
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->d_sums, sizeof(double) * 9 * h->d.nyp);
    if (e != cudaSuccess) {
        cudaFree(h->pw); cudaFree(h->d_me); cudaFree(h->d_sums);
        h->pw = h->d_me = h->d_sums = nullptr;
        return fail(DIABLO_ENOMEM, std::string("work buffers: ") + cudaGetErrorString(e));
    }
    return DIABLO_OK;
}

// POISSON_P_CHAN (channel.f:1217-1453): CP from the current velocity and
// scalars.  The nine gradient fields go to physical space one at a time; the
// products are summed there and transformed forward once.  CF is left as it
// was (the reference uses CF1..CF3 as scratch here, so their values after
// this call are not part of its result).
int diablo_gpu_poisson_p_chan(void* handle) {
    Handle* h = (Handle*)handle;
    if (!h) return fail(DIABLO_EINVAL, "null handle");
    int rc = ensure_work(h);
    if (rc) return rc;
    const Dims& d = h->d;
    const size_t pf = (size_t)d.nyp * d.nz * d.nx;
    double* acc = h->pw;
    double* pa = h->pw + pf;
    double* pb = h->pw + 2 * pf;
    const int j0 = 2, np = d.ny - 1;
    ProfScope ps(h, DIABLO_KERNEL_OTHER);
    auto to_phys = [&](int kind, double* dst) -> cudaError_t {
        cudaError_t e = launch_grad_field(d, kind, h->cu, h->api_s, h->d_kx, h->d_kz, h->d_dyf, h->st);
        if (e == cudaSuccess)
            e = launch_zinv<double>(d, h->api_s, h->s_field, h->xb, h->x_field, 1, j0, np, h->pz, h->twz_d, h->st);
        if (e == cudaSuccess) e = launch_xinv(d, h->xb, dst, j0, np, h->pm, h->twm_d, h->twn_d, h->st);
        h->launches += 3;
        return e;
    };
    // (du/dx)^2 + (dv/dy)^2 + (dw/dz)^2
    for (int k = 0; k < 3; ++k) {
        CK(to_phys(k, pa));
        CK(launch_phys_fma(d, acc, pa, pa, 1.0, k == 0, h->st));
    }
    // 2 (du/dy)(dv/dx), 2 (dw/dy)(dv/dz), 2 (du/dz)(dw/dx)
    for (int k = 3; k < 9; k += 2) {
        CK(to_phys(k, pa));
        CK(to_phys(k + 1, pb));
        CK(launch_phys_fma(d, acc, pa, pb, 2.0, 0, h->st));
    }
    h->launches += 6;
    CK(launch_xfwd(d, acc, h->xb, j0, np, h->pm, h->twm_d, h->twn_d, h->st));
    CK(launch_zfwd_pack(d, h->xb, h->api_s, j0, np, h->pz, h->twz_d, h->st));
    PoissonArgs a;
    a.d = d;
    a.rhs = h->api_s;
    a.cth = h->cu + 3 * h->s_field;
    a.cp = h->cp;
    a.bsc = h->bsc;
    a.gsc = h->gsc;
    a.kx = h->d_kx;
    a.kz = h->d_kz;
    a.dy = h->d_dy;
    a.dyf = h->d_dyf;
    a.gyf = h->d_gyf;
    for (int n = 0; n < 4; ++n) a.ri[n] = n < d.nth ? h->p.ri[n] : 0.0;
    CK(launch_poisson_column(a, h->st));
    h->launches += 3;
    CK(cudaStreamSynchronize(h->st));
    return DIABLO_OK;
}

// SAVE_STATS_CHAN plane statistics (save_stats.f:104-347, 452-536) after
// APPLY_BC_VEL (save_stats.f:28-36), in FP64.  Means are the (0,0) modes;
// fluctuation sums run on the device over the physical fields.
int diablo_gpu_stats(void* handle, double* profiles) {
    Handle* h = (Handle*)handle;
    if (!h || !profiles) return fail(DIABLO_EINVAL, "null pointer argument");
    int rc = ensure_work(h);
    if (rc) return rc;
    const Dims& d = h->d;
    const size_t nyp = (size_t)d.nyp, pf = nyp * d.nz * d.nx;
    const int nstat_f = 3 + (d.nth > 0 ? 1 : 0);
    ProfScope ps(h, DIABLO_KERNEL_OTHER);
    {
        dim3 grid((d.nkxp + 127) / 128, d.nkzt);
        k_apply_bc_vel<<<grid, 128, 0, h->st>>>(d, h->cu, h->d_dy, h->d_dyf, h->p);
        CK(cudaGetLastError());
    }
    // (0,0) modes of U1, U2, U3, TH1 and CP
    std::vector<double2> m00((size_t)5 * nyp, make_double2(0.0, 0.0));
    for (int f = 0; f < 5; ++f) {
        const double2* src = f < 3 ? h->cu + (size_t)f * h->s_field
                           : f == 3 ? (d.nth > 0 ? h->cu + 3 * h->s_field : nullptr) : h->cp;
        if (!src) continue;
        CK(cudaMemcpy2DAsync(m00.data() + (size_t)f * nyp, sizeof(double2), src, sizeof(double2) * h->s_plane,
                             sizeof(double2), nyp, cudaMemcpyDeviceToHost, h->st));
    }
    CK(cudaStreamSynchronize(h->st));
    std::vector<double> me(4 * nyp);
    for (size_t j = 0; j < nyp; ++j)
        for (int f = 0; f < 4; ++f) me[f * nyp + j] = m00[f * nyp + j].x;
    CK(cudaMemcpyAsync(h->d_me, me.data(), sizeof(double) * me.size(), cudaMemcpyHostToDevice, h->st));
    CK(launch_zinv<double>(d, h->cu, h->s_field, h->xb, h->x_field, nstat_f, 0, d.nyp, h->pz, h->twz_d, h->st));
    for (int f = 0; f < nstat_f; ++f)
        CK(launch_xinv(d, (const double2*)h->xb + (size_t)f * h->x_field, h->pw + (size_t)f * pf, 0, d.nyp, h->pm,
                       h->twm_d, h->twn_d, h->st));
    CK(launch_stats_planes(d, h->pw, h->pw + pf, h->pw + 2 * pf, d.nth > 0 ? h->pw + 3 * pf : nullptr, h->d_me,
                           h->d_dy, h->d_dyf, h->d_sums, h->st));
    h->launches += 3 + nstat_f;
    std::vector<double> sums(9 * nyp);
    CK(cudaMemcpyAsync(sums.data(), h->d_sums, sizeof(double) * sums.size(), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    double* out = profiles;
    for (size_t q = 0; q < (size_t)DIABLO_NSTATS * nyp; ++q) out[q] = 0.0;
    auto O = [&](int s, size_t j) -> double& { return out[(size_t)s * nyp + j]; };
    auto S = [&](int k, size_t j) { return sums[(size_t)k * nyp + j]; };
    const double* ume = me.data();
    const double* wme = me.data() + 2 * nyp;
    const double* thme = me.data() + 3 * nyp;
    for (size_t j = 0; j < nyp; ++j) {
        O(DIABLO_STAT_UME, j) = me[j];
        O(DIABLO_STAT_VME, j) = me[nyp + j];
        O(DIABLO_STAT_WME, j) = me[2 * nyp + j];
        O(DIABLO_STAT_CP, j) = m00[4 * nyp + j].x;
    }
    // NX*NZ formed in single precision as in save_stats.f (FLOAT(NZ*NX))
    const double nn = (double)((float)d.nz * (float)d.nx);
    for (int j = 1; j <= d.ny; ++j) {
        const double dg = h->gyf[j] - h->gyf[j - 1];
        O(DIABLO_STAT_URMS, j) = std::sqrt(S(0, j) / nn);
        O(DIABLO_STAT_VRMS, j) = std::sqrt(S(1, j) / nn);
        O(DIABLO_STAT_WRMS, j) = std::sqrt(S(2, j) / nn);
        O(DIABLO_STAT_UV, j) = S(3, j) / nn;
        O(DIABLO_STAT_UW, j) = S(4, j) / nn;
        O(DIABLO_STAT_WV, j) = S(5, j) / nn;
        O(DIABLO_STAT_DUDY, j) = (ume[j] - ume[j - 1]) / dg;
        O(DIABLO_STAT_DWDY, j) = (wme[j] - wme[j - 1]) / dg;
        O(DIABLO_STAT_SHEAR, j) = S(6, j) / (double)(d.nx * d.nz);
        if (d.nth > 0) {
            O(DIABLO_STAT_THME, j) = thme[j];
            O(DIABLO_STAT_THRMS, j) = std::sqrt(S(7, j) / nn);
            O(DIABLO_STAT_THV, j) = S(8, j) / nn;
            O(DIABLO_STAT_DTHDY, j) = (thme[j] - thme[j - 1]) / dg;
        }
    }
    if (d.nth > 0) {
        O(DIABLO_STAT_THME, 0) = thme[0];
        O(DIABLO_STAT_THME, nyp - 1) = thme[nyp - 1];
    }
    return DIABLO_OK;
}

// The remaining profiles of SAVE_STATS_CHAN's mean.h5 and tke.h5
// (save_stats.f:270-347, 452-536, 937-1135): the base statistics above,
// then each Fourier field of k_stats_spec goes to physical space on its own
// and k_plane_terms adds its plane sums.  Physical U1..U3 stay in pw[0..2]
// from the base statistics; pw[3] takes one field at a time.
int diablo_gpu_mean_stats(void* handle, double* chan, double* scal, double* epsilon) {
    Handle* h = (Handle*)handle;
    if (!h || !chan || (h->d.nth > 0 && !scal)) return fail(DIABLO_EINVAL, "null pointer argument");
    const Dims& d = h->d;
    const size_t nyp = (size_t)d.nyp, pf = nyp * d.nz * d.nx;
    std::vector<double> base((size_t)DIABLO_NSTATS * nyp);
    int rc = diablo_gpu_stats(handle, base.data());
    if (rc) return rc;
    const int nsum = 4 + 3 * d.nth;
    if (!h->d_msums) {
        cudaError_t e = cudaMalloc((void**)&h->d_msums, sizeof(double) * (nsum + 1) * nyp);
        if (e != cudaSuccess) {
            h->d_msums = nullptr;
            return fail(DIABLO_ENOMEM, std::string("statistics sums: ") + cudaGetErrorString(e));
        }
        std::vector<double> rg(nyp, 0.0);
        for (int j = 1; j <= d.ny; ++j) rg[j] = 1.0 / (h->gy[j + 1] - h->gy[j - 1]);
        CK(cudaMemcpyAsync(h->d_msums + (size_t)nsum * nyp, rg.data(), sizeof(double) * nyp, cudaMemcpyHostToDevice, h->st));
    }
    ProfScope ps(h, DIABLO_KERNEL_OTHER);
    double* acc = h->d_msums;
    const double* rg = h->d_msums + (size_t)nsum * nyp;
    double *U1 = h->pw, *U2 = h->pw + pf, *U3 = h->pw + 2 * pf, *F = h->pw + 3 * pf;
    const double* ume = h->d_me;
    const double* vme = h->d_me + nyp;
    const double* wme = h->d_me + 2 * nyp;
    double* thm = h->d_me + 3 * nyp;
    // Fourier field `kind` (of CU, or of scalar cs) -> F on planes 1..NY
    auto field = [&](int kind, const double2* cs) -> cudaError_t {
        cudaError_t e = launch_stats_spec(d, kind, h->cu, cs, h->api_s, h->d_kx, h->d_kz, h->d_dyf, h->d_gyf, h->st);
        if (e == cudaSuccess)
            e = launch_zinv<double>(d, h->api_s, h->s_field, h->xb, h->x_field, 1, 1, d.ny, h->pz, h->twz_d, h->st);
        if (e == cudaSuccess) e = launch_xinv(d, h->xb, F, 1, d.ny, h->pm, h->twm_d, h->twn_d, h->st);
        h->launches += 3;
        return e;
    };
    auto term = [&](int mode, const double* f, const double* u, const double* m, const double* m2, int jlo, int jhi,
                    int slot, int init) -> cudaError_t {
        h->launches += 1;
        return launch_plane_terms(d, mode, f, u, m, m2, h->d_dy, h->d_dyf, rg, jlo, jhi, acc + (size_t)slot * nyp,
                                  init, h->st);
    };
    // rms vorticity, planes 1..NY
    for (int c = 0; c < 3; ++c) {
        CK(field(c, nullptr));
        CK(term(0, F, nullptr, nullptr, nullptr, 1, d.ny, c, 1));
    }
    // pseudo-dissipation, planes 2..NY-1, in tkebudget_chan's order of terms
    const int e0 = 2, e1 = d.ny - 1;
    CK(field(3, nullptr)); CK(term(1, F, nullptr, nullptr, nullptr, e0, e1, 3, 1));     // du/dx
    CK(field(4, nullptr)); CK(term(0, F, nullptr, nullptr, nullptr, e0, e1, 3, 0));     // dv/dx
    CK(term(2, nullptr, U1, ume, nullptr, e0, e1, 3, 0));                               // du/dy
    CK(field(5, nullptr)); CK(term(1, F, nullptr, nullptr, nullptr, e0, e1, 3, 0));     // dw/dx
    CK(field(6, nullptr)); CK(term(1, F, nullptr, nullptr, nullptr, e0, e1, 3, 0));     // du/dz
    CK(term(3, nullptr, U2, vme, nullptr, e0, e1, 3, 0));                               // dv/dy
    CK(term(2, nullptr, U3, wme, nullptr, e0, e1, 3, 0));                               // dw/dy
    CK(field(7, nullptr)); CK(term(0, F, nullptr, nullptr, nullptr, e0, e1, 3, 0));     // dv/dz
    CK(field(8, nullptr)); CK(term(1, F, nullptr, nullptr, nullptr, e0, e1, 3, 0));     // dw/dz
    // scalars: TH - THME, its flux with V, and |grad TH|^2
    std::vector<double> thme((size_t)d.nth * nyp);
    for (int n = 0; n < d.nth; ++n) {
        const double2* cs = h->cu + (size_t)(3 + n) * h->s_field;
        std::vector<double2> c00(nyp);
        CK(cudaMemcpy2DAsync(c00.data(), sizeof(double2), cs, sizeof(double2) * h->s_plane, sizeof(double2), nyp,
                             cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
        for (size_t j = 0; j < nyp; ++j) thme[(size_t)n * nyp + j] = c00[j].x;
        CK(cudaMemcpyAsync(thm, thme.data() + (size_t)n * nyp, sizeof(double) * nyp, cudaMemcpyHostToDevice, h->st));
        CK(launch_zinv<double>(d, cs, h->s_field, h->xb, h->x_field, 1, 0, d.nyp, h->pz, h->twz_d, h->st));
        CK(launch_xinv(d, h->xb, F, 0, d.nyp, h->pm, h->twm_d, h->twn_d, h->st));
        h->launches += 2;
        const int s0 = 4 + 3 * n;
        CK(term(4, F, nullptr, thm, nullptr, 1, d.ny, s0, 1));
        CK(term(5, F, U2, thm, vme, 1, d.ny, s0 + 1, 1));
        for (int k = 0; k < 3; ++k) {
            CK(field(9 + k, cs));
            CK(term(0, F, nullptr, nullptr, nullptr, 1, d.ny, s0 + 2, k == 0));
        }
    }
    std::vector<double> sums((size_t)nsum * nyp);
    CK(cudaMemcpyAsync(sums.data(), acc, sizeof(double) * sums.size(), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    auto S = [&](int k, int j) { return sums[(size_t)k * nyp + j]; };
    for (size_t q = 0; q < (size_t)DIABLO_NMEAN * nyp; ++q) chan[q] = 0.0;
    for (int s = 0; s < DIABLO_STAT_THME; ++s)
        for (size_t j = 0; j < nyp; ++j) chan[(size_t)s * nyp + j] = base[(size_t)s * nyp + j];
    const double nxz = (double)d.nx * (double)d.nz;       // DBLE(NX)*DBLE(NZ)
    const double nxzi = (double)(d.nx * d.nz);            // DBLE(NX*NZ)
    const double nn = (double)((float)d.nz * (float)d.nx);  // FLOAT(NZ)*FLOAT(NX)
    for (int c = 0; c < 3; ++c)
        for (int j = 1; j <= d.ny; ++j) chan[(size_t)(DIABLO_MEAN_OMEGA_X + c) * nyp + j] = std::sqrt(S(c, j) / nxz);
    if (epsilon) {
        for (size_t j = 0; j < nyp; ++j) epsilon[j] = 0.0;
        for (int j = e0; j <= e1; ++j) epsilon[j] = h->p.nu * S(3, j) / nxzi;
    }
    for (int n = 0; n < d.nth; ++n) {
        double* o = scal + (size_t)n * DIABLO_NSCAL * nyp;
        const double* tm = thme.data() + (size_t)n * nyp;
        for (size_t q = 0; q < (size_t)DIABLO_NSCAL * nyp; ++q) o[q] = 0.0;
        for (size_t j = 0; j < nyp; ++j) o[DIABLO_SCAL_THME * nyp + j] = tm[j];
        for (int j = 1; j <= d.ny; ++j) {
            o[DIABLO_SCAL_DTHDY * nyp + j] = (tm[j] - tm[j - 1]) / (h->gyf[j] - h->gyf[j - 1]);
            o[DIABLO_SCAL_THRMS * nyp + j] = std::sqrt(S(4 + 3 * n, j) / nn);
            o[DIABLO_SCAL_THV * nyp + j] = S(5 + 3 * n, j) / nn;
            o[DIABLO_SCAL_PE_DISS * nyp + j] = S(6 + 3 * n, j) / nxzi;
        }
    }
    return DIABLO_OK;
}

int diablo_gpu_filter_chan(void* handle, int n) {
    Handle* h = (Handle*)handle;
    if (!h) return fail(DIABLO_EINVAL, "null handle");
    if (n < 1 || n > h->d.nth) return fail(DIABLO_EINVAL, "scalar index outside 1..N_TH");
    { ProfScope ps(h, DIABLO_KERNEL_OTHER);
      CK(launch_filter_chan(h->d, h->cu + (size_t)(3 + n - 1) * h->s_field, h->d_kx, h->d_kz, h->p.lx, h->p.lz,
                            (double)(float)h->p.nx, (double)(float)h->p.nz, h->st)); }
    h->launches += 1;
    CK(cudaStreamSynchronize(h->st));
    return DIABLO_OK;
}

int diablo_gpu_synchronize(void* handle) {
    Handle* h = (Handle*)handle;
    if (!h) return fail(DIABLO_EINVAL, "null handle");
    CK(cudaStreamSynchronize(h->st));
    return take_nan(h);
}

int diablo_gpu_get_stream(void* handle, void** stream) {
    Handle* h = (Handle*)handle;
    if (!h || !stream) return fail(DIABLO_EINVAL, "null pointer argument");
    *stream = (void*)h->st;
    return DIABLO_OK;
}

static void drop_records(Handle* h) {
    for (auto& r : h->recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    h->recs.clear();
}

int diablo_gpu_set_profiling(void* handle, int on) {
    Handle* h = (Handle*)handle;
    if (!h) return fail(DIABLO_EINVAL, "null handle");
    CK(cudaStreamSynchronize(h->st));
    drop_records(h);
    h->profiling = on != 0;
    return DIABLO_OK;
}

int diablo_gpu_kernel_times(void* handle, long long* launches, double* ms) {
    Handle* h = (Handle*)handle;
    if (!h || !launches || !ms) return fail(DIABLO_EINVAL, "null pointer argument");
    CK(cudaStreamSynchronize(h->st));
    for (int k = 0; k < DIABLO_NKERNELS; ++k) { launches[k] = 0; ms[k] = 0.0; }
    for (auto& r : h->recs) {
        float t = 0.f;
        if (cudaEventElapsedTime(&t, r.a, r.b) == cudaSuccess && r.kind >= 0 && r.kind < DIABLO_NKERNELS) {
            launches[r.kind] += 1;
            ms[r.kind] += t;
        }
    }
    drop_records(h);
    return DIABLO_OK;
}

int diablo_gpu_autotune(void* handle, int* prod_chunk, int* zf_planes) {
    Handle* h = (Handle*)handle;
    if (!h) return fail(DIABLO_EINVAL, "null handle");
    if (h->profiling) return fail(DIABLO_EINVAL, "autotune with profiling on");
    const Dims& d = h->d;
    const size_t sb = sizeof(double2) * h->s_field;
    double2* save = nullptr;
    CK(cudaStreamSynchronize(h->st));
    cudaError_t e = cudaMalloc((void**)&save, sb * (2 * (size_t)d.nf + 1));
    if (e != cudaSuccess) return fail(DIABLO_ENOMEM, "autotune: state copy allocation failed");
    auto copy_state = [&](bool restore) -> cudaError_t {
        const cudaMemcpyKind k = cudaMemcpyDeviceToDevice;
        cudaError_t r = restore ? cudaMemcpyAsync(h->cu, save, sb * d.nf, k, h->st)
                                : cudaMemcpyAsync(save, h->cu, sb * d.nf, k, h->st);
        if (r == cudaSuccess)
            r = restore ? cudaMemcpyAsync(h->cf, save + h->s_field * d.nf, sb * d.nf, k, h->st)
                        : cudaMemcpyAsync(save + h->s_field * d.nf, h->cf, sb * d.nf, k, h->st);
        if (r == cudaSuccess)
            r = restore ? cudaMemcpyAsync(h->cp, save + 2 * h->s_field * d.nf, sb, k, h->st)
                        : cudaMemcpyAsync(save + 2 * h->s_field * d.nf, h->cp, sb, k, h->st);
        return r;
    };
    cudaEvent_t ea = nullptr, eb = nullptr;
    int rc = DIABLO_OK;
    double dt = 1e-6;
    double hb[3] = {dt * 8.0 / 15.0, dt * 2.0 / 15.0, dt * 5.0 / 15.0};
    const double bb[3] = {1.0, 25.0 / 8.0, 9.0 / 4.0}, zb[3] = {0.0, -17.0 / 8.0, -5.0 / 4.0};
    // time of one substage (rk_step 2) with the current shapes: best of 3
    auto time_one = [&](float* best) -> int {
        *best = 1e30f;
        for (int rep = 0; rep < 4; ++rep) {
            if ((e = copy_state(true)) != cudaSuccess) return fail(DIABLO_ECUDA, "autotune: restore");
            cudaEventRecord(ea, h->st);
            int r = diablo_gpu_rk_chan_1(h, 2, 1, 0.0, &dt, hb, bb, zb);
            if (r) return r;
            cudaEventRecord(eb, h->st);
            if ((e = cudaEventSynchronize(eb)) != cudaSuccess) return fail(DIABLO_ECUDA, "autotune: sync");
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ea, eb);
            if (rep > 0 && ms < *best) *best = ms;     // the first run warms up
        }
        return DIABLO_OK;
    };
    e = cudaEventCreate(&ea);
    if (e == cudaSuccess) e = cudaEventCreate(&eb);
    if (e == cudaSuccess) e = copy_state(false);
    if (e != cudaSuccess) rc = fail(DIABLO_ECUDA, std::string("autotune: ") + cudaGetErrorString(e));
    if (!rc) {
        // coordinate search: products chunk, then z-forward planes per block
        const int chunks[] = {4, 8, 16, 32, 64}, planes[] = {4, 8, 16};
        float best = 1e30f;
        int bc = h->prod_chunk, bz = h->zf_planes;
        for (int c : chunks) {
            h->prod_chunk = c;
            float t;
            if ((rc = time_one(&t))) break;
            if (t < best) { best = t; bc = c; }
        }
        h->prod_chunk = bc;
        if (!rc) {
            best = 1e30f;
            for (int z : planes) {
                h->zf_planes = z;
                float t;
                if ((rc = time_one(&t))) break;
                if (t < best) { best = t; bz = z; }
            }
            h->zf_planes = bz;
        }
    }
    if (!rc && (e = copy_state(true)) != cudaSuccess) rc = fail(DIABLO_ECUDA, "autotune: restore");
    cudaStreamSynchronize(h->st);
    if (ea) cudaEventDestroy(ea);
    if (eb) cudaEventDestroy(eb);
    cudaFree(save);
    if (rc) return rc;
    if (prod_chunk) *prod_chunk = h->prod_chunk;
    if (zf_planes) *zf_planes = h->zf_planes;
    return DIABLO_OK;
}

}  // extern "C"

namespace {
// Instances of equal shape and precision advance together: each kernel of the
// substage is one launch over the whole group, reading every instance's
// arrays and parameters from device tables (InstPtrs, ColJob).
struct BatchGroup {
    std::vector<Handle*> hs;
    std::vector<double> temp1;            // [n][3] TEMP1 of each instance's substages
    std::vector<double> dt;               // [n] each instance's time step
    InstPtrs* d_ip = nullptr;             // [n]
    ColJob* d_col = nullptr;              // [3][n], one set per RK substage
    int jlo_min = 0;
    cudaStream_t st = nullptr;            // the group's branch of the graph
    cudaEvent_t join = nullptr;
};

struct Batch {
    std::vector<Handle*> hs;
    std::vector<BatchGroup> groups;
    cudaStream_t origin = nullptr;
    cudaEvent_t fork = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

void free_batch(Batch* b) {
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (BatchGroup& g : b->groups) {
        if (g.d_ip) cudaFree(g.d_ip);
        if (g.d_col) cudaFree(g.d_col);
        if (g.join) cudaEventDestroy(g.join);
        if (g.st) cudaStreamDestroy(g.st);
    }
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->origin) cudaStreamDestroy(b->origin);
    delete b;
}

// One RK3 step of a group on its stream: per substage the four kernels of the
// Fourier-space path (channel.f:62-1073 without COURANT), each once for all
// instances.  The CN factors of the batch's fixed time steps are built when
// the batch is made (ensure_cn_tables) and checked before every launch.
template <typename T>
cudaError_t batch_group_step(BatchGroup& g) {
    Handle* h0 = g.hs[0];
    const Dims& d = h0->d;
    const int n = (int)g.hs.size();
    const bool f = std::is_same<T, float>::value;
    const void* twn = f ? h0->twn_f : h0->twn_d;
    const void* twm = f ? h0->twm_f : h0->twm_d;
    const void* twz = f ? h0->twz_f : h0->twz_d;
    // The groups of a batch fill the GPU together, so the block-wide products
    // kernel takes chunks of at least 32 planes: a chunk tuned for one
    // instance's latency recomputes more halo planes than a batch can spare.
    const int bchunk = h0->prod_chunk > 32 ? h0->prod_chunk : 32;
    cudaError_t e = cudaSuccess;
    for (int r = 0; r < 3 && e == cudaSuccess; ++r) {
        e = launch_zinv_b<T>(d, g.d_ip, n, h0->s_field, h0->x_field, h0->pz, twz, g.st, f ? 1 : 0);
        if (e != cudaSuccess) break;
        if (f && products_hw_supported(d))
            e = launch_products_hw_b(d, g.d_ip, n, g.jlo_min, d.ny, h0->prod_chunk, twm, twn, g.st, h0->s_field);
        else
            e = launch_products_b<T>(d, g.d_ip, n, g.jlo_min, d.ny, bchunk, h0->pm, twm, twn, g.st, f ? 1 : 0,
                                     h0->s_field);
        if (e == cudaSuccess) e = launch_zfwd_nl_b<T>(d, g.d_ip, n, g.jlo_min, d.ny, h0->zf_planes, h0->pz, twz, g.st);
        if (e == cudaSuccess) e = launch_colpart_b<cpx<T>>(d, g.d_col + (size_t)r * n, n, h0->pb, g.st);
    }
    return e;
}
}  // namespace

extern "C" {

int diablo_gpu_batch_create(void* const* handles, const double* delta_t, int n, void** batch) {
    if (!handles || !delta_t || !batch || n < 1) return fail(DIABLO_EINVAL, "bad batch arguments");
    *batch = nullptr;
    for (int i = 0; i < n; ++i) {
        Handle* h = (Handle*)handles[i];
        if (!h) return fail(DIABLO_EINVAL, "null handle in batch");
        if (h->p.variable_dt) return fail(DIABLO_ENOTSUP, "batched instances need a fixed time step (variable_dt = 0)");
        if (h->p.f_type == 2) return fail(DIABLO_ENOTSUP, "batched instances cannot have time-dependent forcing");
        if (h->p.les) return fail(DIABLO_ENOTSUP, "batched instances cannot run the LES branch");
        if (h->urhs_fn[0] || h->urhs_fn[1]) return fail(DIABLO_ENOTSUP, "batched instances cannot have user right-hand sides");
        if (h->profiling) return fail(DIABLO_EINVAL, "batched instance with profiling on");
        if (!(delta_t[i] > 0.0)) return fail(DIABLO_EINVAL, "batched instance with delta_t <= 0");
        for (int k = 0; k < i; ++k)
            if (handles[k] == handles[i]) return fail(DIABLO_EINVAL, "an instance appears twice in the batch");
    }
    Batch* b = new Batch();
    auto bail = [&](int code, const std::string& msg) { free_batch(b); return fail(code, msg); };
    // groups of equal shape, number of scalars and precision, in first-seen order
    std::vector<double> dts;
    for (int i = 0; i < n; ++i) {
        Handle* h = (Handle*)handles[i];
        b->hs.push_back(h);
        BatchGroup* g = nullptr;
        for (BatchGroup& q : b->groups) {
            const Handle* r = q.hs[0];
            if (r->d.nx == h->d.nx && r->d.ny == h->d.ny && r->d.nz == h->d.nz && r->d.nth == h->d.nth &&
                r->fp32 == h->fp32)
                g = &q;
        }
        if (!g) { b->groups.emplace_back(); g = &b->groups.back(); }
        g->hs.push_back(h);
    }
    cudaError_t e = cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    for (int i = 0; i < n && e == cudaSuccess; ++i) e = cudaStreamSynchronize(b->hs[i]->st);
    const double bb[3] = {1.0, 25.0 / 8.0, 9.0 / 4.0}, zb[3] = {0.0, -17.0 / 8.0, -5.0 / 4.0};
    for (BatchGroup& g : b->groups) {
        if (e != cudaSuccess) break;
        const int m = (int)g.hs.size();
        std::vector<InstPtrs> ip(m);
        std::vector<ColJob> col(3 * (size_t)m);
        g.temp1.assign(3 * (size_t)m, 0.0);
        g.dt.assign(m, 0.0);
        g.jlo_min = g.hs[0]->jlo_prod;
        for (int i = 0; i < m; ++i) {
            Handle* h = g.hs[i];
            ip[i] = InstPtrs{h->cu, h->xb, h->yb, h->nl, h->d_dy, h->d_dyf, h->d_kx, h->d_kz, h->jlo_prod};
            if (h->jlo_prod < g.jlo_min) g.jlo_min = h->jlo_prod;
            double dt = 0.0;
            for (int k = 0; k < n; ++k)
                if (handles[k] == h) dt = delta_t[k];
            g.dt[i] = dt;
            const double hb[3] = {dt * 8.0 / 15.0, dt * 2.0 / 15.0, dt * 5.0 / 15.0};
            for (int r = 0; r < 3; ++r) {
                CnArgs a = substage_args(h, r + 1, 0.0, hb, bb, zb);
                const double* tabs = nullptr;
                const int rc = ensure_cn_tables(h, a, r, &tabs);
                if (rc) { free_batch(b); return rc; }
                g.temp1[(size_t)i * 3 + r] = a.temp1;
                col[(size_t)r * m + i] = ColJob{dns_col_args(h, a, false), h->nl, tabs};
            }
            if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
        }
        if (e == cudaSuccess) e = cudaMalloc((void**)&g.d_ip, sizeof(InstPtrs) * m);
        if (e == cudaSuccess) e = cudaMalloc((void**)&g.d_col, sizeof(ColJob) * col.size());
        // ordered on the batch's stream and waited for below, before any graph launch reads them
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(g.d_ip, ip.data(), sizeof(InstPtrs) * m, cudaMemcpyHostToDevice, b->origin);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(g.d_col, col.data(), sizeof(ColJob) * col.size(), cudaMemcpyHostToDevice, b->origin);
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->origin);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g.st, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g.join, cudaEventDisableTiming);
    }
    if (e != cudaSuccess)
        return bail(e == cudaErrorMemoryAllocation ? DIABLO_ENOMEM : DIABLO_ECUDA,
                    std::string("batch set-up: ") + cudaGetErrorString(e));
    e = cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) return bail(DIABLO_ECUDA, std::string("batch capture: ") + cudaGetErrorString(e));
    e = cudaEventRecord(b->fork, b->origin);
    for (BatchGroup& g : b->groups) {
        if (e == cudaSuccess) e = cudaStreamWaitEvent(g.st, b->fork, 0);
        if (e == cudaSuccess) e = g.hs[0]->fp32 ? batch_group_step<float>(g) : batch_group_step<double>(g);
        if (e == cudaSuccess) e = cudaEventRecord(g.join, g.st);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b->origin, g.join, 0);
    }
    cudaError_t ee = cudaStreamEndCapture(b->origin, &b->graph);
    if (e != cudaSuccess) return bail(DIABLO_ECUDA, std::string("batch capture: ") + cudaGetErrorString(e));
    if (ee != cudaSuccess) return bail(DIABLO_ECUDA, std::string("batch end capture: ") + cudaGetErrorString(ee));
    e = cudaGraphInstantiate(&b->exec, b->graph, 0);
    if (e != cudaSuccess) return bail(DIABLO_ECUDA, std::string("batch instantiate: ") + cudaGetErrorString(e));
    *batch = b;
    return DIABLO_OK;
}

int diablo_gpu_batch_step(void* batch, int nsteps) {
    Batch* b = (Batch*)batch;
    if (!b || nsteps < 0) return fail(DIABLO_EINVAL, "bad batch arguments");
    // An instance stepped on its own with another time step since the last
    // batch step holds other CN factors: rebuild those of the batch's time step.
    const double bb[3] = {1.0, 25.0 / 8.0, 9.0 / 4.0}, zb[3] = {0.0, -17.0 / 8.0, -5.0 / 4.0};
    for (BatchGroup& g : b->groups)
        for (size_t i = 0; i < g.hs.size(); ++i) {
            Handle* h = g.hs[i];
            bool stale = false;
            for (int r = 0; r < 3; ++r) stale = stale || !h->tab_ok[r] || h->tab_temp1[r] != g.temp1[i * 3 + r];
            if (!stale) continue;
            const double dt = g.dt[i];
            const double hb[3] = {dt * 8.0 / 15.0, dt * 2.0 / 15.0, dt * 5.0 / 15.0};
            for (int r = 0; r < 3; ++r) {
                CnArgs a = substage_args(h, r + 1, 0.0, hb, bb, zb);
                const double* tabs = nullptr;
                int rc = ensure_cn_tables(h, a, r, &tabs);
                if (rc) return rc;
            }
            CK(cudaStreamSynchronize(h->st));
        }
    for (int s = 0; s < nsteps; ++s) CK(cudaGraphLaunch(b->exec, b->origin));
    CK(cudaStreamSynchronize(b->origin));
    return DIABLO_OK;
}

int diablo_gpu_batch_destroy(void* batch) {
    Batch* b = (Batch*)batch;
    if (!b) return fail(DIABLO_EINVAL, "null batch");
    cudaStreamSynchronize(b->origin);
    free_batch(b);
    return DIABLO_OK;
}

long long diablo_gpu_kernel_launches(void* handle) {
    Handle* h = (Handle*)handle;
    return h ? h->launches : -1;
}

}  // extern "C"
