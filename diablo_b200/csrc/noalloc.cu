// noalloc.cu -- REM_DIV_CHAN on caller-owned device arrays, allocating
// nothing.
//
// Who needs it: a host that keeps its fields in device memory it obtained
// itself -- a Fortran code with OpenACC or CUDA Fortran device arrays, a
// framework that hands out memory from its own pool -- and therefore cannot
// let a library call cudaMalloc (the allocation would bypass the runtime or
// pool that owns the device memory).  This entry point only queues two small
// copies of the grid metrics and one kernel on the caller's stream; its
// working storage is the file-scope array below, which is created when the
// library is loaded and held by every GPU that loads it until the process
// exits.
//
// Limits and sharing: the array holds 2^20 doubles (8 MiB).  A call needs
// 2*(NY+2) doubles for the grid metrics plus one double per retained mode and
// plane, (NX/3+1)*(2*(NZ/3)+1)*(NY+2); larger grids are rejected with
// DIABLO_EINVAL.  Every call uses the same array: calls that can overlap on
// the GPU (different streams, or different host threads) race on it and must
// be serialised by the caller.  Nothing in it has to start at zero: each call
// writes every entry it reads.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/diablo_gpu.h"
#include "launch.h"

namespace {

constexpr size_t kScratchDoubles = size_t(1) << 20;
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];


// Device address of g_noalloc_scratch, looked up once per device (with that
// device current) on the first call made on that device.
constexpr int kMaxDevices = 64;
double* g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

int scratch_for_current_device(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        return dgpu::set_error(DIABLO_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    }
    if (dev < 0 || dev >= kMaxDevices) {
        return dgpu::set_error(DIABLO_EINVAL, "device ordinal out of range");
    }
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            return dgpu::set_error(DIABLO_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        }
        g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_ptr[dev];
    return DIABLO_OK;
}

// One pair of lanes per retained (kx,kz) mode: lane 0 the real, lane 1 the
// imaginary part of the phi system (its coefficients are real).  Same rows,
// boundary rows and guarded elimination as REM_DIV_CHAN with
// APPLY_BC_REM_DIV_MPI and the complex MPI Thomas (channel.f:1103-1214,
// mpi.f:700-865, 1239-1278).  Arrays: Fortran layout (0:NXP,0:NZ+1,0:NY+1)
// complex, interleaved.  phi receives phi on J = 1..NY (and holds the
// eliminated right-hand sides in between).
__global__ void k_rem_div_fortran(int nkx, int nkz, int tnkz, int nxp, int nz, int ny, double lx, double lz,
                                  double* cu1, double* cu2, double* cu3, double* phi,
                                  const double* __restrict__ dy, const double* __restrict__ dyf,
                                  double* __restrict__ piv) {
    const int part = threadIdx.x & 1;
    const int nkxp = nkx + 1, nkzt = tnkz + 1;
    const int ncol = nkxp * nkzt;
    const int g = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 1);
    const bool active = g < ncol;
    const int gg = active ? g : ncol - 1;
    const int i = gg % nkxp, m = gg / nkxp;
    const double twopi = 2.0 * 3.14159265358979323846;
    const double KX = (double)i * twopi / lx;
    const double KZ = (m <= nkz) ? (double)m * twopi / lz : -(double)(tnkz + 1 - m) * twopi / lz;
    const bool zero_mode = (i == 0 && m == 0);
    const double sgn = part ? 1.0 : -1.0;    // part of (i K v): re -> -K v.im, im -> +K v.re
    const size_t cx = (size_t)nxp + 1, cz = (size_t)nz + 2;
    auto at = [&](int j) { return 2 * ((size_t)i + cx * ((size_t)m + cz * (size_t)j)); };
    // forward elimination: row 1 is the BC row, rows 2..NY (row NY a BC row)
    double bprev = 1.0, cprev = zero_mode ? 0.0 : -1.0, gprev = 0.0;
    if (active) {
        if (part == 0) piv[(size_t)1 * ncol + g] = bprev;
        phi[at(1) + part] = gprev;
    }
    for (int j = 2; j <= ny; ++j) {
        double A, B, C, G = 0.0;
        if (j < ny) {
            A = 1. / (dy[j] * dyf[j]);
            B = -KX * KX - KZ * KZ - 1. / (dy[j + 1] * dyf[j]) - 1. / (dy[j] * dyf[j]);
            C = 1. / (dy[j + 1] * dyf[j]);
            if (active) {
                const double u1o = cu1[at(j) + (part ^ 1)], u3o = cu3[at(j) + (part ^ 1)];
                const double u2p = cu2[at(j + 1) + part], u2j = cu2[at(j) + part];
                G = sgn * KX * u1o + (u2p - u2j) / dyf[j] + sgn * KZ * u3o;
            }
        } else {
            A = 1.; B = -1.; C = 0.;
        }
        const double Ap = (bprev != 0.0) ? -A / bprev : 0.0;
        B = B + Ap * cprev;
        G = G + Ap * gprev;
        if (active) {
            if (part == 0) piv[(size_t)j * ncol + g] = B;
            phi[at(j) + part] = G;
        }
        bprev = B;
        cprev = C;
        gprev = G;
    }
    __syncwarp();
    // back substitution, then the velocity correction (channel.f:1196-1211)
    double xn = 0.0;
    for (int j = ny; j >= 1; --j) {
        const double B = active ? piv[(size_t)j * ncol + g] : 1.0;
        const double G = active ? phi[at(j) + part] : 0.0;
        double x;
        if (j == ny) x = (B != 0.0) ? G / B : 0.0;
        else {
            const double C = (j == 1) ? (zero_mode ? 0.0 : -1.0) : 1. / (dy[j + 1] * dyf[j]);
            x = (B != 0.0) ? (G - C * xn) / B : 0.0;
        }
        const double xo = __shfl_xor_sync(0xffffffffu, x, 1);
        if (active) {
            phi[at(j) + part] = x;
            cu1[at(j) + part] -= sgn * KX * xo;
            cu3[at(j) + part] -= sgn * KZ * xo;
            if (j + 1 <= ny) cu2[at(j + 1) + part] -= (xn - x) / dy[j + 1];
        }
        xn = x;
    }
}

}  // namespace

extern "C" {

int diablo_gpu_rem_div_chan_noalloc(const diablo_params* p, const double* dy, const double* dyf, double* cu1,
                                    double* cu2, double* cu3, double* phi, void* stream) {
    if (!p || !dy || !dyf || !cu1 || !cu2 || !cu3 || !phi) {
        return dgpu::set_error(DIABLO_EINVAL, "null pointer argument");
    }
    if (p->nx < 8 || p->nz < 8 || p->ny < 4 || p->nx % 2 || p->lx <= 0.0 || p->lz <= 0.0) {
        return dgpu::set_error(DIABLO_EINVAL, "bad dimensions");
    }
    const int nkx = p->nx / 3, nkz = p->nz / 3, tnkz = 2 * nkz, nxp = p->nx / 2, nyp = p->ny + 2;
    const size_t ncol = (size_t)(nkx + 1) * (tnkz + 1);
    const size_t need = 2 * (size_t)nyp + ncol * (size_t)nyp;
    if (need > kScratchDoubles) {
        char msg[256];
        std::snprintf(msg, sizeof(msg),
                      "grid too large for the no-allocation REM_DIV_CHAN: needs %zu doubles of scratch, "
                      "the static array holds %zu ((NX/3+1)*(2*(NZ/3)+1)*(NY+2) + 2*(NY+2) must fit)",
                      need, kScratchDoubles);
        return dgpu::set_error(DIABLO_EINVAL, msg);
    }
    double* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // grid metrics into the front of the scratch array (host -> device copy,
    // no allocation)
    cudaError_t e = cudaMemcpyAsync(scratch, dy, sizeof(double) * nyp, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(scratch + nyp, dyf, sizeof(double) * nyp, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) {
        return dgpu::set_error(DIABLO_ECUDA, std::string("cudaMemcpyAsync: ") + cudaGetErrorString(e));
    }
    const int threads = 128;
    const unsigned blocks = (unsigned)((2 * ncol + threads - 1) / threads);
    k_rem_div_fortran<<<blocks, threads, 0, st>>>(nkx, nkz, tnkz, nxp, p->nz, p->ny, p->lx, p->lz, cu1, cu2, cu3,
                                                  phi, scratch, scratch + nyp, scratch + 2 * nyp);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        return dgpu::set_error(DIABLO_ECUDA, std::string("k_rem_div_fortran: ") + cudaGetErrorString(e));
    }
    return DIABLO_OK;
}

}  // extern "C"
