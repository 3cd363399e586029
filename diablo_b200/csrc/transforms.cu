// transforms.cu -- x/z transform kernels of the channel timestep (sm_100a).
//
// The reference transforms one y-plane at a time with FFTW and an MPI
// all-to-all between the x and z stages (FFT_XZ_TO_FOURIER / _PHYSICAL,
// for/mpi.f:1477-1606).  Here the z stage and the x stage are separate
// kernels over all planes; the transpose between them is the X layout in
// device memory, and the physical-space products of RK_CHAN_1 never leave
// shared memory: one kernel per z-row goes from the x spectra of the state
// to the x spectra of the products.
#include <cuda_runtime.h>

#include "fft.cuh"
#include "kernels.cuh"
#include "launch.h"

namespace dgpu {

template <typename T>
__device__ __forceinline__ cpx<T> ld(const double2* p) {
    double2 v = *p;
    return mk<T>((T)v.x, (T)v.y);
}

// Packed kz index m in [0,TNKZ] -> full z index in [0,NZ) (mpi.f:1530-1539).
__device__ __forceinline__ int m_to_z(int m, int nkz, int nz, int nkzt) {
    return m <= nkz ? m : m + nz - nkzt;
}

// ---------------------------------------------------------------------------
// K1: spectral (FP64) -> x-spectrum (T); inverse z transform along columns.
// Block (kx tile of TX columns, plane J, field f); 256 threads.
// ---------------------------------------------------------------------------
template <typename T, int TX, int VMAX>
__global__ void __launch_bounds__(256) k_zinv(Dims d, const double2* __restrict__ S, size_t s_fstride,
                                              cpx<T>* __restrict__ X, size_t x_fstride, int j0,
                                              FftPlan pz, const cpx<T>* __restrict__ twz) {
    extern __shared__ unsigned char smem_raw[];
    cpx<T>* buf = reinterpret_cast<cpx<T>*>(smem_raw);   // [nz][TX]
    const int kx0 = blockIdx.x * TX;
    const int J = j0 + blockIdx.y;
    const int f = blockIdx.z;
    const int nz = d.nz;
    const double2* src = S + (size_t)f * s_fstride + (size_t)J * d.nkzt * d.ldx;
    for (int e = threadIdx.x; e < nz * TX; e += blockDim.x) {
        const int z = e / TX, c = e % TX;
        const int kx = kx0 + c;
        int m = -1;
        if (z <= d.nkz) m = z;
        else if (z >= nz - d.nkz) m = z - nz + d.nkzt;
        cpx<T> v = mk<T>(0, 0);
        if (m >= 0 && kx < d.nkxp) v = ld<T>(src + (size_t)m * d.ldx + kx);
        buf[e] = v;
    }
    __syncthreads();
    smem_fft<T, VMAX, false>(buf, TX, TX, 1, pz, twz, +1);
    cpx<T>* dst = X + (size_t)f * x_fstride + (size_t)J * nz * d.ldx;
    for (int e = threadIdx.x; e < nz * TX; e += blockDim.x) {
        const int z = e / TX, c = e % TX;
        dst[(size_t)z * d.ldx + kx0 + c] = buf[e];
    }
}

template <typename T>
struct ZTile;
template <>
struct ZTile<float> {
    static constexpr int TX = 16;
    static constexpr int VMAX = 32;
};
template <>
struct ZTile<double> {
    static constexpr int TX = 8;
    static constexpr int VMAX = 16;
};

template <typename T>
cudaError_t launch_zinv(const Dims& d, const double2* S, size_t s_fstride, void* X, size_t x_fstride,
                        int nfields, int j0, int nplanes, const FftPlan& pz, const void* twz,
                        cudaStream_t st) {
    constexpr int TX = ZTile<T>::TX;
    if (nplanes <= 0 || nfields <= 0) return cudaSuccess;
    const size_t smem = sizeof(cpx<T>) * (size_t)d.nz * TX;
    auto kern = k_zinv<T, TX, ZTile<T>::VMAX>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 grid(d.ldx / TX, nplanes, nfields);
    kern<<<grid, 256, smem, st>>>(d, S, s_fstride, (cpx<T>*)X, x_fstride, j0, pz,
                                  (const cpx<T>*)twz);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Two real sequences through one complex transform of length NX.
// ---------------------------------------------------------------------------
// Fill Z_k = A_k + i B_k (k in [0,NX)) from the half spectra a, b (kx <= NKX),
// with A_{NX-k} = conj(A_k); the imaginary part of the DC bin is dropped as
// FFTW's c2r does.  b may be null (B = 0).
template <typename T>
__device__ __forceinline__ void fill_pair_inverse(cpx<T>* z, const cpx<T>* __restrict__ a,
                                                  const cpx<T>* __restrict__ b, int nx, int nkx) {
    for (int k = threadIdx.x; k < nx; k += blockDim.x) {
        cpx<T> A = mk<T>(0, 0), B = mk<T>(0, 0);
        if (k <= nkx) {
            A = a[k];
            if (b) B = b[k];
            if (k == 0) { A.y = 0; B.y = 0; }
        } else if (k >= nx - nkx) {
            A = conjg(a[nx - k]);
            if (b) B = conjg(b[nx - k]);
        }
        z[k] = mk<T>(A.x - B.y, A.y + B.x);
    }
}

// From Z = FFT(a + i b) (a, b real) extract A_k, B_k for k < ldx, scaled,
// zero beyond NKX; write to rows ra, rb (rb may be null).
template <typename T>
__device__ __forceinline__ void extract_pair_forward(const cpx<T>* z, cpx<T>* __restrict__ ra,
                                                     cpx<T>* __restrict__ rb, int nx, int nkx,
                                                     int ldx, T scale) {
    for (int k = threadIdx.x; k < ldx; k += blockDim.x) {
        cpx<T> A = mk<T>(0, 0), B = mk<T>(0, 0);
        if (k <= nkx) {
            const cpx<T> zk = z[k];
            const cpx<T> zn = z[(nx - k) % nx];
            A = mk<T>((zk.x + zn.x) * T(0.5) * scale, (zk.y - zn.y) * T(0.5) * scale);
            B = mk<T>((zk.y + zn.y) * T(0.5) * scale, (zn.x - zk.x) * T(0.5) * scale);
        }
        ra[k] = A;
        if (rb) rb[k] = B;
    }
}

// ---------------------------------------------------------------------------
// K2: per z-row, marching over planes: x-inverse of the fields, physical
// products, x-forward of the products.
// ---------------------------------------------------------------------------
constexpr int PROD_VMAX = 12;   // pairs per group * NX <= 12 * 256

template <typename T>
__global__ void __launch_bounds__(256) k_products(Dims d, const cpx<T>* __restrict__ X,
                                                  cpx<T>* __restrict__ Y, int jlo, int jhi, int chunk,
                                                  int group, const double* __restrict__ dy,
                                                  const double* __restrict__ dyf, FftPlan px,
                                                  const cpx<T>* __restrict__ twx) {
    extern __shared__ unsigned char smem_raw[];
    const int nx = d.nx, nf = d.nf, np = d.np;
    T* ring = reinterpret_cast<T*>(smem_raw);                              // [3][nf][nx]
    cpx<T>* work = reinterpret_cast<cpx<T>*>(ring + (size_t)3 * nf * nx);  // [group][nx]
    const int z = blockIdx.x;
    const int jb = jlo + blockIdx.y * chunk;
    const int je = min(jb + chunk - 1, jhi);
    const size_t xrow = (size_t)d.nz * d.ldx;            // plane stride of X / Y
    const size_t xf = (size_t)d.nyp * xrow;              // field stride of X / Y
    const T inv_nx = T(1.0 / (double)nx);
    const int npair_in = (nf + 1) / 2;
    for (int J = jb - 1; J <= je + 1; ++J) {
        const int slot = (J - (jb - 1)) % 3;
        // --- backward x transform of the fields at plane J, row z ---------
        for (int q = 0; q < npair_in; ++q) {
            const int fa = 2 * q, fb = 2 * q + 1;
            const cpx<T>* a = X + (size_t)fa * xf + (size_t)J * xrow + (size_t)z * d.ldx;
            const cpx<T>* b = fb < nf ? X + (size_t)fb * xf + (size_t)J * xrow + (size_t)z * d.ldx : nullptr;
            fill_pair_inverse(work + (size_t)q * nx, a, b, nx, d.nkx);
        }
        __syncthreads();
        smem_fft<T, PROD_VMAX, true>(work, npair_in, 1, nx, px, twx, +1);
        for (int e = threadIdx.x; e < npair_in * nx; e += blockDim.x) {
            const int q = e / nx, x = e % nx;
            const cpx<T> v = work[e];
            ring[((size_t)slot * nf + 2 * q) * nx + x] = v.x;
            if (2 * q + 1 < nf) ring[((size_t)slot * nf + 2 * q + 1) * nx + x] = v.y;
        }
        __syncthreads();
        const int jp = J - 1;    // plane whose products are now computable
        if (jp < jb) continue;
        const int sm = (jp - 1 - (jb - 1)) % 3, s0 = (jp - (jb - 1)) % 3, sp = (J - (jb - 1)) % 3;
        const T a1 = (T)(dyf[jp] / (2.0 * dy[jp]));
        const T a0 = (T)(dyf[jp - 1] / (2.0 * dy[jp]));
        const T i2dyf = (T)(1.0 / (2.0 * dyf[jp]));
        const T idy = (T)(1.0 / dy[jp]);
        const T* U1m = ring + ((size_t)sm * nf + 0) * nx;
        const T* U1c = ring + ((size_t)s0 * nf + 0) * nx;
        const T* U1p = ring + ((size_t)sp * nf + 0) * nx;
        const T* U2m = ring + ((size_t)sm * nf + 1) * nx;
        const T* U2c = ring + ((size_t)s0 * nf + 1) * nx;
        const T* U2p = ring + ((size_t)sp * nf + 1) * nx;
        const T* U3m = ring + ((size_t)sm * nf + 2) * nx;
        const T* U3c = ring + ((size_t)s0 * nf + 2) * nx;
        const T* U3p = ring + ((size_t)sp * nf + 2) * nx;
        for (int g0 = 0; g0 < np; g0 += 2 * group) {
            const int ng = min(group, (np - g0 + 1) / 2);
            for (int e = threadIdx.x; e < ng * nx; e += blockDim.x) {
                const int q = e / nx, x = e % nx;
                T pv[2];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int p = g0 + 2 * q + h;
                    T v = 0;
                    const T u1 = U1c[x], u2 = U2c[x], u3 = U3c[x];
                    if (p == 0) v = u3 * u1;
                    else if (p == 1) v = u1 * u1;
                    else if (p == 2) v = u3 * u3;
                    else if (p == 3) v = (a1 * u1 + a0 * U1m[x]) * u2;
                    else if (p == 4) v = (a1 * u3 + a0 * U3m[x]) * u2;
                    else if (p == 5) v = (U1p[x] * U2p[x] + u1 * U2p[x] - u1 * u2 - U1m[x] * u2) * i2dyf;
                    else if (p == 6) v = (U3p[x] * U2p[x] + u3 * U2p[x] - u3 * u2 - U3m[x] * u2) * i2dyf;
                    else if (p == 7) {
                        const T s1 = u2 + U2p[x], s2 = u2 + U2m[x];
                        v = (T(0.25) * s1 * s1 - T(0.25) * s2 * s2) * idy;
                    } else if (p < np) {
                        const int n = (p - 8) / 3, r = (p - 8) % 3;
                        const T* THc = ring + ((size_t)s0 * nf + 3 + n) * nx;
                        if (r == 0) v = THc[x] * u1;
                        else if (r == 1) v = THc[x] * u3;
                        else {
                            const T* THm = ring + ((size_t)sm * nf + 3 + n) * nx;
                            const T* THp = ring + ((size_t)sp * nf + 3 + n) * nx;
                            v = (THp[x] * U2p[x] + THc[x] * U2p[x] - THc[x] * u2 - THm[x] * u2) * i2dyf;
                        }
                    }
                    pv[h] = v;
                }
                work[e] = mk<T>(pv[0], pv[1]);
            }
            __syncthreads();
            smem_fft<T, PROD_VMAX, true>(work, ng, 1, nx, px, twx, -1);
            for (int q = 0; q < ng; ++q) {
                const int pa = g0 + 2 * q, pb = pa + 1;
                cpx<T>* ra = Y + (size_t)pa * xf + (size_t)jp * xrow + (size_t)z * d.ldx;
                cpx<T>* rb = pb < np ? Y + (size_t)pb * xf + (size_t)jp * xrow + (size_t)z * d.ldx : nullptr;
                extract_pair_forward(work + (size_t)q * nx, ra, rb, nx, d.nkx, d.ldx, inv_nx);
            }
            __syncthreads();
        }
    }
}

template <typename T>
static int prod_group(int nx) {
    int g = (PROD_VMAX * 256) / nx;
    return g > 6 ? 6 : g;
}

template <typename T>
cudaError_t launch_products(const Dims& d, const void* X, void* Y, int jlo, int jhi, int chunk,
                            const double* dy, const double* dyf, const FftPlan& px, const void* twx,
                            cudaStream_t st) {
    if (jhi < jlo) return cudaSuccess;
    const int group = prod_group<T>(d.nx);
    const int npair_in = (d.nf + 1) / 2;
    if (group < 1 || npair_in > group) return cudaErrorInvalidValue;
    const size_t smem = sizeof(T) * (size_t)3 * d.nf * d.nx + sizeof(cpx<T>) * (size_t)group * d.nx;
    auto kern = k_products<T>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int nchunks = (jhi - jlo + chunk) / chunk;
    dim3 grid(d.nz, nchunks);
    kern<<<grid, 256, smem, st>>>(d, (const cpx<T>*)X, (cpx<T>*)Y, jlo, jhi, chunk, group, dy, dyf, px,
                                  (const cpx<T>*)twx);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// K3: per plane and kx tile: forward z transform of each product, kz
// packing with 1/NZ, derivative combination into the nonlinear terms.
// Product p -> field and multiplier (channel.f:410-571, 670-720):
//   0 U1U3: NL1 -= ikz, NL3 -= ikx     1 U1U1: NL1 -= ikx   2 U3U3: NL3 -= ikz
//   3 U1U2: NL2 -= ikx   4 U3U2: NL2 -= ikz   5,6,7 y-fluxes: NL1,NL3,NL2 -= 1
//   8+3n THU1: NLTH -= ikx   9+3n THU3: NLTH -= ikz   10+3n: NLTH -= 1
// ---------------------------------------------------------------------------
template <typename T, int TX, int VMAX>
__global__ void __launch_bounds__(256) k_zfwd_nl(Dims d, const cpx<T>* __restrict__ Y,
                                                 cpx<T>* __restrict__ NL, int jlo,
                                                 const double* __restrict__ kxw,
                                                 const double* __restrict__ kzw, FftPlan pz,
                                                 const cpx<T>* __restrict__ twz) {
    extern __shared__ unsigned char smem_raw[];
    const int nz = d.nz, nkzt = d.nkzt, nf = d.nf;
    cpx<T>* buf = reinterpret_cast<cpx<T>*>(smem_raw);          // [nz][TX]
    cpx<T>* acc = buf + (size_t)nz * TX;                         // [nf][nkzt][TX]
    const int kx0 = blockIdx.x * TX;
    const int J = jlo + blockIdx.y;
    const size_t xrow = (size_t)nz * d.ldx;
    const size_t xf = (size_t)d.nyp * xrow;
    const T inv_nz = T(1.0 / (double)nz);
    for (int e = threadIdx.x; e < nf * nkzt * TX; e += blockDim.x) acc[e] = mk<T>(0, 0);
    for (int p = 0; p < d.np; ++p) {
        const cpx<T>* src = Y + (size_t)p * xf + (size_t)J * xrow + kx0;
        for (int e = threadIdx.x; e < nz * TX; e += blockDim.x) {
            const int z = e / TX, c = e % TX;
            buf[e] = src[(size_t)z * d.ldx + c];
        }
        __syncthreads();
        smem_fft<T, VMAX, false>(buf, TX, TX, 1, pz, twz, -1);
        int fa, ma, fb = -1, mb = 0;   // target fields, multiplier 0: -1, 1: -ikx, 2: -ikz
        if (p == 0) { fa = 0; ma = 2; fb = 2; mb = 1; }
        else if (p == 1) { fa = 0; ma = 1; }
        else if (p == 2) { fa = 2; ma = 2; }
        else if (p == 3) { fa = 1; ma = 1; }
        else if (p == 4) { fa = 1; ma = 2; }
        else if (p == 5) { fa = 0; ma = 0; }
        else if (p == 6) { fa = 2; ma = 0; }
        else if (p == 7) { fa = 1; ma = 0; }
        else {
            const int n = (p - 8) / 3, r = (p - 8) % 3;
            fa = 3 + n;
            ma = r == 0 ? 1 : (r == 1 ? 2 : 0);
        }
        for (int e = threadIdx.x; e < nkzt * TX; e += blockDim.x) {
            const int m = e / TX, c = e % TX;
            const int zz = m_to_z(m, d.nkz, nz, nkzt);
            const cpx<T> v = buf[(size_t)zz * TX + c] * inv_nz;
            const T KX = (T)kxw[kx0 + c], KZ = (T)kzw[m];
            {
                cpx<T>& a = acc[((size_t)fa * nkzt + m) * TX + c];
                if (ma == 0) a = a - v;
                else { const T K = ma == 1 ? KX : KZ; a = mk<T>(a.x + K * v.y, a.y - K * v.x); }
            }
            if (fb >= 0) {
                cpx<T>& b = acc[((size_t)fb * nkzt + m) * TX + c];
                const T K = mb == 1 ? KX : KZ;
                b = mk<T>(b.x + K * v.y, b.y - K * v.x);
            }
        }
        __syncthreads();
    }
    const size_t sp = (size_t)nkzt * d.ldx;     // plane stride of S
    const size_t sf = (size_t)d.nyp * sp;       // field stride of S
    for (int e = threadIdx.x; e < nf * nkzt * TX; e += blockDim.x) {
        const int f = e / (nkzt * TX), r = e % (nkzt * TX);
        const int m = r / TX, c = r % TX;
        NL[(size_t)f * sf + (size_t)J * sp + (size_t)m * d.ldx + kx0 + c] = acc[e];
    }
}

template <typename T>
cudaError_t launch_zfwd_nl(const Dims& d, const void* Y, void* NL, int jlo, int jhi,
                           const double* kx, const double* kz, const FftPlan& pz, const void* twz,
                           cudaStream_t st) {
    constexpr int TX = ZTile<T>::TX;
    if (jhi < jlo) return cudaSuccess;
    const size_t smem = sizeof(cpx<T>) * ((size_t)d.nz * TX + (size_t)d.nf * d.nkzt * TX);
    auto kern = k_zfwd_nl<T, TX, ZTile<T>::VMAX>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 grid(d.ldx / TX, jhi - jlo + 1);
    kern<<<grid, 256, smem, st>>>(d, (const cpx<T>*)Y, (cpx<T>*)NL, jlo, kx, kz, pz,
                                  (const cpx<T>*)twz);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Transform-API helpers (FP64, one field).
// ---------------------------------------------------------------------------
// Rows r = (J - j0)*NZ + z; a block handles 2*group consecutive rows.
__global__ void __launch_bounds__(256) k_xinv(Dims d, const cpx<double>* __restrict__ X,
                                              double* __restrict__ P, int j0, int nrows, int group,
                                              FftPlan px, const cpx<double>* __restrict__ twx) {
    extern __shared__ unsigned char smem_raw[];
    cpx<double>* work = reinterpret_cast<cpx<double>*>(smem_raw);
    const int nx = d.nx;
    const int r0 = blockIdx.x * 2 * group;
    const int npair = min(group, (nrows - r0 + 1) / 2);
    for (int q = 0; q < npair; ++q) {
        const int ra = r0 + 2 * q, rb = ra + 1;
        const size_t ia = (size_t)j0 * d.nz + ra, ib = (size_t)j0 * d.nz + rb;
        fill_pair_inverse(work + (size_t)q * nx, X + ia * d.ldx, rb < nrows ? X + ib * d.ldx : nullptr,
                          nx, d.nkx);
    }
    __syncthreads();
    smem_fft<double, PROD_VMAX, true>(work, npair, 1, nx, px, twx, +1);
    for (int e = threadIdx.x; e < npair * nx; e += blockDim.x) {
        const int q = e / nx, x = e % nx;
        const int ra = r0 + 2 * q, rb = ra + 1;
        const cpx<double> v = work[e];
        P[((size_t)j0 * d.nz + ra) * nx + x] = v.x;
        if (rb < nrows) P[((size_t)j0 * d.nz + rb) * nx + x] = v.y;
    }
}

__global__ void __launch_bounds__(256) k_xfwd(Dims d, const double* __restrict__ P,
                                              cpx<double>* __restrict__ X, int j0, int nrows, int group,
                                              FftPlan px, const cpx<double>* __restrict__ twx) {
    extern __shared__ unsigned char smem_raw[];
    cpx<double>* work = reinterpret_cast<cpx<double>*>(smem_raw);
    const int nx = d.nx;
    const int r0 = blockIdx.x * 2 * group;
    const int npair = min(group, (nrows - r0 + 1) / 2);
    for (int e = threadIdx.x; e < npair * nx; e += blockDim.x) {
        const int q = e / nx, x = e % nx;
        const int ra = r0 + 2 * q, rb = ra + 1;
        const double a = P[((size_t)j0 * d.nz + ra) * nx + x];
        const double b = rb < nrows ? P[((size_t)j0 * d.nz + rb) * nx + x] : 0.0;
        work[e] = mk<double>(a, b);
    }
    __syncthreads();
    smem_fft<double, PROD_VMAX, true>(work, npair, 1, nx, px, twx, -1);
    for (int q = 0; q < npair; ++q) {
        const int ra = r0 + 2 * q, rb = ra + 1;
        extract_pair_forward(work + (size_t)q * nx, X + ((size_t)j0 * d.nz + ra) * d.ldx,
                             rb < nrows ? X + ((size_t)j0 * d.nz + rb) * d.ldx : nullptr, nx, d.nkx,
                             d.ldx, 1.0 / (double)nx);
    }
}

cudaError_t launch_xinv(const Dims& d, const void* X, double* P, int j0, int nplanes,
                        const FftPlan& px, const void* twx, cudaStream_t st) {
    const int group = prod_group<double>(d.nx);
    const int nrows = nplanes * d.nz;
    if (nrows <= 0) return cudaSuccess;
    const size_t smem = sizeof(cpx<double>) * (size_t)group * d.nx;
    cudaFuncSetAttribute(k_xinv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int nblk = (nrows + 2 * group - 1) / (2 * group);
    k_xinv<<<nblk, 256, smem, st>>>(d, (const cpx<double>*)X, P, j0, nrows, group, px,
                                    (const cpx<double>*)twx);
    return cudaGetLastError();
}

cudaError_t launch_xfwd(const Dims& d, const double* P, void* X, int j0, int nplanes,
                        const FftPlan& px, const void* twx, cudaStream_t st) {
    const int group = prod_group<double>(d.nx);
    const int nrows = nplanes * d.nz;
    if (nrows <= 0) return cudaSuccess;
    const size_t smem = sizeof(cpx<double>) * (size_t)group * d.nx;
    cudaFuncSetAttribute(k_xfwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int nblk = (nrows + 2 * group - 1) / (2 * group);
    k_xfwd<<<nblk, 256, smem, st>>>(d, P, (cpx<double>*)X, j0, nrows, group, px,
                                    (const cpx<double>*)twx);
    return cudaGetLastError();
}

template <int TX, int VMAX>
__global__ void __launch_bounds__(256) k_zfwd_pack(Dims d, const cpx<double>* __restrict__ X,
                                                   double2* __restrict__ S, int j0, FftPlan pz,
                                                   const cpx<double>* __restrict__ twz) {
    extern __shared__ unsigned char smem_raw[];
    cpx<double>* buf = reinterpret_cast<cpx<double>*>(smem_raw);
    const int kx0 = blockIdx.x * TX;
    const int J = j0 + blockIdx.y;
    const int nz = d.nz;
    const cpx<double>* src = X + (size_t)J * nz * d.ldx + kx0;
    for (int e = threadIdx.x; e < nz * TX; e += blockDim.x) {
        const int z = e / TX, c = e % TX;
        buf[e] = src[(size_t)z * d.ldx + c];
    }
    __syncthreads();
    smem_fft<double, VMAX, false>(buf, TX, TX, 1, pz, twz, -1);
    const double inv_nz = 1.0 / (double)nz;
    double2* dst = S + (size_t)J * d.nkzt * d.ldx + kx0;
    for (int e = threadIdx.x; e < d.nkzt * TX; e += blockDim.x) {
        const int m = e / TX, c = e % TX;
        const cpx<double> v = buf[(size_t)m_to_z(m, d.nkz, nz, d.nkzt) * TX + c];
        dst[(size_t)m * d.ldx + c] = make_double2(v.x * inv_nz, v.y * inv_nz);
    }
}

cudaError_t launch_zfwd_pack(const Dims& d, const void* X, double2* S, int j0, int nplanes,
                             const FftPlan& pz, const void* twz, cudaStream_t st) {
    constexpr int TX = ZTile<double>::TX;
    if (nplanes <= 0) return cudaSuccess;
    const size_t smem = sizeof(cpx<double>) * (size_t)d.nz * TX;
    auto kern = k_zfwd_pack<TX, ZTile<double>::VMAX>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 grid(d.ldx / TX, nplanes);
    kern<<<grid, 256, smem, st>>>(d, (const cpx<double>*)X, S, j0, pz, (const cpx<double>*)twz);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// CFL reduction (courant.f:35-47): one block per physical row (J, z), J in
// 1..NY; U1, U2, U3 through two complex transforms; FP64.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void atomic_min_pos(double* addr, double v) {
    // non-negative doubles (and +inf) order like their bit patterns
    atomicMin(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

__global__ void __launch_bounds__(256) k_cfl(Dims d, const cpx<double>* __restrict__ X, size_t x_fstride,
                                             FftPlan px, const cpx<double>* __restrict__ twx,
                                             const double* __restrict__ dy, double cfl, double dx,
                                             double dz, double* dtmin) {
    extern __shared__ unsigned char smem_raw[];
    cpx<double>* work = reinterpret_cast<cpx<double>*>(smem_raw);   // [2][nx]
    __shared__ double red[256];
    const int nx = d.nx;
    const int J = 1 + blockIdx.x / d.nz;
    const int z = blockIdx.x % d.nz;
    const size_t row = ((size_t)J * d.nz + z) * d.ldx;
    fill_pair_inverse(work, X + row, X + x_fstride + row, nx, d.nkx);
    fill_pair_inverse(work + nx, X + 2 * x_fstride + row, (const cpx<double>*)nullptr, nx, d.nkx);
    __syncthreads();
    smem_fft<double, PROD_VMAX, true>(work, 2, 1, nx, px, twx, +1);
    double m = __longlong_as_double(0x7ff0000000000000LL);   // +inf
    const double dyj = dy[J];
    for (int x = threadIdx.x; x < nx; x += blockDim.x) {
        const double u1 = work[x].x, u2 = work[x].y, u3 = work[nx + x].x;
        const double tx = cfl * dx / fabs(u1);
        const double ty = cfl * dyj / fabs(u2);
        const double tz = cfl * dz / fabs(u3);
        m = fmin(m, fmin(tx, fmin(ty, tz)));
    }
    red[threadIdx.x] = m;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] = fmin(red[threadIdx.x], red[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) atomic_min_pos(dtmin, red[0]);
}

cudaError_t launch_cfl(const Dims& d, const void* X, size_t x_fstride, const FftPlan& px,
                       const void* twx, const double* dy, double cfl, double dx, double dz,
                       double* dtmin, cudaStream_t st) {
    const size_t smem = sizeof(cpx<double>) * 2 * (size_t)d.nx;
    cudaFuncSetAttribute(k_cfl, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_cfl<<<d.ny * d.nz, 256, smem, st>>>(d, (const cpx<double>*)X, x_fstride, px,
                                         (const cpx<double>*)twx, dy, cfl, dx, dz, dtmin);
    return cudaGetLastError();
}

// explicit instantiations
template cudaError_t launch_zinv<float>(const Dims&, const double2*, size_t, void*, size_t, int, int, int,
                                        const FftPlan&, const void*, cudaStream_t);
template cudaError_t launch_zinv<double>(const Dims&, const double2*, size_t, void*, size_t, int, int, int,
                                         const FftPlan&, const void*, cudaStream_t);
template cudaError_t launch_products<float>(const Dims&, const void*, void*, int, int, int, const double*,
                                            const double*, const FftPlan&, const void*, cudaStream_t);
template cudaError_t launch_products<double>(const Dims&, const void*, void*, int, int, int, const double*,
                                             const double*, const FftPlan&, const void*, cudaStream_t);
template cudaError_t launch_zfwd_nl<float>(const Dims&, const void*, void*, int, int, const double*,
                                           const double*, const FftPlan&, const void*, cudaStream_t);
template cudaError_t launch_zfwd_nl<double>(const Dims&, const void*, void*, int, int, const double*,
                                            const double*, const FftPlan&, const void*, cudaStream_t);

}  // namespace dgpu
