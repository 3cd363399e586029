// transforms.cu -- x/z transform kernels of the channel timestep (sm_100a).
//
// The reference transforms one y-plane at a time with FFTW and an MPI
// all-to-all between the x and z stages (FFT_XZ_TO_FOURIER / _PHYSICAL,
// for/mpi.f:1477-1606).  Here the z stage and the x stage are separate
// kernels over all planes; the transpose between them is the X layout in
// device memory, and the physical-space products of RK_CHAN_1 never leave
// shared memory: one kernel per z-row goes from the x spectra of the state
// to the x spectra of the products.
//
// Real transforms along x use the half-length complex FFT of one signal
// (even samples in the real part, odd samples in the imaginary part), so
// every row keeps the relative accuracy of its own magnitude in FP32.
// Lengths in the fast lists below run with compile-time sizes (fftct.cuh);
// any other product of 2, 3 and 5 runs with the run-time plan (fft.cuh).
#include <cuda_runtime.h>

#include <stdint.h>

#include <type_traits>

#include "fft.cuh"
#include "fftct.cuh"
#include "kernels.cuh"
#include "launch.h"

namespace dgpu {

template <typename T>
__device__ __forceinline__ cpx<T> ld(const double2* p) {
    double2 v = *p;
    return mk<T>((T)v.x, (T)v.y);
}

// 16-byte asynchronous global -> shared copies (sm_80+ cp.async).
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Packed kz index m in [0,TNKZ] -> full z index in [0,NZ) (mpi.f:1530-1539).
__device__ __forceinline__ int m_to_z(int m, int nkz, int nz, int nkzt) {
    return m <= nkz ? m : m + nz - nkzt;
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

// Column-layout transform of TX interleaved columns of length NC (or the
// run-time plan when NC == 0).
template <typename T, int NC, int TX, int S>
__device__ __forceinline__ void col_fft(cpx<T>* buf, const FftPlan& P, const cpx<T>* __restrict__ tw) {
    ColLayout<TX> lay;
    if constexpr (NC > 0) fft_ct<T, NC, S, ColLayout<TX>, TX, 256, 8>(buf, TX, lay, tw);
    else smem_fft<T, ZTile<T>::VMAX>(buf, TX, lay, P, tw, S);
}

// ---------------------------------------------------------------------------
// K1: spectral (FP64) -> x-spectrum (T); inverse z transform along columns.
// Block (kx tile of TX columns, plane J, field f); 256 threads.
// ---------------------------------------------------------------------------
// With skip_mean the (kx,kz) = (0,0) mode (the plane mean) is left out, so X
// holds the fluctuation about each plane's mean.
template <typename T, int NC, int TX>
__device__ __forceinline__ void zinv_body(const Dims& d, const double2* __restrict__ S, size_t s_fstride,
                                          cpx<T>* __restrict__ X, size_t x_fstride, int j0, const FftPlan& pz,
                                          const cpx<T>* __restrict__ twz, int skip_mean, uint3 bid) {
    extern __shared__ unsigned char smem_raw[];
    cpx<T>* buf = reinterpret_cast<cpx<T>*>(smem_raw);   // [nz][TX]
    const int nz = NC > 0 ? NC : d.nz;
    const int nkz = nz / 3, nkzt = 2 * nkz + 1;
    const int kx0 = bid.x * TX;
    const int J = j0 + bid.y;
    const int f = bid.z;
    const double2* src = S + (size_t)f * s_fstride + (size_t)J * d.splane();
    for (int e = threadIdx.x; e < nz * TX; e += 256) {
        const int z = e / TX, c = e % TX;
        const int kx = kx0 + c;
        int m = -1;
        if (z <= nkz) m = z;
        else if (z >= nz - nkz) m = z - nz + nkzt;
        cpx<T> v = mk<T>(0, 0);
        if (m >= 0 && kx < d.nkxp && !(skip_mean && m == 0 && kx == 0)) v = ld<T>(src + (size_t)m * d.ldx + kx);
        buf[e] = v;
    }
    __syncthreads();
    col_fft<T, NC, TX, +1>(buf, pz, twz);
    cpx<T>* dst = X + (size_t)f * x_fstride + (size_t)J * nz * d.ldx;
    for (int e = threadIdx.x; e < nz * TX; e += 256) {
        const int z = e / TX, c = e % TX;
        dst[(size_t)z * d.ldx + kx0 + c] = buf[e];
    }
}

template <typename T, int NC, int TX>
__global__ void __launch_bounds__(256) k_zinv(Dims d, const double2* __restrict__ S, size_t s_fstride,
                                              cpx<T>* __restrict__ X, size_t x_fstride, int j0,
                                              FftPlan pz, const cpx<T>* __restrict__ twz, int skip_mean) {
    zinv_body<T, NC, TX>(d, S, s_fstride, X, x_fstride, j0, pz, twz, skip_mean, blockIdx);
}

// Batched form: instance blockIdx.z / nfields of a group of equal shape.
template <typename T, int NC, int TX>
__global__ void __launch_bounds__(256) k_zinv_b(const InstPtrs* __restrict__ ip, int nfields, Dims d,
                                                size_t s_fstride, size_t x_fstride, FftPlan pz,
                                                const cpx<T>* __restrict__ twz, int skip_mean) {
    const InstPtrs q = ip[blockIdx.z / nfields];
    zinv_body<T, NC, TX>(d, q.cu, s_fstride, reinterpret_cast<cpx<T>*>(q.xb), x_fstride, 0, pz, twz, skip_mean,
                         make_uint3(blockIdx.x, blockIdx.y, blockIdx.z % nfields));
}

// ---------------------------------------------------------------------------
// Real transforms of length N = 2M through one M-point complex FFT.
// ---------------------------------------------------------------------------
// Row b of buf <- Z_k = (X_k + conj X_{M-k}) + i w^k (X_k - conj X_{M-k}),
// w = exp(2 pi i/N), from the half spectrum x (entries k <= nkx; zero
// beyond, Nyquist zero, imaginary part of the DC bin dropped as FFTW's c2r
// does).  The backward M-point FFT of that row gives x_{2m} + i x_{2m+1}.
template <typename T, class L>
__device__ __forceinline__ void fill_real_inverse(cpx<T>* buf, const L& lay, int b, const cpx<T>* __restrict__ x,
                                                  int M, int nkx, const cpx<T>* __restrict__ twn, int k) {
    cpx<T> a = mk<T>(0, 0), c = mk<T>(0, 0);
    if (k <= nkx) {
        a = x[k];
        if (k == 0) a.y = 0;
    }
    const int kk = M - k;
    if (kk <= nkx) c = conjg(x[kk]);
    const cpx<T> A = a + c;
    const cpx<T> B = cmul(a - c, conjg(twn[k]));
    buf[lay.at(k, b)] = mk<T>(A.x - B.y, A.y + B.x);
}

// From Z = FFT_M(x_{2m} + i x_{2m+1}) (row b of buf): X_k = E_k + W^k O_k,
// E_k = (Z_k + conj Z_{M-k})/2, O_k = (Z_k - conj Z_{M-k})/(2i),
// W = exp(-2 pi i/N); scaled, zero beyond nkx.
template <typename T, class L>
__device__ __forceinline__ cpx<T> extract_real_forward(const cpx<T>* buf, const L& lay, int b, int M, int nkx,
                                                       const cpx<T>* __restrict__ twn, int k, T scale) {
    if (k > nkx) return mk<T>(0, 0);
    const cpx<T> zk = buf[lay.at(k, b)];
    const cpx<T> zm = buf[lay.at(k == 0 ? 0 : M - k, b)];
    const cpx<T> E = mk<T>((zk.x + zm.x) * T(0.5), (zk.y - zm.y) * T(0.5));
    const cpx<T> O = mk<T>((zk.y + zm.y) * T(0.5), (zm.x - zk.x) * T(0.5));
    const cpx<T> X = E + cmul(twn[k], O);
    return X * scale;
}

constexpr int PROD_G = 16;          // rows transformed together by the products kernel
constexpr int RT_VMAX = 12;         // run-time path: values per thread

// nrows <= PROD_G * ZB rows of length M (MC at compile time, else the plan's)
template <typename T, int MC, int S, int ZB = 1, class L>
__device__ __forceinline__ void row_fft(cpx<T>* buf, int nrows, const L& lay, const FftPlan& P,
                                        const cpx<T>* __restrict__ tw) {
    if constexpr (MC > 0) fft_ct<T, MC, S, L, PROD_G * ZB, 256>(buf, nrows, lay, tw);
    else smem_fft<T, RT_VMAX>(buf, nrows, lay, P, tw, S);
}

// z-rows per products block: several at small NX, where one row's transforms
// leave most of the 256 threads idle between barriers (shared memory of four
// FP32 rows or two FP64 rows at NX = 128: 76 KB)
template <typename T, int MC>
__host__ __device__ constexpr int products_zb() { return (MC > 0 && MC <= 64) ? (sizeof(T) == 4 ? 4 : 2) : 1; }

// ---------------------------------------------------------------------------
// K2: per z-row, marching over planes.  Iteration J transforms, in one
// batch of forward M-point FFTs, the fields of plane J back to physical
// space (the backward FFT taken as conj(FFT(conj(.))) so that both halves of
// the batch share one transform) and the products of plane J-2, whose
// neighbours J-3..J-1 are already in the ring of physical planes; then
// unpacks the fields into the ring and writes the products' x spectra.
// ---------------------------------------------------------------------------
constexpr int RING = 4;

// Sources of product output q (x spectra, S layout of the nonlinear terms of
// channel.f:410-571, 670-720): field f = q/2 has
//   q = 2f:   ikx*Pa + Pflux   (the x-derivative and y-flux terms)
//   q = 2f+1: Pz               (the z-derivative term, ikz applied after the z transform)
//   U1: Pa=P1 (U1U1), Pflux=P5, Pz=P0 (U1U3)   U2: Pa=P3, Pflux=P7, Pz=P4
//   U3: Pa=P0 (U1U3), Pflux=P6, Pz=P2          TH_n: Pa=P(8+3n), Pflux=P(10+3n), Pz=P(9+3n)
__device__ __forceinline__ int field_pz(int f) { return f == 0 ? 0 : f == 1 ? 4 : f == 2 ? 2 : 9 + 3 * (f - 3); }
__device__ __forceinline__ int field_sources(int q, int* sp, bool* sx) {
    const int f = q >> 1;
    int pa, pf, pz;
    if (f == 0) { pa = 1; pf = 5; pz = 0; }
    else if (f == 1) { pa = 3; pf = 7; pz = 4; }
    else if (f == 2) { pa = 0; pf = 6; pz = 2; }
    else { const int n = f - 3; pa = 8 + 3 * n; pf = 10 + 3 * n; pz = 9 + 3 * n; }
    if (q & 1) { sp[0] = pz; sx[0] = false; return 1; }
    sp[0] = pa; sx[0] = true;
    sp[1] = pf; sx[1] = false;
    return 2;
}

// ZB z-rows per block (rows z0 .. z0+ZB-1 side by side in every buffer): at
// small NX one row's transforms leave most of the block idle between barriers.
template <typename T, int MC, int ZB>
__device__ __forceinline__ void products_body(const Dims& d, const cpx<T>* __restrict__ X, cpx<T>* __restrict__ Y,
                                              int jlo, int jhi, int chunk, int group, const double* __restrict__ dy,
                                              const double* __restrict__ dyf, const double* __restrict__ kxw,
                                              const FftPlan& pm, const cpx<T>* __restrict__ twm,
                                              const cpx<T>* __restrict__ twn, const double2* __restrict__ means,
                                              size_t means_fs, uint3 bid) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ T smean[RING][MAXF];   // plane means of the ring planes (zero without mean split)
    const int M = MC > 0 ? MC : d.nx / 2;
    const int nx = 2 * M;
    const int nf = d.nf, np = d.np, nrow = nf + np;
    using Lay = typename std::conditional<(MC > 0), RowLayoutCT<MC>, RowLayoutRT>::type;
    Lay lay;
    if constexpr (MC == 0) lay.pitch = row_pitch(M);
    const size_t ringz = (size_t)RING * nf * nx;                              // one z-row's ring
    T* ring0 = reinterpret_cast<T*>(smem_raw);                                // [ZB][RING][nf][nx]
    cpx<T>* stw = reinterpret_cast<cpx<T>*>(ring0 + ringz * ZB);              // twiddles: M then NX
    cpx<T>* buf = stw + 3 * M;                                                // [ZB * group][pitch]
    T* tbuf = reinterpret_cast<T*>(buf);
    // [2][ZB][nf][ldx] x spectra of the fields, the next plane's in flight
    cpx<T>* xs = reinterpret_cast<cpx<T>*>(
        (reinterpret_cast<uintptr_t>(buf + (size_t)ZB * min(group, nrow) * (lay.at(0, 1) - lay.at(0, 0))) + 15) &
        ~(uintptr_t)15);                                                      // 16-byte aligned
    for (int e = threadIdx.x; e < 3 * M; e += 256) stw[e] = e < M ? twm[e] : twn[e - M];
    twm = stw;
    twn = stw + M;
    __syncthreads();
    const int z0 = bid.x * ZB;
    const int jb = jlo + bid.y * chunk;
    const int je = min(jb + chunk - 1, jhi);
    if (jb > jhi) return;                                 // batched form: past this instance's planes
    const size_t xrow = (size_t)d.nz * d.ldx;            // plane stride of X / Y
    const size_t xf = (size_t)d.nyp * xrow;              // field stride of X / Y
    const T inv_nx = T(1.0 / (double)nx);
    auto slot = [&](int j) { return (j - (jb - 1)) % RING; };
    constexpr int CPC = 16 / (int)sizeof(cpx<T>);      // complex numbers per 16-byte copy
    auto stage = [&](int Jn) {
        cpx<T>* dst = xs + (size_t)(Jn & 1) * ZB * nf * d.ldx;
        const int nch = d.ldx / CPC;
        for (int e = threadIdx.x; e < ZB * nf * nch; e += 256) {
            const int zz = e / (nf * nch), rem = e % (nf * nch);
            const int f = rem / nch, q = rem % nch;
            cp_async16(dst + ((size_t)zz * nf + f) * d.ldx + q * CPC,
                       X + (size_t)f * xf + (size_t)Jn * xrow + (size_t)(z0 + zz) * d.ldx + q * CPC);
        }
        cp_async_commit();
    };
    stage(jb - 1);
    for (int J = jb - 1; J <= je + 2; ++J) {
        const bool do_inv = (J <= je + 1);
        if (do_inv && threadIdx.x < nf)   // slot(J) last held plane J-4, which no product reads any more
            smean[slot(J)][threadIdx.x] = means ? (T)means[threadIdx.x * means_fs + (size_t)J * d.splane()].x : T(0);
        if (do_inv) {
            if (J + 1 <= je + 1) {
                stage(J + 1);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();
        }
        const int jp = J - 2;                            // plane whose products are formed
        const bool do_prod = (jp >= jb);
        const int r0 = do_inv ? 0 : nf, r1 = do_prod ? nrow : nf;
        T a1 = 0, a0 = 0, i2dyf = 0, idy = 0;
        if (do_prod) {
            a1 = (T)(dyf[jp] / (2.0 * dy[jp]));
            a0 = (T)(dyf[jp - 1] / (2.0 * dy[jp]));
            i2dyf = (T)(1.0 / (2.0 * dyf[jp]));
            idy = (T)(1.0 / dy[jp]);
        }
        for (int c0 = r0; c0 < r1; c0 += group) {
            const int nr = min(group, r1 - c0);
            // ---- fill: conjugated half spectra of the fields, products ----
            const int nfill = max(0, min(nf, c0 + nr) - c0);        // inverse rows in this chunk
            // buffer row of (z-row zz, row r of this chunk): zz * nr + r
            for (int e = threadIdx.x; e < ZB * nfill * M; e += 256) {
                const int zz = e / (nfill * M), rem = e % (nfill * M);
                const int r = rem / M, k = rem % M, row = zz * nr + r;
                const cpx<T>* xr = xs + (((size_t)(J & 1) * ZB + zz) * nf + c0 + r) * d.ldx;
                fill_real_inverse(buf, lay, row, xr, M, d.nkx, twn, k);
                buf[lay.at(k, row)].y = -buf[lay.at(k, row)].y;
            }
            const int p0 = max(c0, nf) - nf, p1 = c0 + nr - nf;       // products p0..p1-1 here
            if (p1 > p0) {
                const int sm = slot(jp - 1), s0 = slot(jp), sp = slot(jp + 1);
                // The ring holds each field as fluctuation a' about its plane mean
                // abar (abar = 0 without the mean split).  A product ab is formed
                // as its part beyond abar*bbar: a'(bbar + b') + abar b', whose
                // rounding error is relative to the fluctuations, not to the O(1)
                // means.  abar*bbar reaches only the (0,0) mode, which the column
                // kernel adds in FP64.
                const T m1m = smean[sm][0], m1 = smean[s0][0], m1p = smean[sp][0];
                const T m2m = smean[sm][1], m2 = smean[s0][1], m2p = smean[sp][1];
                const T m3m = smean[sm][2], m3 = smean[s0][2], m3p = smean[sp][2];
                for (int ex = threadIdx.x; ex < ZB * nx; ex += 256) {
                    const int zz = ex / nx, x = ex % nx;
                    const T* ring = ring0 + ringz * zz;
                    const T* r_m = ring + (size_t)sm * nf * nx + x;
                    const T* r_c = ring + (size_t)s0 * nf * nx + x;
                    const T* r_p = ring + (size_t)sp * nf * nx + x;
                    const T u1m = r_m[0], u1 = r_c[0], u1p = r_p[0];
                    const T u2m = r_m[nx], u2 = r_c[nx], u2p = r_p[nx];
                    const T u3m = r_m[2 * nx], u3 = r_c[2 * nx], u3p = r_p[2 * nx];
                    const T U1 = m1 + u1, U2 = m2 + u2, U2p = m2p + u2p, U3 = m3 + u3;
                    T v[8];
                    v[0] = u3 * U1 + m3 * u1;                                   // U1 U3
                    v[1] = u1 * (U1 + m1);                                      // U1 U1
                    v[2] = u3 * (U3 + m3);                                      // U3 U3
                    v[3] = (a1 * u1 + a0 * u1m) * U2 + (a1 * m1 + a0 * m1m) * u2;   // (U1 at GY) U2
                    v[4] = (a1 * u3 + a0 * u3m) * U2 + (a1 * m3 + a0 * m3m) * u2;   // (U3 at GY) U2
                    // (U1(j+1) + U1(j)) U2(j+1) - (U1(j) + U1(j-1)) U2(j), over 2 DYF(j)
                    v[5] = ((u1p + u1) * U2p + (m1p + m1) * u2p - (u1 + u1m) * U2 - (m1 + m1m) * u2) * i2dyf;
                    v[6] = ((u3p + u3) * U2p + (m3p + m3) * u2p - (u3 + u3m) * U2 - (m3 + m3m) * u2) * i2dyf;
                    // (U2(j) + U2(j+1))^2/4 - (U2(j) + U2(j-1))^2/4, over DY(j)
                    const T s1 = u2 + u2p, s2 = u2 + u2m, S1 = m2 + m2p, S2 = m2 + m2m;
                    v[7] = T(0.25) * (s1 * (s1 + T(2) * S1) - s2 * (s2 + T(2) * S2)) * idy;
                    const int eoff = 2 * lay.at(x >> 1, zz * nr) + (x & 1);
                    const int rstride = 2 * (lay.at(0, 1) - lay.at(0, 0));
#pragma unroll
                    for (int p = 0; p < 8; ++p)
                        if (p >= p0 && p < p1) tbuf[eoff + (nf + p - c0) * rstride] = v[p];
                    for (int n = 0; n < d.nth; ++n) {
                        const T thm = r_m[(3 + n) * nx], th = r_c[(3 + n) * nx], thp = r_p[(3 + n) * nx];
                        const T tm = smean[sm][3 + n], tc = smean[s0][3 + n], tp = smean[sp][3 + n];
                        T w[3];
                        w[0] = th * U1 + tc * u1;                               // TH U1
                        w[1] = th * U3 + tc * u3;                               // TH U3
                        w[2] = ((thp + th) * U2p + (tp + tc) * u2p - (th + thm) * U2 - (tc + tm) * u2) * i2dyf;
#pragma unroll
                        for (int r = 0; r < 3; ++r) {
                            const int p = 8 + 3 * n + r;
                            if (p >= p0 && p < p1) tbuf[eoff + (nf + p - c0) * rstride] = w[r];
                        }
                    }
                }
            }
            __syncthreads();
            row_fft<T, MC, -1, ZB>(buf, ZB * nr, lay, pm, twm);
            // ---- unpack the fields of plane J, write the products of jp --------
            if (nfill > 0) {
                const int sl = slot(J);
                for (int e = threadIdx.x; e < ZB * nfill * M; e += 256) {
                    const int zz = e / (nfill * M), rem = e % (nfill * M);
                    const int r = rem / M, m = rem % M;
                    const cpx<T> v = buf[lay.at(m, zz * nr + r)];
                    T* dst = ring0 + ringz * zz + ((size_t)sl * nf + c0 + r) * nx + 2 * m;
                    dst[0] = v.x;
                    dst[1] = -v.y;
                }
            }
            if (p0 == 0 && p1 == np && d.nth <= 1) {
                // every product is in this batch (N_TH <= 1): one thread per kx
                // extracts each product spectrum once and forms the 2 outputs of
                // every field (field_sources)
                for (int ek = threadIdx.x; ek < ZB * d.ldx; ek += 256) {
                    const int zz = ek / d.ldx, k = ek % d.ldx;
                    cpx<T>* yk = Y + (size_t)jp * xrow + (size_t)(z0 + zz) * d.ldx + k;
                    if (k > d.nkx) {
                        for (int q = 0; q < 2 * nf; ++q) yk[(size_t)q * xf] = mk<T>(0, 0);
                        continue;
                    }
                    const int km = k == 0 ? 0 : M - k;
                    const cpx<T> w = twn[k];
                    const T hs = T(0.5) * inv_nx;
                    const int ok = lay.at(k, 0), om = lay.at(km, 0);
                    const int rs = lay.at(0, 1) - lay.at(0, 0);
                    auto X = [&](int p) -> cpx<T> {
                        const int row = (zz * nr + nf + p - c0) * rs;
                        const cpx<T> zk = buf[row + ok], zm = buf[row + om];
                        const cpx<T> E = mk<T>(zk.x + zm.x, zk.y - zm.y);
                        const cpx<T> O = mk<T>(zk.y + zm.y, zm.x - zk.x);
                        return (E + cmul(w, O)) * hs;
                    };
                    const T K = (T)kxw[k];
                    auto ikx = [&](cpx<T> v) { return mk<T>(-K * v.y, K * v.x); };
                    const cpx<T> x0 = X(0);
                    yk[0 * xf] = ikx(X(1)) + X(5);
                    yk[1 * xf] = x0;
                    yk[2 * xf] = ikx(X(3)) + X(7);
                    yk[3 * xf] = X(4);
                    yk[4 * xf] = ikx(x0) + X(6);
                    yk[5 * xf] = X(2);
                    if (nf > 3) {
                        yk[6 * xf] = ikx(X(8)) + X(10);
                        yk[7 * xf] = X(9);
                    }
                }
            } else if (p1 > p0) {
                // outputs of field f: 2f = ikx*Pa + Pflux, 2f+1 = Pz (field_sources);
                // an output whose sources span two batches is completed by adding to
                // what the earlier batch stored
                for (int e3 = threadIdx.x; e3 < ZB * nf * d.ldx; e3 += 256) {
                    const int zz = e3 / (nf * d.ldx), e = e3 % (nf * d.ldx);
                    const int f = e / d.ldx, k = e % d.ldx;
                    int sp[2];
                    bool sx[2];
                    field_sources(2 * f, sp, sx);
                    const int pz = field_pz(f);
                    cpx<T>* ya = Y + (size_t)(2 * f) * xf + (size_t)jp * xrow + (size_t)(z0 + zz) * d.ldx + k;
                    const bool ina = sp[0] >= p0 && sp[0] < p1, inf = sp[1] >= p0 && sp[1] < p1;
                    if (ina || inf) {
                        cpx<T> v = mk<T>(0, 0);
                        if (ina) {
                            const cpx<T> x = extract_real_forward(buf, lay, zz * nr + nf + sp[0] - c0, M, d.nkx, twn, k, inv_nx);
                            const T K = (T)kxw[k];
                            v = mk<T>(-K * x.y, K * x.x);
                        }
                        if (inf) v = v + extract_real_forward(buf, lay, zz * nr + nf + sp[1] - c0, M, d.nkx, twn, k, inv_nx);
                        if ((!ina && sp[0] < p0) || (!inf && sp[1] < p0)) v = v + *ya;
                        *ya = v;
                    }
                    if (pz >= p0 && pz < p1)
                        ya[xf] = extract_real_forward(buf, lay, zz * nr + nf + pz - c0, M, d.nkx, twn, k, inv_nx);
                }
            }
            __syncthreads();
        }
    }
}

template <typename T, int MC, int ZB>
__global__ void __launch_bounds__(256, 2) k_products(Dims d, const cpx<T>* __restrict__ X,
                                                     cpx<T>* __restrict__ Y, int jlo, int jhi, int chunk,
                                                     int group, const double* __restrict__ dy,
                                                     const double* __restrict__ dyf,
                                                     const double* __restrict__ kxw, FftPlan pm,
                                                     const cpx<T>* __restrict__ twm,
                                                     const cpx<T>* __restrict__ twn,
                                                     const double2* __restrict__ means, size_t means_fs) {
    products_body<T, MC, ZB>(d, X, Y, jlo, jhi, chunk, group, dy, dyf, kxw, pm, twm, twn, means, means_fs, blockIdx);
}

// Batched form: instance blockIdx.z of a group of equal shape.
template <typename T, int MC, int ZB>
__global__ void __launch_bounds__(256, 2) k_products_b(const InstPtrs* __restrict__ ip, Dims d, int jhi, int chunk,
                                                       int group, FftPlan pm, const cpx<T>* __restrict__ twm,
                                                       const cpx<T>* __restrict__ twn, int mean_split,
                                                       size_t means_fs) {
    const InstPtrs q = ip[blockIdx.z];
    products_body<T, MC, ZB>(d, reinterpret_cast<const cpx<T>*>(q.xb), reinterpret_cast<cpx<T>*>(q.yb), q.jlo_prod,
                             jhi, chunk, group, q.dy, q.dyf, q.kx, pm, twm, twn, mean_split ? q.cu : nullptr,
                             means_fs, make_uint3(blockIdx.x, blockIdx.y, 0));
}

// ---------------------------------------------------------------------------
// K3: per plane, kx tile and field: forward z transform of the two product
// outputs that feed the field, kz packing with 1/NZ, and the derivative
// combination into the nonlinear term (channel.f:410-571, 670-720):
//   U1: -ikz P0 - ikx P1 - P5      U2: -ikx P3 - ikz P4 - P7
//   U3: -ikx P0 - ikz P2 - P6      TH_n: -ikx P(8+3n) - ikz P(9+3n) - P(10+3n)
// with P0 = U1U3, P1 = U1U1, P2 = U3U3, P3/P4 = (U1/U3 at GY) U2,
// P5..P7 the y-flux differences; the ikx and y-flux terms arrive already
// summed from K2.
// ---------------------------------------------------------------------------
// The two product outputs of field f (see field_sources) and their use:
// NL_f = -(z transform of output 2f) - ikz (z transform of output 2f+1).
__device__ __forceinline__ void field_products(int f, int* p, int* mlt) {
    p[0] = 2 * f; mlt[0] = 0;
    p[1] = 2 * f + 1; mlt[1] = 2;
}


// Block: kx tile of TX columns, field f, planes J0 .. J0+zp-1 (zp, the planes
// per block, is a launch parameter).  The 2*zp product tiles it consumes
// stream through two shared buffers
// (cp.async), the next tile in flight while the current one is transformed.
constexpr int ZF_PLANES = 8;   // default planes per block
// kx columns per z-forward block (measured at 512x257x384: FP32 8, FP64 4)
template <typename T>
struct ZfTile { static constexpr int TX = 8; };
template <>
struct ZfTile<double> { static constexpr int TX = 4; };

template <typename T, int NC, int TX>
__device__ __forceinline__ void zfwd_nl_body(const Dims& d, const cpx<T>* __restrict__ Y, cpx<T>* __restrict__ NL,
                                             int jlo, int jhi, int zp, const double* __restrict__ kxw,
                                             const double* __restrict__ kzw, const FftPlan& pz,
                                             const cpx<T>* __restrict__ twz, uint3 bid) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nz = NC > 0 ? NC : d.nz;
    const int nkz = nz / 3, nkzt = 2 * nkz + 1;
    constexpr int QA = NC > 0 ? ((2 * (NC / 3) + 1) * TX + 255) / 256 : 1;
    cpx<T>* bufs = reinterpret_cast<cpx<T>*>(smem_raw);          // [2][nz][TX]
    cpx<T>* sacc = bufs + 2 * (size_t)nz * TX;                    // run-time path: [nkzt][TX]
    const int kx0 = bid.x * TX;
    const int f = bid.z;
    const int J0 = jlo + bid.y * zp;
    const int nplanes = min(zp, jhi - J0 + 1);
    if (nplanes <= 0) return;                             // batched form: past this instance's planes
    const size_t xrow = (size_t)nz * d.ldx;
    const size_t xf = (size_t)d.nyp * xrow;
    const T inv_nz = T(1.0 / (double)nz);
    int prod[2], mlt[2];
    field_products(f, prod, mlt);
    const size_t sp = d.splane();
    const size_t sf = (size_t)d.nyp * sp;
    constexpr int CH = (int)(TX * sizeof(cpx<T>) / 16);           // 16-byte chunks per z row
    auto load = [&](int t, int buf) {                             // tile t = 3*plane + product
        const int J = J0 + t / 2;
        const cpx<T>* src = Y + (size_t)prod[t % 2] * xf + (size_t)J * xrow + kx0;
        unsigned char* dst = reinterpret_cast<unsigned char*>(bufs + (size_t)buf * nz * TX);
        for (int e = threadIdx.x; e < nz * CH; e += 256) {
            const int z = e / CH, q = e % CH;
            cp_async16(dst + (size_t)z * TX * sizeof(cpx<T>) + q * 16,
                       reinterpret_cast<const unsigned char*>(src + (size_t)z * d.ldx) + q * 16);
        }
        cp_async_commit();
    };
    const int ntiles = 2 * nplanes;
    load(0, 0);
    cpx<T> acc[QA];
    for (int t = 0; t < ntiles; ++t) {
        const int pl = t / 2, r = t % 2;
        if (t + 1 < ntiles) {
            load(t + 1, (t + 1) & 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        cpx<T>* buf = bufs + (size_t)(t & 1) * nz * TX;
        col_fft<T, NC, TX, -1>(buf, pz, twz);
        const int mt = mlt[r];
        if (r == 0) {
#pragma unroll
            for (int q = 0; q < QA; ++q) acc[q] = mk<T>(0, 0);
            if constexpr (NC == 0)
                for (int e = threadIdx.x; e < nkzt * TX; e += 256) sacc[e] = mk<T>(0, 0);
        }
        if constexpr (NC > 0) {
#pragma unroll
            for (int q = 0; q < QA; ++q) {
                const int e = threadIdx.x + q * 256;
                if (e < nkzt * TX) {
                    const int m = e / TX, c = e % TX;
                    const cpx<T> v = buf[(size_t)m_to_z(m, nkz, nz, nkzt) * TX + c] * inv_nz;
                    if (mt == 0) acc[q] = acc[q] - v;
                    else {
                        const T K = mt == 1 ? (T)kxw[kx0 + c] : (T)kzw[m];
                        acc[q] = mk<T>(acc[q].x + K * v.y, acc[q].y - K * v.x);
                    }
                }
            }
        } else {
            for (int e = threadIdx.x; e < nkzt * TX; e += 256) {
                const int m = e / TX, c = e % TX;
                const cpx<T> v = buf[(size_t)m_to_z(m, nkz, nz, nkzt) * TX + c] * inv_nz;
                cpx<T> a = sacc[e];
                if (mt == 0) a = a - v;
                else {
                    const T K = mt == 1 ? (T)kxw[kx0 + c] : (T)kzw[m];
                    a = mk<T>(a.x + K * v.y, a.y - K * v.x);
                }
                sacc[e] = a;
            }
        }
        if (r == 1) {
            cpx<T>* dst = NL + (size_t)f * sf + (size_t)(J0 + pl) * sp + kx0;
            if constexpr (NC > 0) {
#pragma unroll
                for (int q = 0; q < QA; ++q) {
                    const int e = threadIdx.x + q * 256;
                    if (e < nkzt * TX) dst[(size_t)(e / TX) * d.ldx + e % TX] = acc[q];
                }
            } else {
                __syncthreads();
                for (int e = threadIdx.x; e < nkzt * TX; e += 256) dst[(size_t)(e / TX) * d.ldx + e % TX] = sacc[e];
            }
        }
        __syncthreads();   // buffer t&1 is refilled by the load issued next iteration
    }
}

template <typename T, int NC, int TX>
__global__ void __launch_bounds__(256, 2) k_zfwd_nl(Dims d, const cpx<T>* __restrict__ Y,
                                                    cpx<T>* __restrict__ NL, int jlo, int jhi, int zp,
                                                    const double* __restrict__ kxw,
                                                    const double* __restrict__ kzw, FftPlan pz,
                                                    const cpx<T>* __restrict__ twz) {
    zfwd_nl_body<T, NC, TX>(d, Y, NL, jlo, jhi, zp, kxw, kzw, pz, twz, blockIdx);
}

// Batched form: instance blockIdx.z / nf of a group of equal shape.
template <typename T, int NC, int TX>
__global__ void __launch_bounds__(256, 2) k_zfwd_nl_b(const InstPtrs* __restrict__ ip, Dims d, int jhi, int zp,
                                                      FftPlan pz, const cpx<T>* __restrict__ twz) {
    const InstPtrs q = ip[blockIdx.z / d.nf];
    zfwd_nl_body<T, NC, TX>(d, reinterpret_cast<const cpx<T>*>(q.yb), reinterpret_cast<cpx<T>*>(q.nl), q.jlo_prod,
                            jhi, zp, q.kx, q.kz, pz, twz, make_uint3(blockIdx.x, blockIdx.y, blockIdx.z % d.nf));
}

// ---------------------------------------------------------------------------
// Launchers with compile-time size dispatch.
// ---------------------------------------------------------------------------
#define DGPU_NZ_LIST(X) X(32) X(48) X(64) X(96) X(128) X(160) X(192) X(256) X(384) X(512)
#define DGPU_M_LIST(X) X(32) X(48) X(64) X(96) X(128) X(192) X(256)

template <typename T>
cudaError_t launch_zinv(const Dims& d, const double2* S, size_t s_fstride, void* X, size_t x_fstride,
                        int nfields, int j0, int nplanes, const FftPlan& pz, const void* twz,
                        cudaStream_t st, int skip_mean) {
    constexpr int TX = ZTile<T>::TX;
    if (nplanes <= 0 || nfields <= 0) return cudaSuccess;
    const size_t smem = sizeof(cpx<T>) * (size_t)d.nz * TX;
    dim3 grid(d.ldx / TX, nplanes, nfields);
    auto go = [&](auto kern) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<grid, 256, smem, st>>>(d, S, s_fstride, (cpx<T>*)X, x_fstride, j0, pz, (const cpx<T>*)twz,
                                      skip_mean);
    };
    switch (d.nz) {
#define CASE(N) case N: go(k_zinv<T, N, TX>); break;
        DGPU_NZ_LIST(CASE)
#undef CASE
        default: go(k_zinv<T, 0, TX>); break;
    }
    return cudaGetLastError();
}

int products_group(int nx) {
    const int m = nx / 2;
    if (m == 32 || m == 48 || m == 64 || m == 96 || m == 128 || m == 192 || m == 256) return PROD_G;
    int g = (RT_VMAX * 256) / m;
    return g > PROD_G ? PROD_G : g;
}

// Dynamic shared memory of a products block of zb z-rows: rings, twiddles,
// transform rows, staged x spectra (products_body's carve-up).
template <typename T>
size_t products_smem(const Dims& d, int group, int zb) {
    const int M = d.nx / 2;
    const int rows = group < d.nf + d.np ? group : d.nf + d.np;
    return zb * (sizeof(T) * (size_t)RING * d.nf * d.nx + sizeof(cpx<T>) * (size_t)rows * row_pitch(M) +
                 sizeof(cpx<T>) * 2 * (size_t)d.nf * d.ldx) +
           sizeof(cpx<T>) * 3 * (size_t)M + 16;
}

template <typename T>
cudaError_t launch_products(const Dims& d, const void* X, void* Y, int jlo, int jhi, int chunk,
                            const double* dy, const double* dyf, const double* kx, const FftPlan& pm,
                            const void* twm, const void* twn, cudaStream_t st, const double2* means,
                            size_t means_fstride) {
    if (jhi < jlo) return cudaSuccess;
    const int group = products_group(d.nx);
    if (group < 1) return cudaErrorInvalidValue;
    const int M = d.nx / 2;
    const int nchunks = (jhi - jlo + chunk) / chunk;
    auto go = [&](auto kern, int zb) {
        const size_t smem = products_smem<T>(d, group, zb);
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<dim3(d.nz / zb, nchunks), 256, smem, st>>>(d, (const cpx<T>*)X, (cpx<T>*)Y, jlo, jhi, chunk, group, dy,
                                                          dyf, kx, pm, (const cpx<T>*)twm, (const cpx<T>*)twn, means,
                                                          means_fstride);
    };
    switch (M) {
#define CASE(N)                                                                   \
    case N:                                                                       \
        if (d.nz % products_zb<T, N>() == 0) go(k_products<T, N, products_zb<T, N>()>, products_zb<T, N>()); \
        else go(k_products<T, N, 1>, 1);                                          \
        break;
        DGPU_M_LIST(CASE)
#undef CASE
        default: go(k_products<T, 0, 1>, 1); break;
    }
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_zfwd_nl(const Dims& d, const void* Y, void* NL, int jlo, int jhi, int zp,
                           const double* kx, const double* kz, const FftPlan& pz, const void* twz,
                           cudaStream_t st) {
    constexpr int TX = ZfTile<T>::TX;
    if (jhi < jlo) return cudaSuccess;
    if (zp < 1) zp = ZF_PLANES;
    dim3 grid(d.ldx / TX, (jhi - jlo + zp) / zp, d.nf);
    auto go = [&](auto kern, bool ct) {
        const size_t smem = sizeof(cpx<T>) * (2 * (size_t)d.nz * TX + (ct ? 0 : (size_t)d.nkzt * TX));
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<grid, 256, smem, st>>>(d, (const cpx<T>*)Y, (cpx<T>*)NL, jlo, jhi, zp, kx, kz, pz,
                                      (const cpx<T>*)twz);
    };
    switch (d.nz) {
#define CASE(N) case N: go(k_zfwd_nl<T, N, TX>, true); break;
        DGPU_NZ_LIST(CASE)
#undef CASE
        default: go(k_zfwd_nl<T, 0, TX>, false); break;
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Batched launchers: one launch covers the instances ip[0..ninst) of a group
// of equal shape; the instance is a grid coordinate and its arrays come from
// the device-side table ip.
// ---------------------------------------------------------------------------
template <typename T>
cudaError_t launch_zinv_b(const Dims& d, const InstPtrs* ip, int ninst, size_t s_fstride, size_t x_fstride,
                          const FftPlan& pz, const void* twz, cudaStream_t st, int skip_mean) {
    constexpr int TX = ZTile<T>::TX;
    const size_t smem = sizeof(cpx<T>) * (size_t)d.nz * TX;
    dim3 grid(d.ldx / TX, d.nyp, d.nf * ninst);
    auto go = [&](auto kern) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<grid, 256, smem, st>>>(ip, d.nf, d, s_fstride, x_fstride, pz, (const cpx<T>*)twz, skip_mean);
    };
    switch (d.nz) {
#define CASE(N) case N: go(k_zinv_b<T, N, TX>); break;
        DGPU_NZ_LIST(CASE)
#undef CASE
        default: go(k_zinv_b<T, 0, TX>); break;
    }
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_products_b(const Dims& d, const InstPtrs* ip, int ninst, int jlo_min, int jhi, int chunk,
                              const FftPlan& pm, const void* twm, const void* twn, cudaStream_t st, int mean_split,
                              size_t means_fstride) {
    if (jhi < jlo_min) return cudaSuccess;
    const int group = products_group(d.nx);
    if (group < 1) return cudaErrorInvalidValue;
    const int M = d.nx / 2;
    auto go = [&](auto kern, int zb) {
        const size_t smem = products_smem<T>(d, group, zb);
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<dim3(d.nz / zb, (jhi - jlo_min + chunk) / chunk, ninst), 256, smem, st>>>(
            ip, d, jhi, chunk, group, pm, (const cpx<T>*)twm, (const cpx<T>*)twn, mean_split, means_fstride);
    };
    switch (M) {
#define CASE(N)                                                                   \
    case N:                                                                       \
        if (d.nz % products_zb<T, N>() == 0) go(k_products_b<T, N, products_zb<T, N>()>, products_zb<T, N>()); \
        else go(k_products_b<T, N, 1>, 1);                                        \
        break;
        DGPU_M_LIST(CASE)
#undef CASE
        default: go(k_products_b<T, 0, 1>, 1); break;
    }
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_zfwd_nl_b(const Dims& d, const InstPtrs* ip, int ninst, int jlo_min, int jhi, int zp,
                             const FftPlan& pz, const void* twz, cudaStream_t st) {
    constexpr int TX = ZfTile<T>::TX;
    if (jhi < jlo_min) return cudaSuccess;
    if (zp < 1) zp = ZF_PLANES;
    dim3 grid(d.ldx / TX, (jhi - jlo_min + zp) / zp, d.nf * ninst);
    auto go = [&](auto kern, bool ct) {
        const size_t smem = sizeof(cpx<T>) * (2 * (size_t)d.nz * TX + (ct ? 0 : (size_t)d.nkzt * TX));
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<grid, 256, smem, st>>>(ip, d, jhi, zp, pz, (const cpx<T>*)twz);
    };
    switch (d.nz) {
#define CASE(N) case N: go(k_zfwd_nl_b<T, N, TX>, true); break;
        DGPU_NZ_LIST(CASE)
#undef CASE
        default: go(k_zfwd_nl_b<T, 0, TX>, false); break;
    }
    return cudaGetLastError();
}

template cudaError_t launch_zinv_b<float>(const Dims&, const InstPtrs*, int, size_t, size_t, const FftPlan&,
                                          const void*, cudaStream_t, int);
template cudaError_t launch_zinv_b<double>(const Dims&, const InstPtrs*, int, size_t, size_t, const FftPlan&,
                                           const void*, cudaStream_t, int);
template cudaError_t launch_products_b<float>(const Dims&, const InstPtrs*, int, int, int, int, const FftPlan&,
                                              const void*, const void*, cudaStream_t, int, size_t);
template cudaError_t launch_products_b<double>(const Dims&, const InstPtrs*, int, int, int, int, const FftPlan&,
                                               const void*, const void*, cudaStream_t, int, size_t);
template cudaError_t launch_zfwd_nl_b<float>(const Dims&, const InstPtrs*, int, int, int, int, const FftPlan&,
                                             const void*, cudaStream_t);
template cudaError_t launch_zfwd_nl_b<double>(const Dims&, const InstPtrs*, int, int, int, int, const FftPlan&,
                                              const void*, cudaStream_t);

// ---------------------------------------------------------------------------
// Transform-API helpers (FP64, one field).  Rows r = (J - j0)*NZ + z; a block
// handles `group` consecutive rows: PROD_G rows through the compile-time FFT
// when M = NX/2 has one (MC > 0), else a smaller group through the run-time
// FFT.  The M- and NX-point twiddles are staged in shared memory.
// ---------------------------------------------------------------------------
template <int MC>
__global__ void __launch_bounds__(256) k_xinv(Dims d, const cpx<double>* __restrict__ X,
                                              double* __restrict__ P, int j0, int nrows, int group,
                                              FftPlan pm, const cpx<double>* __restrict__ twm,
                                              const cpx<double>* __restrict__ twn) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int M = MC > 0 ? MC : d.nx / 2;
    using Lay = typename std::conditional<(MC > 0), RowLayoutCT<MC>, RowLayoutRT>::type;
    Lay lay;
    if constexpr (MC == 0) lay.pitch = row_pitch(M);
    cpx<double>* stw = reinterpret_cast<cpx<double>*>(smem_raw);
    cpx<double>* buf = stw + 3 * M;
    for (int e = threadIdx.x; e < 3 * M; e += 256) stw[e] = e < M ? twm[e] : twn[e - M];
    __syncthreads();
    const int r0 = blockIdx.x * group;
    const int nr = min(group, nrows - r0);
    for (int e = threadIdx.x; e < nr * M; e += 256) {
        const int r = e / M, k = e % M;
        fill_real_inverse(buf, lay, r, X + ((size_t)j0 * d.nz + r0 + r) * d.ldx, M, d.nkx, stw + M, k);
    }
    __syncthreads();
    row_fft<double, MC, +1>(buf, nr, lay, pm, stw);
    for (int e = threadIdx.x; e < nr * M; e += 256) {
        const int r = e / M, m = e % M;
        const cpx<double> v = buf[lay.at(m, r)];
        double2* dst = reinterpret_cast<double2*>(P + ((size_t)j0 * d.nz + r0 + r) * d.nx) + m;
        *dst = make_double2(v.x, v.y);
    }
}

template <int MC>
__global__ void __launch_bounds__(256) k_xfwd(Dims d, const double* __restrict__ P,
                                              cpx<double>* __restrict__ X, int j0, int nrows, int group,
                                              FftPlan pm, const cpx<double>* __restrict__ twm,
                                              const cpx<double>* __restrict__ twn) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int M = MC > 0 ? MC : d.nx / 2;
    using Lay = typename std::conditional<(MC > 0), RowLayoutCT<MC>, RowLayoutRT>::type;
    Lay lay;
    if constexpr (MC == 0) lay.pitch = row_pitch(M);
    cpx<double>* stw = reinterpret_cast<cpx<double>*>(smem_raw);
    cpx<double>* buf = stw + 3 * M;
    for (int e = threadIdx.x; e < 3 * M; e += 256) stw[e] = e < M ? twm[e] : twn[e - M];
    const int r0 = blockIdx.x * group;
    const int nr = min(group, nrows - r0);
    for (int e = threadIdx.x; e < nr * M; e += 256) {
        const int r = e / M, m = e % M;
        const double2 v = reinterpret_cast<const double2*>(P + ((size_t)j0 * d.nz + r0 + r) * d.nx)[m];
        buf[lay.at(m, r)] = mk<double>(v.x, v.y);
    }
    __syncthreads();
    row_fft<double, MC, -1>(buf, nr, lay, pm, stw);
    for (int e = threadIdx.x; e < nr * d.ldx; e += 256) {
        const int r = e / d.ldx, k = e % d.ldx;
        X[((size_t)j0 * d.nz + r0 + r) * d.ldx + k] =
            extract_real_forward(buf, lay, r, M, d.nkx, stw + M, k, 1.0 / (double)d.nx);
    }
}

static int api_group(int nx) {
    int g = (RT_VMAX * 256) / (nx / 2);
    return g > 8 ? 8 : g;
}

static bool ct_length(int m) {
    switch (m) {
#define CASE(N) case N: return true;
        DGPU_M_LIST(CASE)
#undef CASE
        default: return false;
    }
}

template <bool INV>
static cudaError_t launch_xapi(const Dims& d, const void* src, void* dst, int j0, int nplanes, const FftPlan& pm,
                               const void* twm, const void* twn, cudaStream_t st) {
    const int M = d.nx / 2;
    const int group = ct_length(M) ? PROD_G : api_group(d.nx);
    const int nrows = nplanes * d.nz;
    if (nrows <= 0) return cudaSuccess;
    const size_t smem = sizeof(cpx<double>) * ((size_t)group * row_pitch(M) + 3 * (size_t)M);
    auto go = [&](auto kern) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if constexpr (INV)
            kern<<<(nrows + group - 1) / group, 256, smem, st>>>(d, (const cpx<double>*)src, (double*)dst, j0, nrows,
                                                                group, pm, (const cpx<double>*)twm,
                                                                (const cpx<double>*)twn);
        else
            kern<<<(nrows + group - 1) / group, 256, smem, st>>>(d, (const double*)src, (cpx<double>*)dst, j0, nrows,
                                                                group, pm, (const cpx<double>*)twm,
                                                                (const cpx<double>*)twn);
    };
    switch (M) {
#define CASE(N) case N: if constexpr (INV) go(k_xinv<N>); else go(k_xfwd<N>); break;
        DGPU_M_LIST(CASE)
#undef CASE
        default: if constexpr (INV) go(k_xinv<0>); else go(k_xfwd<0>); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_xinv(const Dims& d, const void* X, double* P, int j0, int nplanes, const FftPlan& pm,
                        const void* twm, const void* twn, cudaStream_t st) {
    return launch_xapi<true>(d, X, P, j0, nplanes, pm, twm, twn, st);
}

cudaError_t launch_xfwd(const Dims& d, const double* P, void* X, int j0, int nplanes, const FftPlan& pm,
                        const void* twm, const void* twn, cudaStream_t st) {
    return launch_xapi<false>(d, P, X, j0, nplanes, pm, twm, twn, st);
}

template <int NC, int TX>
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
    col_fft<double, NC, TX, -1>(buf, pz, twz);
    const double inv_nz = 1.0 / (double)nz;
    double2* dst = S + (size_t)J * d.splane() + kx0;
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
    dim3 grid(d.ldx / TX, nplanes);
    auto go = [&](auto kern) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<grid, 256, smem, st>>>(d, (const cpx<double>*)X, S, j0, pz, (const cpx<double>*)twz);
    };
    switch (d.nz) {
#define CASE(N) case N: go(k_zfwd_pack<N, TX>); break;
        DGPU_NZ_LIST(CASE)
#undef CASE
        default: go(k_zfwd_pack<0, TX>); break;
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// CFL reduction (courant.f:35-47): one block per physical row (J, z), J in
// 1..NY; U1, U2, U3 inverse x transforms in FP64.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void atomic_min_pos(double* addr, double v) {
    // non-negative doubles (and +inf) order like their bit patterns
    atomicMin(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

__global__ void __launch_bounds__(256) k_cfl(Dims d, const cpx<double>* __restrict__ X, size_t x_fstride,
                                             FftPlan pm, const cpx<double>* __restrict__ twm,
                                             const cpx<double>* __restrict__ twn,
                                             const double* __restrict__ dy, double cfl, double dx,
                                             double dz, double* dtmin) {
    extern __shared__ unsigned char smem_raw[];
    cpx<double>* buf = reinterpret_cast<cpx<double>*>(smem_raw);   // [3][pitch]
    __shared__ double red[256];
    const int M = d.nx / 2;
    RowLayoutRT lay{row_pitch(M)};
    const int J = 1 + blockIdx.x / d.nz;
    const int z = blockIdx.x % d.nz;
    const size_t row = ((size_t)J * d.nz + z) * d.ldx;
    for (int e = threadIdx.x; e < 3 * M; e += blockDim.x) {
        const int f = e / M, k = e % M;
        fill_real_inverse(buf, lay, f, X + f * x_fstride + row, M, d.nkx, twn, k);
    }
    __syncthreads();
    smem_fft<double, RT_VMAX>(buf, 3, lay, pm, twm, +1);
    double m = __longlong_as_double(0x7ff0000000000000LL);   // +inf
    const double dyj = dy[J];
    for (int x = threadIdx.x; x < d.nx; x += blockDim.x) {
        const cpx<double> a = buf[lay.at(x >> 1, 0)], b = buf[lay.at(x >> 1, 1)], c = buf[lay.at(x >> 1, 2)];
        const double u1 = (x & 1) ? a.y : a.x, u2 = (x & 1) ? b.y : b.x, u3 = (x & 1) ? c.y : c.x;
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

cudaError_t launch_cfl(const Dims& d, const void* X, size_t x_fstride, const FftPlan& pm, const void* twm,
                       const void* twn, const double* dy, double cfl, double dx, double dz, double* dtmin,
                       cudaStream_t st) {
    const size_t smem = sizeof(cpx<double>) * 3 * (size_t)row_pitch(d.nx / 2);
    cudaFuncSetAttribute(k_cfl, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_cfl<<<d.ny * d.nz, 256, smem, st>>>(d, (const cpx<double>*)X, x_fstride, pm, (const cpx<double>*)twm,
                                         (const cpx<double>*)twn, dy, cfl, dx, dz, dtmin);
    return cudaGetLastError();
}

// explicit instantiations
template cudaError_t launch_zinv<float>(const Dims&, const double2*, size_t, void*, size_t, int, int, int,
                                        const FftPlan&, const void*, cudaStream_t, int);
template cudaError_t launch_zinv<double>(const Dims&, const double2*, size_t, void*, size_t, int, int, int,
                                         const FftPlan&, const void*, cudaStream_t, int);
template cudaError_t launch_products<float>(const Dims&, const void*, void*, int, int, int, const double*,
                                            const double*, const double*, const FftPlan&, const void*, const void*,
                                            cudaStream_t, const double2*, size_t);
template cudaError_t launch_products<double>(const Dims&, const void*, void*, int, int, int, const double*,
                                             const double*, const double*, const FftPlan&, const void*, const void*,
                                             cudaStream_t, const double2*, size_t);
template cudaError_t launch_zfwd_nl<float>(const Dims&, const void*, void*, int, int, int, const double*,
                                           const double*, const FftPlan&, const void*, cudaStream_t);
template cudaError_t launch_zfwd_nl<double>(const Dims&, const void*, void*, int, int, int, const double*,
                                            const double*, const FftPlan&, const void*, cudaStream_t);

}  // namespace dgpu
