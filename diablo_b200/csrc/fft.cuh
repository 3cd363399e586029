// fft.cuh -- batched mixed-radix (2,3,4,5,8) FFTs in shared memory.
//
// Replaces the FFTW 3.3.10 plans of INIT_FFT (for/fft.f:73-89): complex DFTs
// X_k = sum_j x_j exp(s 2 pi i jk/n), s = -1 forward, s = +1 backward, both
// unnormalised.  The transform is a self-sorting Stockham formulation: at a
// stage of radix R, with Ns the product of the radices already applied,
// butterfly j reads x[j + r n/R] (r < R), multiplies by exp(s 2 pi i (j mod
// Ns) r / (Ns R)), does an R-point DFT in registers and writes
// y[(j/Ns) Ns R + (j mod Ns) + r Ns].  Every thread first loads and computes
// all of its butterflies, the block synchronises, then all results are
// stored, so one shared buffer serves as both input and output.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace dgpu {

template <typename T>
struct __align__(2 * sizeof(T)) cpx {
    T x, y;
};

template <typename T>
__host__ __device__ __forceinline__ cpx<T> mk(T a, T b) {
    cpx<T> r;
    r.x = a;
    r.y = b;
    return r;
}
template <typename T>
__device__ __forceinline__ cpx<T> operator+(cpx<T> a, cpx<T> b) { return mk(a.x + b.x, a.y + b.y); }
template <typename T>
__device__ __forceinline__ cpx<T> operator-(cpx<T> a, cpx<T> b) { return mk(a.x - b.x, a.y - b.y); }
template <typename T>
__device__ __forceinline__ cpx<T> operator*(cpx<T> a, T s) { return mk(a.x * s, a.y * s); }
template <typename T>
__device__ __forceinline__ cpx<T> cmul(cpx<T> a, cpx<T> b) {
    return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T>
__device__ __forceinline__ cpx<T> conjg(cpx<T> a) { return mk(a.x, -a.y); }
// a * (s i) for s = +-1
template <typename T>
__device__ __forceinline__ cpx<T> muli(cpx<T> a, int s) { return s > 0 ? mk(-a.y, a.x) : mk(a.y, -a.x); }

// Factorisation of a transform length; radices are applied in order.
struct FftPlan {
    int n;
    int nst;
    int rad[16];
};

// ---- small DFTs in registers (sign s: exponent exp(s 2 pi i pq / R)) --------
template <typename T>
__device__ __forceinline__ void dft2(cpx<T>* a, int) {
    cpx<T> t = a[0];
    a[0] = t + a[1];
    a[1] = t - a[1];
}

template <typename T>
__device__ __forceinline__ void dft3(cpx<T>* a, int s) {
    const T h = T(0.86602540378443864676);   // sqrt(3)/2
    cpx<T> t = a[1] + a[2];
    cpx<T> u = muli(a[1] - a[2], s) * h;
    cpx<T> b = a[0] - t * T(0.5);
    a[0] = a[0] + t;
    a[1] = b + u;
    a[2] = b - u;
}

template <typename T>
__device__ __forceinline__ void dft4(cpx<T>* a, int s) {
    cpx<T> t0 = a[0] + a[2], t1 = a[0] - a[2];
    cpx<T> t2 = a[1] + a[3], t3 = muli(a[1] - a[3], s);
    a[0] = t0 + t2;
    a[2] = t0 - t2;
    a[1] = t1 + t3;
    a[3] = t1 - t3;
}

template <typename T>
__device__ __forceinline__ void dft5(cpx<T>* a, int s) {
    const T c1 = T(0.30901699437494742410);    // cos(2 pi/5)
    const T c2 = T(-0.80901699437494742410);   // cos(4 pi/5)
    const T s1 = T(0.95105651629515357212);    // sin(2 pi/5)
    const T s2 = T(0.58778525229247312917);    // sin(4 pi/5)
    cpx<T> t1 = a[1] + a[4], t2 = a[2] + a[3];
    cpx<T> t3 = a[1] - a[4], t4 = a[2] - a[3];
    cpx<T> b1 = mk(a[0].x + c1 * t1.x + c2 * t2.x, a[0].y + c1 * t1.y + c2 * t2.y);
    cpx<T> b2 = mk(a[0].x + c2 * t1.x + c1 * t2.x, a[0].y + c2 * t1.y + c1 * t2.y);
    cpx<T> d1 = muli(mk(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y), s);
    cpx<T> d2 = muli(mk(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y), s);
    a[0] = a[0] + t1 + t2;
    a[1] = b1 + d1;
    a[4] = b1 - d1;
    a[2] = b2 + d2;
    a[3] = b2 - d2;
}

template <typename T>
__device__ __forceinline__ void dft8(cpx<T>* a, int s) {
    const T c = T(0.70710678118654752440);     // sqrt(2)/2
    cpx<T> e[4] = {a[0], a[2], a[4], a[6]};
    cpx<T> o[4] = {a[1], a[3], a[5], a[7]};
    dft4(e, s);
    dft4(o, s);
    // W8^1 = c(1 + s i), W8^2 = s i, W8^3 = c(-1 + s i)
    cpx<T> w1 = (o[1] + muli(o[1], s)) * c;
    cpx<T> w2 = muli(o[2], s);
    cpx<T> w3 = (muli(o[3], s) - o[3]) * c;
    a[0] = e[0] + o[0];
    a[4] = e[0] - o[0];
    a[1] = e[1] + w1;
    a[5] = e[1] - w1;
    a[2] = e[2] + w2;
    a[6] = e[2] - w2;
    a[3] = e[3] + w3;
    a[7] = e[3] - w3;
}

template <typename T, int R>
__device__ __forceinline__ void dftR(cpx<T>* a, int s) {
    if constexpr (R == 2) dft2(a, s);
    else if constexpr (R == 3) dft3(a, s);
    else if constexpr (R == 4) dft4(a, s);
    else if constexpr (R == 5) dft5(a, s);
    else dft8(a, s);
}

// Twiddle exp(s 2 pi i m / n) from the table tw[m] = exp(-2 pi i m / n).
template <typename T>
__device__ __forceinline__ cpx<T> twid(const cpx<T>* __restrict__ tw, int m, int s) {
    cpx<T> w = tw[m];
    return s > 0 ? conjg(w) : w;
}

// Shared-memory layouts of a batch of transforms: element p of transform b.
//  ColLayout<TX>  at p*TX + b: TX transforms interleaved (consecutive
//                 threads take consecutive transforms: conflict-free).
//  RowLayoutCT<M> / RowLayoutRT  at b*pitch + p + p/16: one transform per
//                 row, with a pad word every 16 elements so that the strided
//                 Stockham writes of the early stages hit distinct banks.
template <int TX>
struct ColLayout {
    static constexpr bool kRowMajor = false;
    static constexpr int kBatch = TX;
    __device__ __forceinline__ int at(int p, int b) const { return p * TX + b; }
};

template <int M>
struct RowLayoutCT {
    static constexpr bool kRowMajor = true;
    static constexpr int PITCH = M + M / 16 + 1;
    __device__ __forceinline__ int at(int p, int b) const { return b * PITCH + p + (p >> 4); }
};

struct RowLayoutRT {
    static constexpr bool kRowMajor = true;
    int pitch;
    __device__ __forceinline__ int at(int p, int b) const { return b * pitch + p + (p >> 4); }
};

__host__ __device__ constexpr int row_pitch(int m) { return m + m / 16 + 1; }

// One Stockham stage over a batch of transforms held in shared memory, for
// a length known only at run time.  VMAX bounds the complex values a thread
// holds: n*nbatch <= VMAX*blockDim.x.
template <typename T, int R, int VMAX, class L>
__device__ __forceinline__ void stockham_stage(cpx<T>* buf, int n, int nbatch, const L& lay, int Ns,
                                               const cpx<T>* __restrict__ tw, int s) {
    constexpr int QMAX = (VMAX + R - 1) / R;
    const int nR = n / R;
    const int nb = nR * nbatch;
    const int tstep = n / (Ns * R);
    cpx<T> v[QMAX][R];
#pragma unroll
    for (int q = 0; q < QMAX; ++q) {
        const int b = threadIdx.x + q * blockDim.x;
        if (b < nb) {
            int j, col;
            if (L::kRowMajor) { j = b % nR; col = b / nR; }
            else { col = b % nbatch; j = b / nbatch; }
            const int k = j % Ns;
#pragma unroll
            for (int r = 0; r < R; ++r) v[q][r] = buf[lay.at(j + r * nR, col)];
            if (Ns > 1) {
                const int m = k * tstep;
#pragma unroll
                for (int r = 1; r < R; ++r) v[q][r] = cmul(v[q][r], twid(tw, m * r, s));
            }
            dftR<T, R>(v[q], s);
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < QMAX; ++q) {
        const int b = threadIdx.x + q * blockDim.x;
        if (b < nb) {
            int j, col;
            if (L::kRowMajor) { j = b % nR; col = b / nR; }
            else { col = b % nbatch; j = b / nbatch; }
            const int k = j % Ns;
            const int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) buf[lay.at(idxD + r * Ns, col)] = v[q][r];
        }
    }
    __syncthreads();
}

// Full transform of every batch member; callers synchronise before (data
// in place) and the routine ends synchronised.
template <typename T, int VMAX, class L>
__device__ void smem_fft(cpx<T>* buf, int nbatch, const L& lay, const FftPlan& P,
                         const cpx<T>* __restrict__ tw, int s) {
    int Ns = 1;
    for (int st = 0; st < P.nst; ++st) {
        const int R = P.rad[st];
        switch (R) {
            case 8: stockham_stage<T, 8, VMAX>(buf, P.n, nbatch, lay, Ns, tw, s); break;
            case 4: stockham_stage<T, 4, VMAX>(buf, P.n, nbatch, lay, Ns, tw, s); break;
            case 2: stockham_stage<T, 2, VMAX>(buf, P.n, nbatch, lay, Ns, tw, s); break;
            case 3: stockham_stage<T, 3, VMAX>(buf, P.n, nbatch, lay, Ns, tw, s); break;
            default: stockham_stage<T, 5, VMAX>(buf, P.n, nbatch, lay, Ns, tw, s); break;
        }
        Ns *= R;
    }
}

// Host: radix list for n (8 first, then 4, 2, 3, 5); returns false when n
// has a prime factor other than 2, 3 and 5.
inline bool make_plan(int n, FftPlan* P) {
    P->n = n;
    P->nst = 0;
    int m = n;
    const int rads[5] = {8, 4, 2, 3, 5};
    for (int q = 0; q < 5; ++q)
        while (m % rads[q] == 0 && m > 1) {
            if (P->nst >= 16) return false;
            P->rad[P->nst++] = rads[q];
            m /= rads[q];
        }
    return m == 1 && n > 1;
}

}  // namespace dgpu
