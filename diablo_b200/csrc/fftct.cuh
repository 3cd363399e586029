// fftct.cuh -- compile-time-length FFTs in shared memory.
//
// Same self-sorting Stockham formulation as fft.cuh (stage radix R, Ns the
// product of the radices already applied; butterfly j reads x[j + r n/R],
// twiddles by exp(s 2 pi i (j mod Ns) r/(Ns R)), writes
// y[(j/Ns) Ns R + j mod Ns + r Ns]), but the length, every radix, the sign
// and the thread mapping are template constants, so all index arithmetic
// folds into shifts and constant multiplies and the radix-R DFTs are
// straight-line code.  Radices: 16, 8, 6, 5, 4, 3, 2 (largest first).
//
// The buffer layouts (ColLayout, RowLayoutCT, RowLayoutRT) are those of
// fft.cuh.
#pragma once

#include "fft.cuh"

namespace dgpu {

// First radix applied to a remaining length n; RMAX caps it (a radix-16
// stage holds 16 values per butterfly, which costs registers when a thread
// owns several butterflies).
__host__ __device__ constexpr int ct_radix(int n, int rmax) {
    return (rmax >= 16 && n % 16 == 0) ? 16 : n % 8 == 0 ? 8 : n % 6 == 0 ? 6 : n % 4 == 0 ? 4
         : n % 5 == 0 ? 5 : n % 3 == 0 ? 3 : 2;
}

// cos / sin of 2 pi m / 16
__host__ __device__ constexpr double cos16(int m) {
    constexpr double c1 = 0.92387953251128675613, s1 = 0.38268343236508977173, r2 = 0.70710678118654752440;
    const double t[16] = {1, c1, r2, s1, 0, -s1, -r2, -c1, -1, -c1, -r2, -s1, 0, s1, r2, c1};
    return t[m & 15];
}
__host__ __device__ constexpr double sin16(int m) { return cos16(m - 4); }

template <typename T, int S>
__device__ __forceinline__ cpx<T> muli_c(cpx<T> a) {   // a * (S i)
    if constexpr (S > 0) return mk<T>(-a.y, a.x);
    else return mk<T>(a.y, -a.x);
}

template <typename T, int S, int M>
__device__ __forceinline__ cpx<T> w16mul(cpx<T> a) {   // a * exp(S 2 pi i M/16)
    constexpr int m = M & 15;
    if constexpr (m == 0) return a;
    else if constexpr (m == 4) return muli_c<T, S>(a);
    else if constexpr (m == 8) return mk<T>(-a.x, -a.y);
    else if constexpr (m == 12) return muli_c<T, -S>(a);
    else {
        constexpr T c = (T)cos16(m), s = (T)(S * sin16(m));
        return mk<T>(a.x * c - a.y * s, a.x * s + a.y * c);
    }
}

template <typename T, int S>
__device__ __forceinline__ void ct_dft2(cpx<T>* a) {
    const cpx<T> t = a[0];
    a[0] = t + a[1];
    a[1] = t - a[1];
}
template <typename T, int S>
__device__ __forceinline__ void ct_dft3(cpx<T>* a) {
    const T h = T(0.86602540378443864676);
    const cpx<T> t = a[1] + a[2];
    const cpx<T> u = muli_c<T, S>(a[1] - a[2]) * h;
    const cpx<T> b = a[0] - t * T(0.5);
    a[0] = a[0] + t;
    a[1] = b + u;
    a[2] = b - u;
}
template <typename T, int S>
__device__ __forceinline__ void ct_dft4(cpx<T>* a) {
    const cpx<T> t0 = a[0] + a[2], t1 = a[0] - a[2];
    const cpx<T> t2 = a[1] + a[3], t3 = muli_c<T, S>(a[1] - a[3]);
    a[0] = t0 + t2;
    a[2] = t0 - t2;
    a[1] = t1 + t3;
    a[3] = t1 - t3;
}
template <typename T, int S>
__device__ __forceinline__ void ct_dft5(cpx<T>* a) {
    dft5<T>(a, S);
}
template <typename T, int S>
__device__ __forceinline__ void ct_dft6(cpx<T>* a) {
    cpx<T> e[3] = {a[0], a[2], a[4]};
    cpx<T> o[3] = {a[1], a[3], a[5]};
    ct_dft3<T, S>(e);
    ct_dft3<T, S>(o);
    const T h = T(0.86602540378443864676);
    // w = exp(S i pi/3) = 1/2 + S i sqrt(3)/2, w^2 = -1/2 + S i sqrt(3)/2
    const cpx<T> o1 = mk<T>(T(0.5) * o[1].x - T(S) * h * o[1].y, T(0.5) * o[1].y + T(S) * h * o[1].x);
    const cpx<T> o2 = mk<T>(-T(0.5) * o[2].x - T(S) * h * o[2].y, -T(0.5) * o[2].y + T(S) * h * o[2].x);
    a[0] = e[0] + o[0];
    a[3] = e[0] - o[0];
    a[1] = e[1] + o1;
    a[4] = e[1] - o1;
    a[2] = e[2] + o2;
    a[5] = e[2] - o2;
}
template <typename T, int S>
__device__ __forceinline__ void ct_dft8(cpx<T>* a) {
    cpx<T> e[4] = {a[0], a[2], a[4], a[6]};
    cpx<T> o[4] = {a[1], a[3], a[5], a[7]};
    ct_dft4<T, S>(e);
    ct_dft4<T, S>(o);
    const cpx<T> w1 = w16mul<T, S, 2>(o[1]);
    const cpx<T> w2 = w16mul<T, S, 4>(o[2]);
    const cpx<T> w3 = w16mul<T, S, 6>(o[3]);
    a[0] = e[0] + o[0];
    a[4] = e[0] - o[0];
    a[1] = e[1] + w1;
    a[5] = e[1] - w1;
    a[2] = e[2] + w2;
    a[6] = e[2] - w2;
    a[3] = e[3] + w3;
    a[7] = e[3] - w3;
}
// 16 = 4 x 4: four DFT4 over q (stride 4), twiddles W16^(q k1), four DFT4.
template <typename T, int S>
__device__ __forceinline__ void ct_dft16(cpx<T>* a) {
    cpx<T> e[4][4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        e[q][0] = a[q];
        e[q][1] = a[q + 4];
        e[q][2] = a[q + 8];
        e[q][3] = a[q + 12];
        ct_dft4<T, S>(e[q]);
    }
    cpx<T> t[4];
    // k1 = 0
    t[0] = e[0][0]; t[1] = e[1][0]; t[2] = e[2][0]; t[3] = e[3][0];
    ct_dft4<T, S>(t);
    a[0] = t[0]; a[4] = t[1]; a[8] = t[2]; a[12] = t[3];
    // k1 = 1
    t[0] = e[0][1]; t[1] = w16mul<T, S, 1>(e[1][1]); t[2] = w16mul<T, S, 2>(e[2][1]); t[3] = w16mul<T, S, 3>(e[3][1]);
    ct_dft4<T, S>(t);
    a[1] = t[0]; a[5] = t[1]; a[9] = t[2]; a[13] = t[3];
    // k1 = 2
    t[0] = e[0][2]; t[1] = w16mul<T, S, 2>(e[1][2]); t[2] = w16mul<T, S, 4>(e[2][2]); t[3] = w16mul<T, S, 6>(e[3][2]);
    ct_dft4<T, S>(t);
    a[2] = t[0]; a[6] = t[1]; a[10] = t[2]; a[14] = t[3];
    // k1 = 3
    t[0] = e[0][3]; t[1] = w16mul<T, S, 3>(e[1][3]); t[2] = w16mul<T, S, 6>(e[2][3]); t[3] = w16mul<T, S, 9>(e[3][3]);
    ct_dft4<T, S>(t);
    a[3] = t[0]; a[7] = t[1]; a[11] = t[2]; a[15] = t[3];
}

template <typename T, int R, int S>
__device__ __forceinline__ void ct_dft(cpx<T>* a) {
    if constexpr (R == 2) ct_dft2<T, S>(a);
    else if constexpr (R == 3) ct_dft3<T, S>(a);
    else if constexpr (R == 4) ct_dft4<T, S>(a);
    else if constexpr (R == 5) ct_dft5<T, S>(a);
    else if constexpr (R == 6) ct_dft6<T, S>(a);
    else if constexpr (R == 8) ct_dft8<T, S>(a);
    else ct_dft16<T, S>(a);
}

// One Stockham stage.  nbatch <= MAXB transforms; NTHR threads.
template <typename T, int N, int R, int NS, int S, class L, int MAXB, int NTHR>
__device__ __forceinline__ void ct_stage(cpx<T>* buf, int nbatch, const L& lay, const cpx<T>* __restrict__ tw) {
    constexpr int NR = N / R;
    constexpr int QMAX = (NR * MAXB + NTHR - 1) / NTHR;
    constexpr int TSTEP = N / (NS * R);
    const int nb = NR * nbatch;
    cpx<T> v[QMAX][R];
#pragma unroll
    for (int q = 0; q < QMAX; ++q) {
        const int b = threadIdx.x + q * NTHR;
        if (b < nb) {
            int j, col;
            if constexpr (L::kRowMajor) { j = b % NR; col = b / NR; }
            else { col = b % MAXB; j = b / MAXB; }
#pragma unroll
            for (int r = 0; r < R; ++r) v[q][r] = buf[lay.at(j + r * NR, col)];
            if constexpr (NS > 1) {
                const int m = (j % NS) * TSTEP;
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    cpx<T> w = tw[m * r];
                    if constexpr (S > 0) w = conjg(w);
                    v[q][r] = cmul(v[q][r], w);
                }
            }
            ct_dft<T, R, S>(v[q]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < QMAX; ++q) {
        const int b = threadIdx.x + q * NTHR;
        if (b < nb) {
            int j, col;
            if constexpr (L::kRowMajor) { j = b % NR; col = b / NR; }
            else { col = b % MAXB; j = b / MAXB; }
            const int idxD = (j / NS) * NS * R + (j % NS);
#pragma unroll
            for (int r = 0; r < R; ++r) buf[lay.at(idxD + r * NS, col)] = v[q][r];
        }
    }
    __syncthreads();
}

template <typename T, int N, int NS, int S, class L, int MAXB, int NTHR, int RMAX>
__device__ __forceinline__ void ct_stages(cpx<T>* buf, int nbatch, const L& lay, const cpx<T>* __restrict__ tw) {
    if constexpr (NS < N) {
        constexpr int R = ct_radix(N / NS, RMAX);
        ct_stage<T, N, R, NS, S, L, MAXB, NTHR>(buf, nbatch, lay, tw);
        ct_stages<T, N, NS * R, S, L, MAXB, NTHR, RMAX>(buf, nbatch, lay, tw);
    }
}

// Transform every batch member (the caller synchronised after filling
// buf); ends synchronised.  tw[m] = exp(-2 pi i m / N).
template <typename T, int N, int S, class L, int MAXB, int NTHR, int RMAX = 16>
__device__ __forceinline__ void fft_ct(cpx<T>* buf, int nbatch, const L& lay, const cpx<T>* __restrict__ tw) {
    ct_stages<T, N, 1, S, L, MAXB, NTHR, RMAX>(buf, nbatch, lay, tw);
}

}  // namespace dgpu
