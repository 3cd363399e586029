// products_hw.cu -- the physical-space products of one RK_CHAN_1 substage
// for NX = 512 in FP32 (channel.f:410-571, 670-720 with the x transforms of
// FFT_XZ_TO_PHYSICAL / _FOURIER, mpi.f:1493-1508, 1589-1604).
//
// One block per z-row, marching over a chunk of y-planes with a ring of the
// last four physical planes in shared memory.  Every half-warp owns one
// 256-point complex transform per plane:
//   * the inverse half-warps (one per field) take the field's x spectrum of
//     plane J (staged by cp.async one plane ahead) back to physical space --
//     a real transform of length 512 as one complex transform of length 256
//     -- into the ring;
//   * at the same time the product half-warps (one per product) form their
//     product of plane J-2 from ring planes J-3..J-1, transform it forward
//     and extract its x spectrum (1/NX, kx <= NKX); the two halves of a warp
//     hold the two products of one output ikx Pa + Pflux and combine them by
//     a shuffle, as K2 of transforms.cu writes its outputs.
// One block barrier per plane guards the ring.
//
// The 256-point transform of a half-warp: lane a holds the 16 points
// m = a + 16 b; a 16-point DFT in registers over b, the twiddles
// W256^(ac), one transpose through shared memory (XOR-swizzled, conflict
// free) and a second 16-point DFT give Z(c + 16 d) in lane c.  The inverse
// runs the same steps with the opposite sign from that layout back to the
// first one, so a lane forms its products from the physical points it holds
// after the inverse transform and feeds them to the forward transform with
// no reshuffle.
//
// Fields are carried as fluctuations about their plane means (the (0,0)
// mode, left out by K1 and kept FP64 in the state); each product is formed
// without its mean x mean part, which the column kernel adds to the (0,0)
// mode in FP64.
#include <cuda_runtime.h>
#include <stdint.h>

#include "fftct.cuh"
#include "kernels.cuh"
#include "launch.h"

namespace dgpu {

namespace {

constexpr int HM = 256;          // complex transform length (NX/2)
constexpr int HRING = 4;         // physical planes held
constexpr int HD = 11;           // output rows of 16 spectral entries: ldx = 176 for NKX = 170

using c32 = cpx<float>;

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// 256-point DFT with exponent sign S of the 16 values of each lane of a
// half-warp.  In: v[r] = x(lane + 16 r).  Out: v[r] = X(lane + 16 r) with the
// roles of the two index digits exchanged: the forward transform maps "lane
// a holds m = a + 16 b" to "lane c holds k = c + 16 d" and the inverse maps
// back.  tw[r*16 + lane] = W256^(r lane) (symmetric in r and lane).  The
// transpose stores element (row r, column lane) at r*16 + (lane ^ r).
template <int S>
__device__ __forceinline__ void fft256(c32 (&v)[16], c32* tb, const c32* __restrict__ tw, int lane,
                                       unsigned mask) {
    ct_dft16<float, S>(v);
#pragma unroll
    for (int r = 0; r < 16; ++r) {
        c32 w = tw[r * 16 + lane];
        if constexpr (S > 0) w = conjg(w);
        v[r] = cmul(v[r], w);
    }
#pragma unroll
    for (int r = 0; r < 16; ++r) tb[r * 16 + (lane ^ r)] = v[r];
    __syncwarp(mask);
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = tb[lane * 16 + (r ^ lane)];
    __syncwarp(mask);
    ct_dft16<float, S>(v);
}

// x spectrum of a real row from the forward transform Z (v[d] = Z(c + 16 d)
// in lane c): X_k = (E_k + W512^k O_k)/NX with E, O the even and odd parts
// (Z_k and conj Z_{256-k}), zero beyond NKX.  Z passes through tb.
__device__ __forceinline__ void extract(const c32 (&v)[16], c32 (&out)[HD], c32* tb, const c32* __restrict__ twn,
                                        int lane, unsigned mask, int nkx, float inv_nx) {
#pragma unroll
    for (int d = 0; d < 16; ++d) tb[lane + 16 * d] = v[d];
    __syncwarp(mask);
    const float hs = 0.5f * inv_nx;
#pragma unroll
    for (int d = 0; d < HD; ++d) {
        const int k = lane + 16 * d;
        const c32 zk = v[d];
        const c32 zm = tb[(HM - k) & (HM - 1)];
        const c32 E = mk<float>(zk.x + zm.x, zk.y - zm.y);
        const c32 O = mk<float>(zk.y + zm.y, zm.x - zk.x);
        const c32 X = (E + cmul(twn[k], O)) * hs;
        out[d] = k <= nkx ? X : mk<float>(0.f, 0.f);
    }
    __syncwarp(mask);
}

// Warps of a block: (nf+1)/2 inverse warps (half-warp = field), then the
// product warps.  Product warp pw, half h -> product id (channel.f order:
// P0 U1U3, P1 U1U1, P2 U3U3, P3 (U1 at GY) U2, P4 (U3 at GY) U2, P5..P7 the
// y-fluxes of U1U2, U3U2, U2U2, P(8+3n) TH_n U1, P(9+3n) TH_n U3, P(10+3n)
// the y-flux of TH_n U2) and what its half writes:
//   pw 0: P1 | P5 -> out 0 = ikx P1 + P5
//   pw 1: P3 | P7 -> out 2 = ikx P3 + P7
//   pw 2: P0 | P6 -> out 4 = ikx P0 + P6, and out 1 = P0 (half 0)
//   pw 3: P2 -> out 5 | P4 -> out 3
//   pw 4+n: P(8+3n) | P(10+3n) -> out 6+2n = ikx P8 + P10
//   pw 4+nth+i: P(9+3n) -> out 7+2n for n = 2i (half 0), 2i+1 (half 1)
__host__ __device__ __forceinline__ int product_warps(int nth) { return 4 + nth + (nth + 1) / 2; }
__host__ __device__ __forceinline__ int block_warps(int nf) { return (nf + 1) / 2 + product_warps(nf - 3); }

struct Role {
    int prod;     // product id, -1: none
    int pair;     // 1: combine with the other half into out `pairq`
    int pairq;
    int single;   // output written from this half's spectrum alone, -1: none
};
__device__ __forceinline__ Role product_role(int pw, int h, int nth) {
    Role r{-1, 0, -1, -1};
    if (pw == 0) { r.prod = h ? 5 : 1; r.pair = 1; r.pairq = 0; }
    else if (pw == 1) { r.prod = h ? 7 : 3; r.pair = 1; r.pairq = 2; }
    else if (pw == 2) { r.prod = h ? 6 : 0; r.pair = 1; r.pairq = 4; r.single = h ? -1 : 1; }
    else if (pw == 3) { r.prod = h ? 4 : 2; r.single = h ? 3 : 5; }
    else if (pw < 4 + nth) { const int n = pw - 4; r.prod = h ? 10 + 3 * n : 8 + 3 * n; r.pair = 1; r.pairq = 6 + 2 * n; }
    else {
        const int n = 2 * (pw - 4 - nth) + h;
        if (n < nth) { r.prod = 9 + 3 * n; r.single = 7 + 2 * n; }
    }
    return r;
}

__device__ __forceinline__ void products_hw_body(const Dims& d, const c32* __restrict__ X, c32* __restrict__ Y, int jlo,
                                                 int jhi, int chunk, const double* __restrict__ dy,
                                                 const double* __restrict__ dyf, const double* __restrict__ kxw,
                                                 const c32* __restrict__ twm, const c32* __restrict__ twn,
                                                 const double2* __restrict__ means, size_t means_fs, uint3 bid) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ float smean[HRING][MAXF];
    const int nf = d.nf, nth = d.nth, ldx = d.ldx;
    const int tid = threadIdx.x, lane = tid & 15, h = (tid >> 4) & 1, w = tid >> 5;
    const unsigned mask = 0xffffu << (16 * h);
    const int ninv = (nf + 1) / 2;
    const bool inv = w < ninv;
    const int f = 2 * w + h;                                   // field of an inverse half-warp
    const bool inv_active = inv && f < nf;
    const Role role = inv ? Role{-1, 0, -1, -1} : product_role(w - ninv, h, nth);
    c32* ring = reinterpret_cast<c32*>(smem_raw);               // [HRING][nf][16 b][16 a]
    c32* stw = ring + (size_t)HRING * nf * HM;                  // W256^(rc) at [r*16 + c]
    c32* stn = stw + HM;                                        // W512^k, k < 256
    c32* tb = stn + HM + (size_t)(2 * w + h) * HM;              // transpose / extraction buffer
    c32* stg = stn + HM + (size_t)2 * blockDim.x / 32 * HM + (size_t)(inv_active ? f : 0) * ldx;
    for (int e = tid; e < HM; e += blockDim.x) {
        stw[e] = twm[((e & 15) * (e >> 4)) & (HM - 1)];
        stn[e] = twn[e];
    }
    const int z = bid.x;
    const int jb = jlo + bid.y * chunk;
    const int je = min(jb + chunk - 1, jhi);
    if (jb > jhi) return;                          // batched form: past this instance's planes
    const size_t xrow = (size_t)d.nz * ldx;       // plane stride of X / Y
    const size_t xf = (size_t)d.nyp * xrow;       // field stride of X / Y
    const size_t ps = d.splane();
    const int nkx = d.nkx;
    const float inv_nx = 1.0f / (float)(2 * HM);
    auto stage = [&](int J) {
        const c32* src = X + (size_t)f * xf + (size_t)J * xrow + (size_t)z * ldx;
        for (int e = lane; e < ldx / 2; e += 16) cp_async16(stg + 2 * e, src + 2 * e);
        cp_async_commit();
    };
    if (inv_active) stage(jb - 1);
    __syncthreads();                               // twiddle tables
    for (int J = jb - 1; J <= je + 2; ++J) {
        const int jp = J - 2;
        const bool do_inv = inv_active && J <= je + 1;             // field f of plane J to physical space
        const bool do_prod = !inv && jp >= jb && role.prod >= 0;   // product role.prod of plane jp
        const int s = (J - jb + 1) & (HRING - 1);
        c32 v[16];
        if (do_inv) {
            // ---- field f of plane J to physical space ---------------------------
            cp_async_wait_all();
            __syncwarp(mask);
            if (lane == 0) smean[s][f] = means ? (float)means[(size_t)f * means_fs + (size_t)J * ps].x : 0.0f;
            // Zc_k = (X_k + conj X_{M-k}) + i W512^-k (X_k - conj X_{M-k}) at
            // k = lane + 16 r; its backward 256-point transform is
            // x_{2m} + i x_{2m+1} (DC imaginary part and Nyquist dropped).  One
            // transform routine (forward sign) serves both kinds of half-warp,
            // so their code stays in the instruction cache together.
#pragma unroll
            for (int r = 0; r < 16; ++r) {
                const int k = lane + 16 * r;
                c32 xa = mk<float>(0.f, 0.f), xc = mk<float>(0.f, 0.f);
                if (k <= nkx) {
                    xa = stg[k];
                    if (k == 0) xa.y = 0.f;
                }
                const int kk = HM - k;
                if (kk <= nkx) xc = conjg(stg[kk]);
                const c32 A = xa + xc;
                const c32 B = cmul(xa - xc, conjg(stn[k]));
                v[r] = mk<float>(A.x - B.y, -(A.y + B.x));      // conjugated: the backward
                                                                 // transform as conj(forward(conj))
            }
            __syncwarp(mask);                      // the row is consumed: stage the next one
            if (J + 1 <= je + 1) stage(J + 1);
        } else if (do_prod) {
            // ---- product role.prod of plane jp from ring planes jp-1..jp+1 ----
            const int sm = (jp - jb) & (HRING - 1), s0 = (jp - jb + 1) & (HRING - 1), sp = (jp - jb + 2) & (HRING - 1);
            const c32* Rm = ring + (size_t)sm * nf * HM + lane;
            const c32* R0 = ring + (size_t)s0 * nf * HM + lane;
            const c32* Rp = ring + (size_t)sp * nf * HM + lane;
            auto fld = [&](const c32* R, int g, int r) { return R[(size_t)g * HM + r * 16]; };
            const float m1m = smean[sm][0], m1 = smean[s0][0], m1p = smean[sp][0];
            const float m2m = smean[sm][1], m2 = smean[s0][1], m2p = smean[sp][1];
            const float m3m = smean[sm][2], m3 = smean[s0][2], m3p = smean[sp][2];
            const int p = role.prod;
            // lower-case: fluctuation about the plane mean mN; each product is
            // its part beyond the mean x mean product
            if (p == 0 || p == 1 || p == 2 || p >= 8 && (p - 8) % 3 != 2) {
                // pointwise: P0 U1U3, P1 U1U1, P2 U3U3, P8 TH U1, P9 TH U3
                int ga, gb;
                float ma, mb;
                if (p == 0) { ga = 2; gb = 0; ma = m3; mb = m1; }
                else if (p == 1) { ga = 0; gb = 0; ma = m1; mb = m1; }
                else if (p == 2) { ga = 2; gb = 2; ma = m3; mb = m3; }
                else {
                    const int n = (p - 8) / 3;
                    ga = 3 + n; ma = smean[s0][3 + n];
                    if ((p - 8) % 3 == 0) { gb = 0; mb = m1; } else { gb = 2; mb = m3; }
                }
#pragma unroll
                for (int r = 0; r < 16; ++r) {
                    const c32 qa = fld(R0, ga, r), qb = fld(R0, gb, r);
                    v[r] = mk<float>(qa.x * (mb + qb.x) + ma * qb.x, qa.y * (mb + qb.y) + ma * qb.y);
                }
            } else if (p == 3 || p == 4) {
                // (U at GY) U2: (a1 U(j) + a0 U(j-1)) U2(j)
                const float a1 = (float)(dyf[jp] / (2.0 * dy[jp]));
                const float a0 = (float)(dyf[jp - 1] / (2.0 * dy[jp]));
                const int g = p == 3 ? 0 : 2;
                const float mi = p == 3 ? a1 * m1 + a0 * m1m : a1 * m3 + a0 * m3m;
#pragma unroll
                for (int r = 0; r < 16; ++r) {
                    const c32 qm = fld(Rm, g, r), q0 = fld(R0, g, r), u2 = fld(R0, 1, r);
                    auto pr = [&](float a_, float b_, float w_) { return (a1 * b_ + a0 * a_) * (m2 + w_) + mi * w_; };
                    v[r] = mk<float>(pr(qm.x, q0.x, u2.x), pr(qm.y, q0.y, u2.y));
                }
            } else if (p == 7) {
                // (U2(j) + U2(j+1))^2/4 - (U2(j) + U2(j-1))^2/4, over DY(j)
                const float idy = (float)(1.0 / dy[jp]);
                const float S1 = m2 + m2p, S2 = m2 + m2m;
#pragma unroll
                for (int r = 0; r < 16; ++r) {
                    const c32 wm = fld(Rm, 1, r), w0 = fld(R0, 1, r), wp = fld(Rp, 1, r);
                    auto pr = [&](float a_, float b_, float c_) {
                        const float s1 = b_ + c_, s2 = b_ + a_;
                        return 0.25f * (s1 * (s1 + 2.f * S1) - s2 * (s2 + 2.f * S2)) * idy;
                    };
                    v[r] = mk<float>(pr(wm.x, w0.x, wp.x), pr(wm.y, w0.y, wp.y));
                }
            } else {
                // y-flux: (Q(j+1) + Q(j)) U2(j+1) - (Q(j) + Q(j-1)) U2(j), over 2 DYF(j),
                // Q = U1 (P5), U3 (P6), TH_n (P(10+3n))
                const float i2dyf = (float)(1.0 / (2.0 * dyf[jp]));
                int g;
                float qmm, qm0, qmp;
                if (p == 5) { g = 0; qmm = m1m; qm0 = m1; qmp = m1p; }
                else if (p == 6) { g = 2; qmm = m3m; qm0 = m3; qmp = m3p; }
                else {
                    g = 3 + (p - 10) / 3;
                    qmm = smean[sm][g]; qm0 = smean[s0][g]; qmp = smean[sp][g];
                }
#pragma unroll
                for (int r = 0; r < 16; ++r) {
                    const c32 qm = fld(Rm, g, r), q0 = fld(R0, g, r), qp = fld(Rp, g, r);
                    const c32 u2 = fld(R0, 1, r), u2p = fld(Rp, 1, r);
                    auto flux = [&](float a_, float b_, float c_, float w0, float wp) {
                        return ((c_ + b_) * (m2p + wp) + (qmp + qm0) * wp - (b_ + a_) * (m2 + w0) - (qm0 + qmm) * w0) *
                               i2dyf;
                    };
                    v[r] = mk<float>(flux(qm.x, q0.x, qp.x, u2.x, u2p.x), flux(qm.y, q0.y, qp.y, u2.y, u2p.y));
                }
            }
        }
        if (do_inv || do_prod) fft256<-1>(v, tb, stw, lane, mask);
        if (do_inv) {
            c32* dst = ring + ((size_t)s * nf + f) * HM + lane;
#pragma unroll
            for (int r = 0; r < 16; ++r) dst[r * 16] = conjg(v[r]);
        } else if (do_prod) {
            c32 o[HD];
            extract(v, o, tb, stn, lane, mask, nkx, inv_nx);
            c32* yrow = Y + (size_t)jp * xrow + (size_t)z * ldx + lane;
            if (role.single >= 0) {
                c32* yq = yrow + (size_t)role.single * xf;
#pragma unroll
                for (int dd = 0; dd < HD; ++dd) yq[16 * dd] = o[dd];
            }
            if (role.pair) {
                // half 0 holds Pa, half 1 Pflux: out = ikx Pa + Pflux, the rows
                // split between the halves
                c32* yq = yrow + (size_t)role.pairq * xf;
#pragma unroll
                for (int dd = 0; dd < HD; ++dd) {
                    const c32 other = mk<float>(__shfl_xor_sync(0xffffffffu, o[dd].x, 16),
                                                __shfl_xor_sync(0xffffffffu, o[dd].y, 16));
                    const c32 xa = h ? other : o[dd], xfl = h ? o[dd] : other;
                    const float K = (float)kxw[lane + 16 * dd];
                    const c32 val = mk<float>(-K * xa.y + xfl.x, K * xa.x + xfl.y);
                    if ((dd < (HD + 1) / 2) == (h == 0)) yq[16 * dd] = val;
                }
            }
        }
        __syncthreads();                           // the next plane overwrites the ring slot of J-3
    }
}

template <int NW>
__global__ void __launch_bounds__(32 * NW, NW <= 8 ? 3 : 1)
k_products_hw(Dims d, const c32* __restrict__ X, c32* __restrict__ Y, int jlo, int jhi, int chunk,
              const double* __restrict__ dy, const double* __restrict__ dyf, const double* __restrict__ kxw,
              const c32* __restrict__ twm, const c32* __restrict__ twn, const double2* __restrict__ means,
              size_t means_fs) {
    products_hw_body(d, X, Y, jlo, jhi, chunk, dy, dyf, kxw, twm, twn, means, means_fs, blockIdx);
}

// Batched form: instance blockIdx.z of a group of equal shape.
template <int NW>
__global__ void __launch_bounds__(32 * NW, NW <= 8 ? 3 : 1)
k_products_hw_b(const InstPtrs* __restrict__ ip, Dims d, int jhi, int chunk, const c32* __restrict__ twm,
                const c32* __restrict__ twn, size_t means_fs) {
    const InstPtrs q = ip[blockIdx.z];
    products_hw_body(d, reinterpret_cast<const c32*>(q.xb), reinterpret_cast<c32*>(q.yb), q.jlo_prod, jhi, chunk, q.dy,
                     q.dyf, q.kx, twm, twn, q.cu, means_fs, make_uint3(blockIdx.x, blockIdx.y, 0));
}

}  // namespace

bool products_hw_supported(const Dims& d) { return d.nx == 2 * HM && d.ldx == 16 * HD && d.nf <= MAXF; }

size_t products_hw_smem(const Dims& d) {
    return sizeof(c32) * ((size_t)HRING * d.nf * HM + 2 * HM + (size_t)2 * block_warps(d.nf) * HM +
                          (size_t)d.nf * d.ldx);
}

cudaError_t launch_products_hw(const Dims& d, const void* X, void* Y, int jlo, int jhi, int chunk, const double* dy,
                               const double* dyf, const double* kx, const void* twm, const void* twn, cudaStream_t st,
                               const double2* means, size_t means_fstride) {
    if (jhi < jlo) return cudaSuccess;
    if (!products_hw_supported(d)) return cudaErrorInvalidValue;
    const size_t smem = products_hw_smem(d);
    const int nchunks = (jhi - jlo + chunk) / chunk;
    dim3 grid(d.nz, nchunks);
    const int nw = block_warps(d.nf);
    auto go = [&](auto kern) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kern<<<grid, 32 * nw, smem, st>>>(d, (const c32*)X, (c32*)Y, jlo, jhi, chunk, dy, dyf, kx, (const c32*)twm,
                                          (const c32*)twn, means, means_fstride);
        return cudaGetLastError();
    };
    return nw <= 8 ? go(k_products_hw<8>) : go(k_products_hw<14>);
}

cudaError_t launch_products_hw_b(const Dims& d, const InstPtrs* ip, int ninst, int jlo_min, int jhi, int chunk,
                                 const void* twm, const void* twn, cudaStream_t st, size_t means_fstride) {
    if (jhi < jlo_min) return cudaSuccess;
    if (!products_hw_supported(d)) return cudaErrorInvalidValue;
    const size_t smem = products_hw_smem(d);
    dim3 grid(d.nz, (jhi - jlo_min + chunk) / chunk, ninst);
    const int nw = block_warps(d.nf);
    auto go = [&](auto kern) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kern<<<grid, 32 * nw, smem, st>>>(ip, d, jhi, chunk, (const c32*)twm, (const c32*)twn, means_fstride);
        return cudaGetLastError();
    };
    return nw <= 8 ? go(k_products_hw_b<8>) : go(k_products_hw_b<14>);
}

}  // namespace dgpu
