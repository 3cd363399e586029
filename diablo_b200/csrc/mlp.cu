// mlp.cu -- the learned subgrid-stress closure: an MLP from 11 features
// (the 9 resolved velocity gradients, the wall distance y+ and the filter
// width) through 3 hidden layers of 64 GELU units to the 6 stresses tau_ij.
// The reference has no such model; this is the library's own.
//
// Arithmetic: weights and activations in BF16 on the tensor cores
// (mma.sync m16n8k16, BF16 x BF16 -> FP32), accumulation, biases, GELU (tanh
// form), losses, gradients and the Adam state in FP32.  Each warp owns a tile of
// 16 samples.  Every product is a 16 x 8 x 16 tile read from shared memory
// with one of four fragment loaders, so the forward pass (H W^T), the
// backward pass (delta W) and the weight gradients (delta^T H) share them.
//
// Parameter vector (FP32, include/diablo_gpu.h order): W1[64][11] b1[64] W2[64][64]
// b2[64] W3[64][64] b3[64] W4[6][64] b4[6], then the input means [11], the
// input scales [11] and the output scales [6].  The network works on
// normalised inputs (x - mean)/scale and produces outputs / out_scale.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/diablo_gpu.h"
#include "launch.h"

namespace dgpu {
namespace {

constexpr int NIN = DIABLO_MLP_NIN, NH = DIABLO_MLP_NHIDDEN, NOUT = DIABLO_MLP_NOUT;
constexpr int K1 = 16;           // inputs padded to one k tile
constexpr int LD1 = K1 + 8;      // bf16 row stride of 16-wide rows (bank-conflict padding)
constexpr int LDW = NH + 8;      // bf16 row stride of 64-wide rows
constexpr int NW = 4;            // warps per block
constexpr int TS = 16;           // samples per warp tile

// parameter offsets (floats)
constexpr int OW1 = 0, OB1 = OW1 + NH * NIN, OW2 = OB1 + NH, OB2 = OW2 + NH * NH, OW3 = OB2 + NH, OB3 = OW3 + NH * NH,
              OW4 = OB3 + NH, OB4 = OW4 + NOUT * NH, NTRAIN = OB4 + NOUT, OMEAN = NTRAIN, OSCALE = OMEAN + NIN,
              OOUT = OSCALE + NIN, NPARAM = OOUT + NOUT;
static_assert(NTRAIN == DIABLO_MLP_NTRAIN && NPARAM == DIABLO_MLP_NPARAM, "parameter layout");

// packed BF16 weights in the shared-memory layout (padded rows)
constexpr int SW1 = 0, SW2 = SW1 + NH * LD1, SW3 = SW2 + NH * LDW, SW4 = SW3 + NH * LDW, SWN = SW4 + 16 * LDW;

__device__ __forceinline__ uint32_t pack2(uint16_t lo, uint16_t hi) { return (uint32_t)lo | ((uint32_t)hi << 16); }
__device__ __forceinline__ uint16_t bf(float v) { return __bfloat16_as_ushort(__float2bfloat16_rn(v)); }

__device__ __forceinline__ void mma(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Fragment loaders for the m16n8k16 tile at the given origin (g = lane/4,
// t = lane%4).  A is 16 x 16 (rows m, columns k), B is 16 x 8 (rows k,
// columns n).
// A[m][k] = s[m*ld + k]
__device__ __forceinline__ void lda_row(uint32_t (&a)[4], const uint16_t* s, int ld, int g, int t) {
    a[0] = *reinterpret_cast<const uint32_t*>(s + g * ld + 2 * t);
    a[1] = *reinterpret_cast<const uint32_t*>(s + (g + 8) * ld + 2 * t);
    a[2] = *reinterpret_cast<const uint32_t*>(s + g * ld + 2 * t + 8);
    a[3] = *reinterpret_cast<const uint32_t*>(s + (g + 8) * ld + 2 * t + 8);
}
// A[m][k] = s[k*ld + m]
__device__ __forceinline__ void lda_tr(uint32_t (&a)[4], const uint16_t* s, int ld, int g, int t) {
    a[0] = pack2(s[(2 * t) * ld + g], s[(2 * t + 1) * ld + g]);
    a[1] = pack2(s[(2 * t) * ld + g + 8], s[(2 * t + 1) * ld + g + 8]);
    a[2] = pack2(s[(2 * t + 8) * ld + g], s[(2 * t + 9) * ld + g]);
    a[3] = pack2(s[(2 * t + 8) * ld + g + 8], s[(2 * t + 9) * ld + g + 8]);
}
// B[k][n] = s[n*ld + k]  (a weight matrix W[out=n][in=k])
__device__ __forceinline__ void ldb_col(uint32_t (&b)[2], const uint16_t* s, int ld, int g, int t) {
    b[0] = *reinterpret_cast<const uint32_t*>(s + g * ld + 2 * t);
    b[1] = *reinterpret_cast<const uint32_t*>(s + g * ld + 2 * t + 8);
}
// B[k][n] = s[k*ld + n]
__device__ __forceinline__ void ldb_row(uint32_t (&b)[2], const uint16_t* s, int ld, int g, int t) {
    b[0] = pack2(s[(2 * t) * ld + g], s[(2 * t + 1) * ld + g]);
    b[1] = pack2(s[(2 * t + 8) * ld + g], s[(2 * t + 9) * ld + g]);
}

// GELU in its tanh form, 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))),
// with tanh u = 1 - 2 / (exp(2u) + 1) on the clamped argument (|u| <= 9,
// where tanh is 1 to FP32 precision) from the fast exponential; and its
// derivative for the backward pass.
__device__ __forceinline__ float tanh_c(float u) {
    u = fminf(fmaxf(u, -9.0f), 9.0f);
    return 1.0f - __fdividef(2.0f, __expf(2.0f * u) + 1.0f);
}
__device__ __forceinline__ float gelu(float z) {
    return 0.5f * z * (1.0f + tanh_c(0.79788456080286536f * (z + 0.044715f * z * z * z)));
}
__device__ __forceinline__ float gelu_d(float z) {
    const float t = tanh_c(0.79788456080286536f * (z + 0.044715f * z * z * z));
    return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * 0.79788456080286536f * (1.0f + 0.134145f * z * z);
}
// two floats to a packed BF16 pair (round to nearest even), low half first
__device__ __forceinline__ uint32_t bf2(float lo, float hi) {
    __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&h);
}

struct MlpDev {
    const uint16_t* wb;     // packed BF16 weights (SWN entries)
    const float* p;         // FP32 parameters (biases, normalisation)
};

// Shared memory of one block: the packed weights, the biases, and per warp
// the input tile, three hidden tiles (BF16), the pre-activations (FP32,
// training only) and two delta tiles.
struct WarpTiles {
    uint16_t* x;            // [16][LD1]
    uint16_t* h[3];         // [16][LDW]
    float* z[3];            // [16][NH] or null
};

__device__ void load_weights(const MlpDev& m, uint16_t* sw, float* sb) {
    for (int e = threadIdx.x; e < SWN / 2; e += blockDim.x)
        reinterpret_cast<uint32_t*>(sw)[e] = reinterpret_cast<const uint32_t*>(m.wb)[e];
    for (int e = threadIdx.x; e < 3 * NH + 8; e += blockDim.x) {
        float v = 0.0f;
        if (e < NH) v = m.p[OB1 + e];
        else if (e < 2 * NH) v = m.p[OB2 + e - NH];
        else if (e < 3 * NH) v = m.p[OB3 + e - 2 * NH];
        else if (e - 3 * NH < NOUT) v = m.p[OB4 + e - 3 * NH];
        sb[e] = v;
    }
}

// Normalised BF16 input tile of samples s0..s0+15 (rows past n are zero).
__device__ void load_inputs(const MlpDev& m, const float* __restrict__ x, long long n, long long s0, uint16_t* xs,
                            int lane) {
    for (int e = lane; e < TS * K1; e += 32) {
        const int r = e / K1, c = e % K1;
        float v = 0.0f;
        if (c < NIN && s0 + r < n) v = (x[(s0 + r) * NIN + c] - m.p[OMEAN + c]) / m.p[OSCALE + c];
        xs[r * LD1 + c] = bf(v);
    }
}

// Forward pass of one warp tile.  y receives the 16 x 8 output fragment
// (normalised outputs, columns >= 6 unused).
__device__ void forward_tile(const uint16_t* sw, const float* sb, const WarpTiles& w, float (&y)[4], int g, int t) {
    // layer 1: [16 x 16] x W1^T
    for (int nt = 0; nt < NH / 8; ++nt) {
        float acc[4] = {sb[nt * 8 + 2 * t], sb[nt * 8 + 2 * t + 1], sb[nt * 8 + 2 * t], sb[nt * 8 + 2 * t + 1]};
        uint32_t a[4], b[2];
        lda_row(a, w.x, LD1, g, t);
        ldb_col(b, sw + SW1 + nt * 8 * LD1, LD1, g, t);
        mma(acc, a, b);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = g + (q >> 1) * 8, c = nt * 8 + 2 * t + (q & 1);
            if (w.z[0]) w.z[0][r * NH + c] = acc[q];
            w.h[0][r * LDW + c] = bf(gelu(acc[q]));
        }
    }
    __syncwarp();
    // layers 2 and 3: [16 x 64] x W^T
    for (int l = 1; l < 3; ++l) {
        const uint16_t* W = sw + (l == 1 ? SW2 : SW3);
        const float* bias = sb + l * NH;
        for (int nt = 0; nt < NH / 8; ++nt) {
            float acc[4] = {bias[nt * 8 + 2 * t], bias[nt * 8 + 2 * t + 1], bias[nt * 8 + 2 * t],
                            bias[nt * 8 + 2 * t + 1]};
#pragma unroll
            for (int kt = 0; kt < NH / 16; ++kt) {
                uint32_t a[4], b[2];
                lda_row(a, w.h[l - 1] + kt * 16, LDW, g, t);
                ldb_col(b, W + nt * 8 * LDW + kt * 16, LDW, g, t);
                mma(acc, a, b);
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int r = g + (q >> 1) * 8, c = nt * 8 + 2 * t + (q & 1);
                if (w.z[l]) w.z[l][r * NH + c] = acc[q];
                w.h[l][r * LDW + c] = bf(gelu(acc[q]));
            }
        }
        __syncwarp();
    }
    // output layer: [16 x 64] x W4^T (8 padded outputs)
    float acc[4] = {sb[3 * NH + 2 * t], sb[3 * NH + 2 * t + 1], sb[3 * NH + 2 * t], sb[3 * NH + 2 * t + 1]};
#pragma unroll
    for (int kt = 0; kt < NH / 16; ++kt) {
        uint32_t a[4], b[2];
        lda_row(a, w.h[2] + kt * 16, LDW, g, t);
        ldb_col(b, sw + SW4 + kt * 16, LDW, g, t);
        mma(acc, a, b);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) y[q] = acc[q];
}

constexpr size_t fwd_smem() { return sizeof(uint16_t) * SWN + sizeof(float) * (3 * NH + 8); }

// Inference: activations stay in registers.  The m16n8 accumulators of n
// tiles 2kt and 2kt+1 hold exactly the m16k16 A fragment of k tile kt of the
// next layer, so a layer's GELU output is packed to BF16 in place and fed to
// the next layer's mma without touching shared memory; only the weights
// (B fragments) are read from it.  The inputs are read straight from
// global memory into the first layer's A fragment.  8 warps per block,
// grid-stride over 16-sample tiles.
constexpr int FW = 8;   // warps per inference block

__device__ __forceinline__ void gelu_pack(const float (&acc)[NH / 8][4], uint32_t (&a)[NH / 16][4]) {
#pragma unroll
    for (int kt = 0; kt < NH / 16; ++kt) {
        a[kt][0] = bf2(gelu(acc[2 * kt][0]), gelu(acc[2 * kt][1]));
        a[kt][1] = bf2(gelu(acc[2 * kt][2]), gelu(acc[2 * kt][3]));
        a[kt][2] = bf2(gelu(acc[2 * kt + 1][0]), gelu(acc[2 * kt + 1][1]));
        a[kt][3] = bf2(gelu(acc[2 * kt + 1][2]), gelu(acc[2 * kt + 1][3]));
    }
}

__global__ void __launch_bounds__(32 * FW) k_mlp_forward(MlpDev m, const float* __restrict__ x, long long n,
                                                          float* __restrict__ y) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint16_t* sw = reinterpret_cast<uint16_t*>(smem);
    float* sb = reinterpret_cast<float*>(sw + SWN);
    __shared__ float s_mean[NIN], s_scale[NIN], s_out[NOUT];
    load_weights(m, sw, sb);
    if (threadIdx.x < NIN) {
        s_mean[threadIdx.x] = m.p[OMEAN + threadIdx.x];
        s_scale[threadIdx.x] = m.p[OSCALE + threadIdx.x];
    }
    if (threadIdx.x < NOUT) s_out[threadIdx.x] = m.p[OOUT + threadIdx.x];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const long long ntile = (n + TS - 1) / TS;
    for (long long tile = (long long)blockIdx.x * FW + warp; tile < ntile; tile += (long long)gridDim.x * FW) {
        const long long s0 = tile * TS;
        // layer-1 A fragment: normalised inputs of rows g, g+8, columns 2t..2t+1, 2t+8..2t+9
        auto xin = [&](int r, int c) -> uint16_t {
            if (c >= NIN || s0 + r >= n) return 0;
            return bf((x[(s0 + r) * NIN + c] - s_mean[c]) / s_scale[c]);
        };
        uint32_t a1[4];
        a1[0] = pack2(xin(g, 2 * t), xin(g, 2 * t + 1));
        a1[1] = pack2(xin(g + 8, 2 * t), xin(g + 8, 2 * t + 1));
        a1[2] = pack2(xin(g, 2 * t + 8), xin(g, 2 * t + 9));
        a1[3] = pack2(xin(g + 8, 2 * t + 8), xin(g + 8, 2 * t + 9));
        float acc[NH / 8][4];
#pragma unroll
        for (int nt = 0; nt < NH / 8; ++nt) {
            const float b0 = sb[nt * 8 + 2 * t], b1 = sb[nt * 8 + 2 * t + 1];
            acc[nt][0] = b0; acc[nt][1] = b1; acc[nt][2] = b0; acc[nt][3] = b1;
            uint32_t b[2];
            ldb_col(b, sw + SW1 + nt * 8 * LD1, LD1, g, t);
            mma(acc[nt], a1, b);
        }
        uint32_t a[NH / 16][4];
#pragma unroll
        for (int l = 1; l < 3; ++l) {
            gelu_pack(acc, a);
            const uint16_t* W = sw + (l == 1 ? SW2 : SW3);
            const float* bias = sb + l * NH;
#pragma unroll
            for (int nt = 0; nt < NH / 8; ++nt) {
                const float b0 = bias[nt * 8 + 2 * t], b1 = bias[nt * 8 + 2 * t + 1];
                acc[nt][0] = b0; acc[nt][1] = b1; acc[nt][2] = b0; acc[nt][3] = b1;
#pragma unroll
                for (int kt = 0; kt < NH / 16; ++kt) {
                    uint32_t b[2];
                    ldb_col(b, W + nt * 8 * LDW + kt * 16, LDW, g, t);
                    mma(acc[nt], a[kt], b);
                }
            }
        }
        gelu_pack(acc, a);
        float o[4] = {sb[3 * NH + 2 * t], sb[3 * NH + 2 * t + 1], sb[3 * NH + 2 * t], sb[3 * NH + 2 * t + 1]};
#pragma unroll
        for (int kt = 0; kt < NH / 16; ++kt) {
            uint32_t b[2];
            ldb_col(b, sw + SW4 + kt * 16, LDW, g, t);
            mma(o, a[kt], b);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = g + (q >> 1) * 8, c = 2 * t + (q & 1);
            if (c < NOUT && s0 + r < n) y[(s0 + r) * NOUT + c] = o[q] * s_out[c];
        }
    }
}

// ---------------------------------------------------------------------------
// Loss and gradients: L = sum over samples and outputs of
// 0.5 (y_n - t / out_scale)^2 / n_batch (y_n the normalised output).  Per
// warp tile: the forward pass keeping the pre-activations; the output
// deltas; delta_l = (delta_{l+1} W_{l+1}) * GELU'(z_l) down the layers; the
// weight gradients delta^T H and the bias gradients accumulated in FP32
// shared memory; one global atomic add per parameter and block at the end.
// ---------------------------------------------------------------------------
constexpr int GW1 = 0, GW2 = GW1 + NH * K1, GW3 = GW2 + NH * NH, GW4 = GW3 + NH * NH, GB = GW4 + NOUT * NH,
              GN = GB + 3 * NH + NOUT;   // shared-memory gradient layout (dW1 keeps its padded columns)

constexpr size_t grad_smem() {
    return sizeof(uint16_t) * (SWN + NW * (TS * LD1 + 3 * TS * LDW + TS * LD1 + 2 * TS * LDW)) +
           sizeof(float) * (3 * NH + 8 + NW * 3 * TS * NH + GN);
}

__global__ void __launch_bounds__(32 * NW) k_mlp_grad(MlpDev m, const float* __restrict__ x,
                                                       const float* __restrict__ tgt, long long s_begin,
                                                       long long n, float inv_batch, float lam,
                                                       float* __restrict__ grad, double* __restrict__ loss) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint16_t* sw = reinterpret_cast<uint16_t*>(smem);
    uint16_t* tiles = sw + SWN;
    constexpr int WT = TS * LD1 + 3 * TS * LDW + TS * LD1 + 2 * TS * LDW;   // bf16 per warp
    float* sb = reinterpret_cast<float*>(tiles + NW * WT);
    float* zs = sb + 3 * NH + 8;
    float* sg = zs + NW * 3 * TS * NH;
    load_weights(m, sw, sb);
    for (int e = threadIdx.x; e < GN; e += blockDim.x) sg[e] = 0.0f;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    WarpTiles w;
    w.x = tiles + warp * WT;
    for (int l = 0; l < 3; ++l) {
        w.h[l] = w.x + TS * LD1 + l * TS * LDW;
        w.z[l] = zs + (warp * 3 + l) * TS * NH;
    }
    uint16_t* d4 = w.x + TS * LD1 + 3 * TS * LDW;   // [16][LD1] output deltas, columns >= 6 zero
    uint16_t* dA = d4 + TS * LD1;                   // [16][LDW]
    uint16_t* dB = dA + TS * LDW;                   // [16][LDW]
    double lsum = 0.0;
    const long long ntile = (n + TS - 1) / TS;
    // bias gradient of a 16 x 8 fragment's columns, summed over its rows
    auto bias_grad = [&](const float (&acc)[4], float* dst, int cols) {
        float c0 = acc[0] + acc[2], c1 = acc[1] + acc[3];
#pragma unroll
        for (int o = 4; o < 32; o <<= 1) {
            c0 += __shfl_xor_sync(0xffffffffu, c0, o);
            c1 += __shfl_xor_sync(0xffffffffu, c1, o);
        }
        if (g == 0) {
            if (2 * t < cols) atomicAdd(dst + 2 * t, c0);
            if (2 * t + 1 < cols) atomicAdd(dst + 2 * t + 1, c1);
        }
    };
    for (long long tile = (long long)blockIdx.x * NW + warp; tile < ntile; tile += (long long)gridDim.x * NW) {
        const long long s0 = tile * TS;
        load_inputs(m, x + s_begin * NIN, n, s0, w.x, lane);
        __syncwarp();
        float o[4];
        forward_tile(sw, sb, w, o, g, t);
        // output deltas.  With the dissipation weight lam the loss adds
        // lam/2 (Pi(y) - Pi(t))^2 per sample, Pi = -sum c_k tau_k S_k the
        // subgrid dissipation of the dimensionless stresses (c_k = 1 for the
        // diagonal, 2 for the off-diagonal ones, S_k from the sample's
        // gradient features): Pi(y) - Pi(t) = sum_k pe_k e_k with
        // pe_k = -c_k out_scale_k S_k, reduced over the quad of lanes that
        // holds a row's outputs.
        float e4[4], pe4[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = g + (q >> 1) * 8, c = 2 * t + (q & 1);
            float e = 0.0f, pe = 0.0f;
            if (c < NOUT && s0 + r < n) {
                e = o[q] - tgt[(s_begin + s0 + r) * NOUT + c] / m.p[OOUT + c];
                if (lam != 0.0f) {
                    const float* xr = x + (s_begin + s0 + r) * NIN;
                    const int ia = c < 3 ? c : (c == 5 ? 1 : 0), ib = c < 3 ? c : (c == 3 ? 1 : 2);
                    const float S = 0.5f * (xr[3 * ia + ib] + xr[3 * ib + ia]);
                    pe = -(c < 3 ? 1.0f : 2.0f) * m.p[OOUT + c] * S;
                }
            }
            e4[q] = e;
            pe4[q] = pe;
        }
        float dpi[2] = {pe4[0] * e4[0] + pe4[1] * e4[1], pe4[2] * e4[2] + pe4[3] * e4[3]};
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            dpi[h] += __shfl_xor_sync(0xffffffffu, dpi[h], 1);
            dpi[h] += __shfl_xor_sync(0xffffffffu, dpi[h], 2);
        }
        float d[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = g + (q >> 1) * 8, c = 2 * t + (q & 1);
            const float e = e4[q];
            const float v = (e + lam * dpi[q >> 1] * pe4[q]) * inv_batch;
            lsum += 0.5 * (double)e * (double)e * (double)inv_batch;
            d[q] = v;
            d4[r * LD1 + c] = bf(v);
            d4[r * LD1 + c + 8] = 0;
        }
        if (t == 0)
            lsum += 0.5 * (double)lam * ((double)dpi[0] * dpi[0] + (double)dpi[1] * dpi[1]) * (double)inv_batch;
        bias_grad(d, sg + GB + 3 * NH, NOUT);
        __syncwarp();
        // dW4 = d4^T H3 (rows 0..5 kept)
        for (int nt = 0; nt < NH / 8; ++nt) {
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            uint32_t a[4], b[2];
            lda_tr(a, d4, LD1, g, t);
            ldb_row(b, w.h[2] + nt * 8, LDW, g, t);
            mma(acc, a, b);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int r = g + (q >> 1) * 8, c = nt * 8 + 2 * t + (q & 1);
                if (r < NOUT) atomicAdd(sg + GW4 + r * NH + c, acc[q]);
            }
        }
        // delta3 = (d4 W4) * GELU'(z3), then delta2, delta1
        const uint16_t* din = d4;
        int ldin = LD1, kin = 16;
        uint16_t* dout = dA;
        for (int l = 2; l >= 0; --l) {
            const uint16_t* W = sw + (l == 2 ? SW4 : l == 1 ? SW3 : SW2);
            for (int nt = 0; nt < NH / 8; ++nt) {
                float acc[4] = {0.f, 0.f, 0.f, 0.f};
                for (int kt = 0; kt < kin / 16; ++kt) {
                    uint32_t a[4], b[2];
                    lda_row(a, din + kt * 16, ldin, g, t);
                    ldb_row(b, W + kt * 16 * LDW + nt * 8, LDW, g, t);
                    mma(acc, a, b);
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int r = g + (q >> 1) * 8, c = nt * 8 + 2 * t + (q & 1);
                    acc[q] *= gelu_d(w.z[l][r * NH + c]);
                    if (s0 + r >= n) acc[q] = 0.0f;
                    dout[r * LDW + c] = bf(acc[q]);
                }
                bias_grad(acc, sg + GB + l * NH + nt * 8, 8);
            }
            __syncwarp();
            // dW_{l+1} = delta_l^T H_{l-1} (X for l = 0)
            const uint16_t* hin = l > 0 ? w.h[l - 1] : w.x;
            const int ldh = l > 0 ? LDW : LD1, nin = l > 0 ? NH : K1;
            float* dst = sg + (l == 2 ? GW3 : l == 1 ? GW2 : GW1);
            for (int mt = 0; mt < NH / 16; ++mt)
                for (int nt = 0; nt < nin / 8; ++nt) {
                    float acc[4] = {0.f, 0.f, 0.f, 0.f};
                    uint32_t a[4], b[2];
                    lda_tr(a, dout + mt * 16, LDW, g, t);
                    ldb_row(b, hin + nt * 8, ldh, g, t);
                    mma(acc, a, b);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int r = mt * 16 + g + (q >> 1) * 8, c = nt * 8 + 2 * t + (q & 1);
                        atomicAdd(dst + r * nin + c, acc[q]);
                    }
                }
            din = dout;
            ldin = LDW;
            kin = NH;
            dout = (dout == dA) ? dB : dA;
            __syncwarp();
        }
    }
    __syncthreads();
    // block sums to the global FP32 gradient (parameter-vector order)
    for (int e = threadIdx.x; e < NTRAIN; e += blockDim.x) {
        float v;
        if (e < OB1) v = sg[GW1 + (e / NIN) * K1 + e % NIN];
        else if (e < OW2) v = sg[GB + e - OB1];
        else if (e < OB2) v = sg[GW2 + e - OW2];
        else if (e < OW3) v = sg[GB + NH + e - OB2];
        else if (e < OB3) v = sg[GW3 + e - OW3];
        else if (e < OW4) v = sg[GB + 2 * NH + e - OB3];
        else if (e < OB4) v = sg[GW4 + e - OW4];
        else v = sg[GB + 3 * NH + e - OB4];
        atomicAdd(grad + e, v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    if (lane == 0) atomicAdd(loss, lsum);
}

// BF16 copies of the weights in the padded shared-memory layout.
__global__ void k_mlp_pack(const float* __restrict__ p, uint16_t* __restrict__ wb) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < SWN; e += gridDim.x * blockDim.x) {
        float v = 0.0f;
        if (e < SW2) {
            const int r = e / LD1, c = e % LD1;
            if (c < NIN) v = p[OW1 + r * NIN + c];
        } else if (e < SW4) {
            const int q = e < SW3 ? e - SW2 : e - SW3;
            const int r = q / LDW, c = q % LDW;
            if (c < NH) v = p[(e < SW3 ? OW2 : OW3) + r * NH + c];
        } else {
            const int q = e - SW4;
            const int r = q / LDW, c = q % LDW;
            if (r < NOUT && c < NH) v = p[OW4 + r * NH + c];
        }
        wb[e] = bf(v);
    }
}

// Adam on the FP32 parameters (the normalisation entries are not trained);
// the gradient is cleared for the next step.
__global__ void k_mlp_adam(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m1,
                           float* __restrict__ m2, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= NTRAIN) return;
    const float gv = g[e];
    const float a = b1 * m1[e] + (1.0f - b1) * gv;
    const float b = b2 * m2[e] + (1.0f - b2) * gv * gv;
    m1[e] = a;
    m2[e] = b;
    p[e] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
    g[e] = 0.0f;
}

struct Mlp {
    float* p = nullptr;       // NPARAM
    float* g = nullptr;       // NTRAIN
    float* m1 = nullptr;
    float* m2 = nullptr;
    uint16_t* wb = nullptr;   // SWN
    double* loss = nullptr;
    float* xbuf = nullptr;    // staged host data
    float* tbuf = nullptr;
    size_t cap = 0;
    float diss_weight = 0.0f;  // weight of the subgrid-dissipation term of the loss
    long long adam_t = 0;
    int nblocks = 148;
    cudaStream_t st = nullptr;
};

int mfail(int code, const std::string& s) { return set_error(code, s); }
#define MCK(call)                                                                               \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess) return mfail(DIABLO_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

int stage(Mlp* m, const float* x, const float* t, long long n) {
    const size_t need = (size_t)n;
    if (need > m->cap) {
        cudaFree(m->xbuf);
        cudaFree(m->tbuf);
        m->xbuf = m->tbuf = nullptr;
        m->cap = 0;
        MCK(cudaMalloc((void**)&m->xbuf, sizeof(float) * NIN * need));
        MCK(cudaMalloc((void**)&m->tbuf, sizeof(float) * NOUT * need));
        m->cap = need;
    }
    MCK(cudaMemcpyAsync(m->xbuf, x, sizeof(float) * NIN * n, cudaMemcpyHostToDevice, m->st));
    if (t) MCK(cudaMemcpyAsync(m->tbuf, t, sizeof(float) * NOUT * n, cudaMemcpyHostToDevice, m->st));
    return DIABLO_OK;
}

int run_grad(Mlp* m, long long s_begin, long long n, float inv_batch) {
    MlpDev md{m->wb, m->p};
    const size_t smem = grad_smem();
    MCK(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long long tiles = (n + TS - 1) / TS;
    long long nb = (tiles + NW - 1) / NW;
    if (nb > m->nblocks) nb = m->nblocks;
    k_mlp_grad<<<(unsigned)nb, 32 * NW, smem, m->st>>>(md, m->xbuf, m->tbuf, s_begin, n, inv_batch, m->diss_weight,
                                                        m->g, m->loss);
    MCK(cudaGetLastError());
    return DIABLO_OK;
}

}  // namespace

// Forward pass on device arrays (used by the LES branch): x [n][11] -> y [n][6].
cudaError_t launch_mlp_forward(const void* mlp, const float* x, long long n, float* y, cudaStream_t st) {
    const Mlp* m = (const Mlp*)mlp;
    MlpDev md{m->wb, m->p};
    const size_t smem = fwd_smem();
    cudaError_t e = cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const long long tiles = (n + TS - 1) / TS;
    long long nb = (tiles + FW - 1) / FW;
    if (nb > 148 * 4) nb = 148 * 4;
    if (nb < 1) return cudaSuccess;
    k_mlp_forward<<<(unsigned)nb, 32 * FW, smem, st>>>(md, x, n, y);
    return cudaGetLastError();
}

}  // namespace dgpu

using namespace dgpu;

extern "C" {

int diablo_mlp_create(void** mlp) {
    if (!mlp) return mfail(DIABLO_EINVAL, "null pointer argument");
    *mlp = nullptr;
    Mlp* m = new Mlp();
    cudaError_t e = cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc((void**)&m->p, sizeof(float) * NPARAM);
    if (e == cudaSuccess) e = cudaMalloc((void**)&m->g, sizeof(float) * NTRAIN);
    if (e == cudaSuccess) e = cudaMalloc((void**)&m->m1, sizeof(float) * NTRAIN);
    if (e == cudaSuccess) e = cudaMalloc((void**)&m->m2, sizeof(float) * NTRAIN);
    if (e == cudaSuccess) e = cudaMalloc((void**)&m->wb, sizeof(uint16_t) * SWN);
    if (e == cudaSuccess) e = cudaMalloc((void**)&m->loss, sizeof(double));
    // Zeroed on the network's own non-blocking stream and waited for here: a memset on the
    // legacy default stream is not ordered before the later uploads and packing on m->st,
    // and could land after them (packed weights wiped to zero, Adam moments reset mid-run).
    if (e == cudaSuccess) e = cudaMemsetAsync(m->p, 0, sizeof(float) * NPARAM, m->st);
    if (e == cudaSuccess) e = cudaMemsetAsync(m->g, 0, sizeof(float) * NTRAIN, m->st);
    if (e == cudaSuccess) e = cudaMemsetAsync(m->m1, 0, sizeof(float) * NTRAIN, m->st);
    if (e == cudaSuccess) e = cudaMemsetAsync(m->m2, 0, sizeof(float) * NTRAIN, m->st);
    if (e == cudaSuccess) e = cudaMemsetAsync(m->wb, 0, sizeof(uint16_t) * SWN, m->st);
    if (e == cudaSuccess) e = cudaMemsetAsync(m->loss, 0, sizeof(double), m->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->st);
    int dev = 0, sms = 148;
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) {
        diablo_mlp_destroy(m);
        return mfail(DIABLO_ECUDA, std::string("MLP set-up: ") + cudaGetErrorString(e));
    }
    m->nblocks = sms;
    *mlp = m;
    return DIABLO_OK;
}

int diablo_mlp_destroy(void* mlp) {
    Mlp* m = (Mlp*)mlp;
    if (!m) return mfail(DIABLO_EINVAL, "null MLP");
    if (m->st) cudaStreamSynchronize(m->st);
    void* ptrs[] = {m->p, m->g, m->m1, m->m2, m->wb, m->loss, m->xbuf, m->tbuf};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    if (m->st) cudaStreamDestroy(m->st);
    delete m;
    return DIABLO_OK;
}

int diablo_mlp_set_params(void* mlp, const float* params) {
    Mlp* m = (Mlp*)mlp;
    if (!m || !params) return mfail(DIABLO_EINVAL, "null pointer argument");
    for (int i = 0; i < NIN; ++i)
        if (!(params[OSCALE + i] != 0.0f)) return mfail(DIABLO_EINVAL, "input scales must be non-zero");
    for (int i = 0; i < NOUT; ++i)
        if (!(params[OOUT + i] != 0.0f)) return mfail(DIABLO_EINVAL, "output scales must be non-zero");
    MCK(cudaMemcpyAsync(m->p, params, sizeof(float) * NPARAM, cudaMemcpyHostToDevice, m->st));
    k_mlp_pack<<<(SWN + 255) / 256, 256, 0, m->st>>>(m->p, m->wb);
    MCK(cudaGetLastError());
    MCK(cudaMemsetAsync(m->m1, 0, sizeof(float) * NTRAIN, m->st));
    MCK(cudaMemsetAsync(m->m2, 0, sizeof(float) * NTRAIN, m->st));
    MCK(cudaMemsetAsync(m->g, 0, sizeof(float) * NTRAIN, m->st));
    m->adam_t = 0;
    MCK(cudaStreamSynchronize(m->st));
    return DIABLO_OK;
}

int diablo_mlp_set_dissipation_weight(void* mlp, float weight) {
    Mlp* m = (Mlp*)mlp;
    if (!m) return mfail(DIABLO_EINVAL, "null MLP");
    if (!(weight >= 0.0f) || !std::isfinite(weight)) return mfail(DIABLO_EINVAL, "dissipation weight must be >= 0");
    m->diss_weight = weight;
    return DIABLO_OK;
}

int diablo_mlp_get_params(void* mlp, float* params) {
    Mlp* m = (Mlp*)mlp;
    if (!m || !params) return mfail(DIABLO_EINVAL, "null pointer argument");
    MCK(cudaMemcpyAsync(params, m->p, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost, m->st));
    MCK(cudaStreamSynchronize(m->st));
    return DIABLO_OK;
}

int diablo_mlp_forward(void* mlp, const float* x, long long n, float* y) {
    Mlp* m = (Mlp*)mlp;
    if (!m || !x || !y || n < 0) return mfail(DIABLO_EINVAL, "bad MLP forward arguments");
    if (n == 0) return DIABLO_OK;
    int rc = stage(m, x, nullptr, n);
    if (rc) return rc;
    MCK(launch_mlp_forward(m, m->xbuf, n, m->tbuf, m->st));
    MCK(cudaMemcpyAsync(y, m->tbuf, sizeof(float) * NOUT * n, cudaMemcpyDeviceToHost, m->st));
    MCK(cudaStreamSynchronize(m->st));
    return DIABLO_OK;
}

int diablo_mlp_gradient(void* mlp, const float* x, const float* t, long long n, double* loss, float* grad) {
    Mlp* m = (Mlp*)mlp;
    if (!m || !x || !t || n <= 0 || !loss || !grad) return mfail(DIABLO_EINVAL, "bad MLP gradient arguments");
    int rc = stage(m, x, t, n);
    if (rc) return rc;
    MCK(cudaMemsetAsync(m->g, 0, sizeof(float) * NTRAIN, m->st));
    MCK(cudaMemsetAsync(m->loss, 0, sizeof(double), m->st));
    if ((rc = run_grad(m, 0, n, 1.0f / (float)n))) return rc;
    MCK(cudaMemcpyAsync(grad, m->g, sizeof(float) * NTRAIN, cudaMemcpyDeviceToHost, m->st));
    MCK(cudaMemcpyAsync(loss, m->loss, sizeof(double), cudaMemcpyDeviceToHost, m->st));
    MCK(cudaMemsetAsync(m->g, 0, sizeof(float) * NTRAIN, m->st));
    MCK(cudaStreamSynchronize(m->st));
    return DIABLO_OK;
}

int diablo_mlp_train(void* mlp, const float* x, const float* t, long long n, int batch, int steps, float lr,
                     double* losses) {
    Mlp* m = (Mlp*)mlp;
    if (!m || !x || !t || n <= 0 || batch <= 0 || steps < 0) return mfail(DIABLO_EINVAL, "bad MLP training arguments");
    int rc = stage(m, x, t, n);
    if (rc) return rc;
    const long long nb = (n + batch - 1) / batch;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int s = 0; s < steps; ++s) {
        const long long s0 = (long long)(s % nb) * batch;
        const long long cnt = s0 + batch <= n ? batch : n - s0;
        MCK(cudaMemsetAsync(m->loss, 0, sizeof(double), m->st));
        if ((rc = run_grad(m, s0, cnt, 1.0f / (float)cnt))) return rc;
        ++m->adam_t;
        const float c1 = 1.0f - std::pow(b1, (float)m->adam_t), c2 = 1.0f - std::pow(b2, (float)m->adam_t);
        k_mlp_adam<<<(NTRAIN + 255) / 256, 256, 0, m->st>>>(m->p, m->g, m->m1, m->m2, lr, b1, b2, eps, c1, c2);
        MCK(cudaGetLastError());
        k_mlp_pack<<<(SWN + 255) / 256, 256, 0, m->st>>>(m->p, m->wb);
        MCK(cudaGetLastError());
        if (losses) MCK(cudaMemcpyAsync(losses + s, m->loss, sizeof(double), cudaMemcpyDeviceToHost, m->st));
    }
    MCK(cudaStreamSynchronize(m->st));
    return DIABLO_OK;
}

}  // extern "C"
