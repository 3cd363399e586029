// filter.cu -- filter_chan(n) (for/filter.f:1-98) on the device: the
// scalar's Fourier columns damped by a sharpened raised cosine of the
// horizontal wavenumber (rows J = 0..NY), then, for I >= 1 and K >= 1, the
// vertical compact filter of the reference with alpha = 0 -- its tridiagonal
// matrix is the identity, so the filter is the explicit 5-point stencil of
// its right-hand side on rows J = 2..NY-1.  Row J = 0 keeps its horizontally
// filtered value (the reference copies an element of VEC_C it never sets
// there); row NY+1 is untouched, as in the reference.  One thread per
// retained (kx,kz) column, FP64.
#include <cuda_runtime.h>

#include <string>

#include "../../include/diablo_gpu.h"
#include "kernels.cuh"
#include "launch.h"

namespace dgpu {

__global__ void k_filter_chan(Dims d, double2* __restrict__ cth, const double* __restrict__ kxw,
                              const double* __restrict__ kzw, double lx, double lz, double fnx, double fnz) {
    const size_t ps = d.splane();
    const size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ps) return;
    const int i = (int)(g % d.ldx), m = (int)(g / d.ldx);
    if (i >= d.nkxp || m >= d.nkzt) return;
    const int ny = d.ny;
    const double a1 = kxw[i] * lx * 1.0 / fnx, a2 = kzw[m] * lz * 1.0 / fnz;
    const double s0 = 0.5 * (1.0 + cos(sqrt(pow(a1, 2.0) + pow(a2, 2.0))));
    const double sg = pow(s0, 4.0) * (35.0 - 84.0 * s0 + 70.0 * pow(s0, 2.0) - 20.0 * pow(s0, 3.0));
    double2* c = cth + g;
    auto hf = [&](int j) {   // horizontally filtered row j (row NY+1 is not filtered)
        const double2 v = c[(size_t)j * ps];
        return j <= ny ? make_double2(sg * v.x, sg * v.y) : v;
    };
    if (i == 0 || m == 0) {
        for (int j = 0; j <= ny; ++j) c[(size_t)j * ps] = hf(j);
        return;
    }
    const double alpha = 0.0;
    const double fa = (1.0 / 8.0) * (5.0 + 6.0 * alpha), fb = 0.5 * (1.0 + 2.0 * alpha),
                 fc = (-1.0 / 8.0) * (1.0 - 2.0 * alpha);
    // window h[j-2..j+2] of horizontally filtered values, row j written when
    // its stencil is complete (the writes trail the reads by two rows)
    double2 w0 = hf(0), w1 = hf(1), w2 = hf(2), w3 = ny >= 3 ? hf(3) : make_double2(0.0, 0.0);
    c[0] = w0;
    c[ps] = w1;
    for (int j = 2; j <= ny; ++j) {
        const double2 w4 = j + 2 <= ny + 1 ? hf(j + 2) : make_double2(0.0, 0.0);
        double2 out = w2;
        if (j <= ny - 1) {
            out.x = fa * w2.x + (fb / 2.0) * (w3.x + w1.x) + (fc / 2.0) * (w4.x + w0.x);
            out.y = fa * w2.y + (fb / 2.0) * (w3.y + w1.y) + (fc / 2.0) * (w4.y + w0.y);
        }
        c[(size_t)j * ps] = out;
        w0 = w1; w1 = w2; w2 = w3; w3 = w4;
    }
}

}  // namespace dgpu

namespace dgpu {
cudaError_t launch_filter_chan(const Dims& d, double2* cth, const double* kx, const double* kz, double lx,
                               double lz, double fnx, double fnz, cudaStream_t st) {
    const size_t n = d.splane();
    k_filter_chan<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(d, cth, kx, kz, lx, lz, fnx, fnz);
    return cudaGetLastError();
}
}  // namespace dgpu
