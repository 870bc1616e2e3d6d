// lcmc_pairtest.cu - the pair term on given inputs, FP32 and FP64 arithmetic
// (test and error-statistics hook behind lcmc_pair_terms).
#include <cuda_runtime.h>

#include "lcmc_gb.cuh"
#include "lcmc_internal.h"

namespace lcmc {

__global__ void k_pair_terms32(GBConsts k, int n, const double *d, const double *ei, const double *ej, double *out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const FastK K = fast_consts(k);
    const bool spec21 = k.mu_code == 2 && k.nu_code == 1 && k.f_sigma0 == 1.0f;
    float dx = (float)d[3 * i], dy = (float)d[3 * i + 1], dz = (float)d[3 * i + 2];
    float r2 = dx * dx + dy * dy + dz * dz;
    double ni = sqrt(ei[3 * i] * ei[3 * i] + ei[3 * i + 1] * ei[3 * i + 1] + ei[3 * i + 2] * ei[3 * i + 2]);
    double nj = sqrt(ej[3 * i] * ej[3 * i] + ej[3 * i + 1] * ej[3 * i + 1] + ej[3 * i + 2] * ej[3 * i + 2]);
    const float a0 = (float)(ei[3 * i] / ni), a1 = (float)(ei[3 * i + 1] / ni), a2 = (float)(ei[3 * i + 2] / ni);
    const float b0 = (float)(ej[3 * i] / nj), b1 = (float)(ej[3 * i + 1] / nj), b2 = (float)(ej[3 * i + 2] / nj);
    // the specialised term the sweep kernels run for GB(kappa, kappa', 2, 1), else the general one
    float e = spec21 ? pair_fast_t<true>(K, dx, dy, dz, r2, a0, a1, a2, b0, b1, b2)
                     : pair_fast_t<false>(K, dx, dy, dz, r2, a0, a1, a2, b0, b1, b2);
    out[i] = r2 < K.rc2 ? (double)e : 0.0;
}

} // namespace lcmc

#include "lcmc_launch.h"

namespace lcmc {
void launch_pair_terms32(const GBConsts &k, int n, const double *d, const double *ei, const double *ej, double *out,
                         cudaStream_t s)
{
    k_pair_terms32<<<(n + 127) / 128, 128, 0, s>>>(k, n, d, ei, ej, out);
}
} // namespace lcmc
