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
    FastK K;
    K.rc2 = k.f_rc2;
    K.chi = k.f_chi;
    K.chi_sq = k.f_chi_sq;
    K.chip = k.f_chip;
    K.chip_sq = k.f_chip_sq;
    K.sigma0 = k.f_sigma0;
    K.four_eps0 = k.f_4eps0;
    K.half_chi = k.f_half_chi;
    K.half_chip = k.f_half_chip;
    K.mu_code = k.mu_code;
    K.nu_code = k.nu_code;
    K.mu = (float)k.mu;
    K.nu = (float)k.nu;
    float dx = (float)d[3 * i], dy = (float)d[3 * i + 1], dz = (float)d[3 * i + 2];
    float r2 = dx * dx + dy * dy + dz * dz;
    double ni = sqrt(ei[3 * i] * ei[3 * i] + ei[3 * i + 1] * ei[3 * i + 1] + ei[3 * i + 2] * ei[3 * i + 2]);
    double nj = sqrt(ej[3 * i] * ej[3 * i] + ej[3 * i + 1] * ej[3 * i + 1] + ej[3 * i + 2] * ej[3 * i + 2]);
    float e = pair_fast(K, dx, dy, dz, r2, (float)(ei[3 * i] / ni), (float)(ei[3 * i + 1] / ni),
                        (float)(ei[3 * i + 2] / ni), (float)(ej[3 * i] / nj), (float)(ej[3 * i + 1] / nj),
                        (float)(ej[3 * i + 2] / nj));
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
