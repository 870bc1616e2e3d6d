// lcmc_pairtest64.cu - the pair term on given inputs in the FP64 kernel's
// arithmetic (compiled without FMA contraction, like lcmc_sweep_exact.cu).
#include <cuda_runtime.h>

#include "lcmc_gb.cuh"
#include "lcmc_internal.h"

namespace lcmc {

__global__ void k_pair_terms64(GBConsts k, int n, const double *d, const double *ei, const double *ej, double *out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double dr[3] = {d[3 * i], d[3 * i + 1], d[3 * i + 2]};
    double a[3] = {ei[3 * i], ei[3 * i + 1], ei[3 * i + 2]};
    double b[3] = {ej[3 * i], ej[3 * i + 1], ej[3 * i + 2]};
    double xs = dr[0] * dr[0], ys = dr[1] * dr[1], zs = dr[2] * dr[2];
    double r2 = xs + ys + zs;
    out[i] = r2 < k.rc2 ? pair_exact(k, r2, dr, a, b) : 0.0;
}

} // namespace lcmc

#include "lcmc_launch.h"

namespace lcmc {
void launch_pair_terms64(const GBConsts &k, int n, const double *d, const double *ei, const double *ej, double *out,
                         cudaStream_t s)
{
    k_pair_terms64<<<(n + 127) / 128, 128, 0, s>>>(k, n, d, ei, ej, out);
}
} // namespace lcmc
