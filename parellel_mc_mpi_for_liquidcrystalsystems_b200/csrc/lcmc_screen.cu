// lcmc_screen.cu - stage 1 of delayed-acceptance volume moves from the energy
// change evaluated with FP32 pair terms (no reference counterpart: the
// reference has no NPT move, MCnptColloid.c:3978).
//
// The screen's energy U32(x) sums, in FP64, the FP32 Gay-Berne term of every
// unordered in-cutoff pair plus the FP64 colloid term of every particle:
//   * in/out of the cutoff is decided on the FP32 copy of the state
//     (cell-local coordinates) and, within 1e-5 of rc^2, by the FP64 distance,
//     so the pair set is exactly the FP64 kernel's;
//   * each pair term takes the FP64 minimum-image vector rounded to FP32 and
//     the orientations of the FP32 state copy (unit_f32 of the FP64
//     orientation, however the copy was written), so it is a function of the
//     two particles' FP64 coordinates alone.
// U32 is therefore a function of the configuration (up to the order of its
// FP64 additions), and dU~(x -> y) = U32(y) - U32(x) is odd under x <-> y: the
// two-stage test of Christen & Fox (J. Comput. Graph. Stat. 14 (2005) 795)
//   stage 1: ln A1 = -beta (dU~ + P dV) + (N + 1) delta   (the plain move's draw)
//   stage 2: ln A2 = -beta (dU - dU~)                     (exact FP64 dU)
// keeps detailed balance.  |dU - dU~| is ~1e-3 kT at N = 2^18, so stage 2
// almost always accepts what stage 1 passed, and the FP64 recompute runs only
// for the moves the plain test would have a chance to accept.  The scaled
// configuration's vectors are formed exactly as the reverse move forms them
// (positions r lambda, box L lambda), so U32(y) here equals, up to summation
// order, the U32 of the reverse move.  Systems on the FP32 kernel only (the
// FP32 state copy exists there).
#include <cuda_runtime.h>

#include "lcmc_gb.cuh"
#include "lcmc_internal.h"
#include "lcmc_launch.h"
#include "lcmc_reduce.cuh"
#include "lcmc_rng.cuh"
#include "lcmc_trial.cuh"
#include "lcmc_volume_cells.cuh"

namespace lcmc {

// Stage 1, block per replica: dU~ from the chunk sums of the screen's
// energies (k = 0 U32(V), 1 U32(V'), 2 hard-core hits at V').
__global__ void __launch_bounds__(256) k_screen_stage1(DevView v)
{
    const int r = blockIdx.x;
    Replica &p = v.rep[r];
    if (p.ensemble != 2 || p.da_kind != 2 || !p.use_fast) return;
    double su[3];
    finish_sums<3>(v, r, su);
    if (threadIdx.x == 0) {
        if (su[2] > 0.0) { // a rod centre inside the colloid at V': the exact test rejects too
            p.vol_dU_sur = 0.0;
            p.vol_stage1 = 0;
            return;
        }
        const double dUs = su[1] - su[0];
        const double V = p.L[0] * p.L[1] * p.L[2];
        const double dV = V * expm1_small(p.vol_delta);
        const double lnA1 = -p.k.beta * (dUs + p.pressure * dV) + (double)(p.n + 1) * p.vol_delta;
        U4 o = draw(p.key, SWEEP_ID, p.sweep, TAG_VOLUME);
        p.vol_dU_sur = dUs;
        p.vol_stage1 = (lnA1 >= 0.0 || log_unit(u01(o.y)) <= lnA1) ? 2 : 0;
    }
}

int screen_blocks_per_sm()
{
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_volume_cells<false, true>, 128, 0) != cudaSuccess || b < 1) {
        cudaGetLastError();
        b = 4;
    }
    return b;
}

void launch_screen(const DevView &v, cudaStream_t s, double *e0, double *e1, int *hard, int grid, bool spec21)
{
    if (spec21) k_volume_cells<false, true><<<grid, 128, 0, s>>>(v, e0, e1, hard);
    else k_volume_cells<false, false><<<grid, 128, 0, s>>>(v, e0, e1, hard);
    launch_chunk_sums_volume(v, s, e0, e1, hard);
    k_screen_stage1<<<v.R, 256, 0, s>>>(v);
}

} // namespace lcmc
