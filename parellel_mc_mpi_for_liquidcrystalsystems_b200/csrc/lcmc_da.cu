// lcmc_da.cu - delayed-acceptance volume moves with the learned surrogate,
// training-sample recording and per-sweep history (no reference counterpart:
// the reference has no NPT move, MCnptColloid.c:3978).
//
// Features of a configuration x (8 channels on an 8^3 grid of the box in
// fractional coordinates, channel-major, then the move's |delta ln V|):
//   0  number density / 0.3
//   1-5 Q tensor: <ux ux> - 1/3, <ux uy>, <ux uz>, <uy uy> - 1/3, <uy uz>
//   6  radial alignment <(u . r_hat)^2> - 1/3, r_hat from the colloid centre
//   7  (density / 0.3)^2
//   4096: |delta| / delta_max
// The network g predicts the slope dU / (N delta) of a move of size |delta|.
// The surrogate energy change is
//   dU~(x -> y) = N s delta [g(phi(x), |delta|) + g(phi(y), |delta|)] / 2,
// symmetric in its two evaluations and odd in delta, so dU~(y -> x) =
// -dU~(x -> y) exactly and the two-stage test (Christen & Fox, J. Comput.
// Graph. Stat. 14 (2005) 795) keeps detailed balance:
//   stage 1: ln A1 = -beta (dU~ + P dV) + (N + 1) delta
//   stage 2 (exact FP64 dU, only after stage 1 passed): ln A2 = -beta (dU - dU~)
// Under the affine volume move the features of the scaled configuration y
// follow from those of x (cells, orientations and radial directions are
// unchanged; only the density channels see the new volume), so both rows are
// built from one pass over x.  The two network rows are averaged, not
// differenced: a difference of two nearly equal BF16-input outputs would be
// mostly rounding.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "lcmc_internal.h"
#include "lcmc_launch.h"
#include "lcmc_reduce.cuh"
#include "lcmc_rng.cuh"

namespace lcmc {

constexpr int FG = 8, FC = FG * FG * FG;
// Pooled sums are accumulated as 64-bit fixed point (2^-32 units) with integer
// atomics: integer addition is associative, so the features, and with them
// every delayed-acceptance decision, do not depend on the order in which the
// threads add.  Terms are in [-1, 1]; a cell of 2^30 particles cannot overflow.
constexpr double FIX_ONE = 4294967296.0;

__device__ __forceinline__ void add_fixed(unsigned long long *a, double x)
{
    atomicAdd(a, (unsigned long long)__double2ll_rn(x * FIX_ONE));
}

__global__ void k_feat_accum(DevView v)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < v.ntot; i += gridDim.x * blockDim.x) {
        const int r = v.p2r[i];
        const Replica &p = v.rep[r];
        if (p.ensemble != 2 || !(p.da_kind == 1 || v.rec_cap > 0)) continue;
        int c3[3];
        const double pos[3] = {v.px[i], v.py[i], v.pz[i]};
        double d[3], dd = 0.0;
        for (int a = 0; a < 3; a++) {
            int c = (int)(pos[a] / p.L[a] * FG);
            c3[a] = c < 0 ? 0 : (c >= FG ? FG - 1 : c);
            d[a] = pos[a] - 0.5 * p.L[a];
            dd += d[a] * d[a];
        }
        const int cell = (c3[2] * FG + c3[1]) * FG + c3[0];
        const double ux = v.ox[i], uy = v.oy[i], uz = v.oz[i];
        const double inv = 1.0 / sqrt(ux * ux + uy * uy + uz * uz);
        const double x = ux * inv, y = uy * inv, z = uz * inv;
        const double rad = dd > 0.0 ? (x * d[0] + y * d[1] + z * d[2]) / sqrt(dd) : 0.0;
        unsigned long long *a = v.feat_acc + ((size_t)r * FC + cell) * 7;
        atomicAdd(a + 0, 1ull);
        add_fixed(a + 1, x * x);
        add_fixed(a + 2, x * y);
        add_fixed(a + 3, x * z);
        add_fixed(a + 4, y * y);
        add_fixed(a + 5, y * z);
        add_fixed(a + 6, rad * rad);
    }
}

__device__ __forceinline__ double from_fixed(unsigned long long a) { return (double)(long long)a / FIX_ONE; }

// rows 2r (x) and 2r + 1 (y), both with |delta|, of the surrogate's BF16
// input; the x row also in FP32 (feat_f) for sample recording.
__global__ void k_feat_finalize(DevView v, __nv_bfloat16 *X, int ldx)
{
    const int r = blockIdx.x;
    const Replica &p = v.rep[r];
    if (p.ensemble != 2 || !(p.da_kind == 1 || v.rec_cap > 0)) return;
    const double V = p.L[0] * p.L[1] * p.L[2];
    const double inv_vc = (double)FC / V / 0.3;
    // The y row is what these kernels compute for the scaled configuration
    // itself (box L lambda, exactly as an accepted move sets it): same cells,
    // same orientation sums, density from the scaled volume.  So the reverse
    // move y -> x sees bit for bit the rows of this one, swapped.
    const double lam = p.vol_lambda;
    const double Vy = (p.L[0] * lam) * (p.L[1] * lam) * (p.L[2] * lam);
    const double inv_vc_y = (double)FC / Vy / 0.3;
    const float dn = (float)(p.dlnv_max > 0.0 ? fabs(p.vol_delta) / p.dlnv_max : 0.0);
    __nv_bfloat16 *rx = X ? X + (size_t)(2 * r) * ldx : nullptr;
    __nv_bfloat16 *ry = X ? X + (size_t)(2 * r + 1) * ldx : nullptr;
    float *rf = v.feat_f + (size_t)r * LCMC_FEAT;
    for (int c = threadIdx.x; c < FC; c += blockDim.x) {
        const unsigned long long *a = v.feat_acc + ((size_t)r * FC + c) * 7;
        const double n = (double)a[0];
        const double in = n > 0.0 ? 1.0 / n : 0.0;
        const double t = n > 0.0 ? 1.0 / 3.0 : 0.0;
        float f[8];
        f[0] = (float)(n * inv_vc);
        f[1] = (float)(from_fixed(a[1]) * in - t);
        f[2] = (float)(from_fixed(a[2]) * in);
        f[3] = (float)(from_fixed(a[3]) * in);
        f[4] = (float)(from_fixed(a[4]) * in - t);
        f[5] = (float)(from_fixed(a[5]) * in);
        f[6] = (float)(from_fixed(a[6]) * in - t);
        f[7] = f[0] * f[0];
        const float g0 = (float)(n * inv_vc_y);
        for (int ch = 0; ch < 8; ch++) {
            rf[ch * FC + c] = f[ch];
            if (rx) {
                const float g = ch == 0 ? g0 : (ch == 7 ? g0 * g0 : f[ch]);
                rx[ch * FC + c] = __float2bfloat16(f[ch]);
                ry[ch * FC + c] = __float2bfloat16(g);
            }
        }
    }
    if (threadIdx.x == 0) {
        rf[8 * FC] = dn;
        if (rx) {
            rx[8 * FC] = __float2bfloat16(dn);
            ry[8 * FC] = __float2bfloat16(dn);
        }
    }
}

// Stage 1 of the delayed-acceptance test, one thread per replica.
__global__ void k_da_stage1(DevView v, const float *y)
{
    for (int r = threadIdx.x; r < v.R; r += blockDim.x) {
        Replica &p = v.rep[r];
        if (p.ensemble != 2 || !p.da_on || p.da_kind != 1) continue;
        const double dUs = (double)p.n * p.da_scale * p.vol_delta * 0.5 * ((double)y[2 * r] + (double)y[2 * r + 1]);
        const double V = p.L[0] * p.L[1] * p.L[2];
        const double dV = V * expm1_small(p.vol_delta);
        const double lnA1 = -p.k.beta * (dUs + p.pressure * dV) + (double)(p.n + 1) * p.vol_delta;
        U4 o = draw(p.key, SWEEP_ID, p.sweep, TAG_VOLUME);
        p.vol_dU_sur = dUs;
        p.vol_stage1 = (lnA1 >= 0.0 || log_unit(u01(o.z)) <= lnA1) ? 2 : 0;
    }
}

// Copy this sweep's (features of x with |delta|, exact slope dU / (N delta))
// of every NPT replica whose exact volume energy was computed into the sample
// ring, in replica order (one block, so the ring's order repeats run to run).
// delta is never 0: it is dlnV_max (2u - 1) with u = (k + 1/2) / 2^32.
__global__ void k_record_samples(DevView v)
{
    if (v.rec_cap <= 0) return;
    int slot = *v.rec_count;
    for (int r = 0; r < v.R; r++) {
        const Replica &p = v.rep[r];
        if (p.ensemble != 2 || p.vol_state == 3 || p.vol_stage1 == 0) continue;
        if (slot < v.rec_cap) {
            const float *src = v.feat_f + (size_t)r * LCMC_FEAT;
            float *dst = v.rec_x + (size_t)slot * LCMC_FEAT;
            for (int k = threadIdx.x; k < LCMC_FEAT; k += blockDim.x) dst[k] = src[k];
            if (threadIdx.x == 0)
                v.rec_y[slot] = (float)((p.vol_U_new - p.vol_U_old) / ((double)p.n * p.vol_delta));
        }
        slot++;
    }
    __syncthreads(); // every thread has read the old count
    if (threadIdx.x == 0) *v.rec_count = slot;
}

// Per-sweep history of every replica: sweep, Q-tensor sums (6), energy, volume.
__global__ void __launch_bounds__(256) k_hist_record(DevView v)
{
    const int r = blockIdx.x;
    const Replica &p = v.rep[r];
    double s[6];
    finish_sums<6>(v, r, s); // Q-tensor chunk sums, launched just before
    if (threadIdx.x == 0) {
        const unsigned long long sw = p.sweep - 1ull; // finalize already counted this sweep
        double *row = v.hist + ((size_t)r * v.hist_cap + (size_t)(sw % (unsigned long long)v.hist_cap)) * 9;
        row[0] = (double)sw;
        for (int k = 0; k < 6; k++) row[1 + k] = s[k];
        row[7] = v.stats[r].energy;
        row[8] = p.L[0] * p.L[1] * p.L[2];
    }
}

void launch_features(const DevView &v, cudaStream_t s, void *X, int ldx, int grid)
{
    cudaMemsetAsync(v.feat_acc, 0, sizeof(unsigned long long) * (size_t)v.R * FC * 7, s);
    k_feat_accum<<<grid, 256, 0, s>>>(v);
    k_feat_finalize<<<v.R, 256, 0, s>>>(v, (__nv_bfloat16 *)X, ldx);
}

void launch_da_stage1(const DevView &v, cudaStream_t s, const float *y) { k_da_stage1<<<1, 256, 0, s>>>(v, y); }
void launch_record_samples(const DevView &v, cudaStream_t s) { k_record_samples<<<1, 256, 0, s>>>(v); }
void launch_hist_record(const DevView &v, cudaStream_t s)
{
    launch_q_chunk_sums(v, s);
    k_hist_record<<<v.R, 256, 0, s>>>(v);
}

} // namespace lcmc
