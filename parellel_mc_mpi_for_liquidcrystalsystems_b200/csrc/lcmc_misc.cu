// lcmc_misc.cu - per-replica reductions, the NPT volume move, the order
// parameter sums and the id-order copies used by upload/download.
#include <cuda_runtime.h>

#include "lcmc_internal.h"
#include "lcmc_rng.cuh"

namespace lcmc {

// Block-wide sum in a fixed order (thread-strided partials, then a tree).
template <typename T>
__device__ __forceinline__ T block_sum(T x, T *sh)
{
    sh[threadIdx.x] = x;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    T r = sh[0];
    __syncthreads();
    return r;
}

// Block per replica: total energy = sum of per-particle energies (deterministic).
// Resets the running energy to the recomputed value and records the drift.
__global__ void k_energy_reduce(DevView v, const double *e0, int replica_only)
{
    const int r = blockIdx.x;
    if (replica_only >= 0 && r != replica_only) return;
    const Replica &p = v.rep[r];
    __shared__ double sh[256];
    double s = 0.0;
    for (int i = threadIdx.x; i < p.n; i += blockDim.x) s += e0[p.p_off + i];
    double tot = block_sum(s, sh);
    if (threadIdx.x == 0) {
        DevStats &st = v.stats[r];
        st.drift = st.energy - tot;
        st.energy = tot;
        st.last_recompute = tot;
        v.scratch_d[r] = tot;
    }
}

// NPT: draw the ln V step of this sweep (one per NPT replica).
__global__ void k_volume_propose(DevView v)
{
    for (int r = threadIdx.x; r < v.R; r += blockDim.x) {
        Replica &p = v.rep[r];
        if (p.ensemble != 2) {
            p.vol_lambda = 1.0;
            p.vol_state = 0;
            continue;
        }
        U4 o = draw(p.key, SWEEP_ID, p.sweep, TAG_VOLUME);
        p.vol_delta = p.dlnv_max * (2.0 * u01(o.x) - 1.0);
        p.vol_lambda = 1.0 + expm1_small(p.vol_delta / 3.0);
        p.vol_stage1 = 1; // the surrogate's stage 1 may clear it
        p.vol_dU_sur = 0.0;
    }
}

// NPT: block per replica.  Sums U(V), U(V') and hard-core hits, then the
// Metropolis test of the ln V walk:
//   ln A = -beta (dU + P dV) + (N + 1) delta,  dV = V (e^delta - 1).
__global__ void k_volume_accept(DevView v, const double *e0, const double *e1, const int *hard)
{
    const int r = blockIdx.x;
    Replica &p = v.rep[r];
    if (p.ensemble != 2) return;
    if (p.da_on && !p.vol_stage1) { // rejected by the surrogate: no exact energy was computed
        if (threadIdx.x == 0) {
            v.stats[r].vol_att += 1ull;
            v.stats[r].vol_s1rej += 1ull;
            p.vol_state = 4;
        }
        return;
    }
    __shared__ double sh[256];
    __shared__ int shi[256];
    double a = 0.0, b = 0.0;
    int h = 0;
    for (int i = threadIdx.x; i < p.n; i += blockDim.x) {
        a += e0[p.p_off + i];
        b += e1[p.p_off + i];
        h |= hard[p.p_off + i];
    }
    double U0 = block_sum(a, sh);
    double U1 = block_sum(b, sh);
    int H = block_sum(h, shi);
    if (threadIdx.x == 0) {
        DevStats &st = v.stats[r];
        st.drift = st.energy - U0;
        st.last_recompute = U0;
        st.vol_att += 1ull;
        p.vol_U_old = U0;
        p.vol_U_new = U1;
        int state;
        if (H) {
            state = 3;
        } else if (p.da_on) { // stage 2 of delayed acceptance: exact dU against the surrogate's
            const double lnA2 = -p.k.beta * ((U1 - U0) - p.vol_dU_sur);
            U4 o = draw(p.key, SWEEP_ID, p.sweep, TAG_VOLUME);
            state = (lnA2 >= 0.0 || log_unit(u01(o.w)) <= lnA2) ? 1 : 2;
        } else {
            const double V = p.L[0] * p.L[1] * p.L[2];
            const double dV = V * expm1_small(p.vol_delta);
            const double lnA = -p.k.beta * ((U1 - U0) + p.pressure * dV) + (double)(p.n + 1) * p.vol_delta;
            U4 o = draw(p.key, SWEEP_ID, p.sweep, TAG_VOLUME);
            state = (lnA >= 0.0 || log_unit(u01(o.y)) <= lnA) ? 1 : 2;
        }
        p.vol_state = state;
        if (state == 1) {
            st.vol_acc += 1ull;
            st.energy = U1;
            for (int k = 0; k < 3; k++) p.L[k] = p.L[k] * p.vol_lambda;
        } else {
            st.energy = U0;
        }
    }
}

__global__ void k_volume_scale(DevView v)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < v.ntot; i += gridDim.x * blockDim.x) {
        const Replica &p = v.rep[v.p2r[i]];
        if (p.vol_state != 1) continue;
        const double lam = p.vol_lambda;
        v.px[i] = v.px[i] * lam;
        v.py[i] = v.py[i] * lam;
        v.pz[i] = v.pz[i] * lam;
    }
}

// Q-tensor sums of one replica: out[0..5] = sum u_x u_x, u_x u_y, u_x u_z,
// u_y u_y, u_y u_z, u_z u_z (compute_liquid_crystal_order_parameters,
// MCnptColloid.c:2149-2167, in FP64).
__global__ void k_order_sums(DevView v, int r, double *out)
{
    const Replica &p = v.rep[r];
    __shared__ double sh[256];
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < p.n; i += blockDim.x) {
        const int g = p.p_off + i;
        const double x = v.ox[g], y = v.oy[g], z = v.oz[g];
        s[0] += x * x;
        s[1] += x * y;
        s[2] += x * z;
        s[3] += y * y;
        s[4] += y * z;
        s[5] += z * z;
    }
    for (int k = 0; k < 6; k++) {
        double t = block_sum(s[k], sh);
        if (threadIdx.x == 0) out[k] = t;
    }
}

// Copy one replica's sorted slots into id order (download) in the q* buffer.
__global__ void k_to_id_order(DevView v, int r)
{
    const Replica &p = v.rep[r];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += gridDim.x * blockDim.x) {
        const int g = p.p_off + i;
        const int d = p.p_off + v.id[g];
        v.qx[d] = v.px[g];
        v.qy[d] = v.py[g];
        v.qz[d] = v.pz[g];
        v.qux[d] = v.ox[g];
        v.quy[d] = v.oy[g];
        v.quz[d] = v.oz[g];
    }
}

} // namespace lcmc

#include "lcmc_launch.h"

namespace lcmc {

void launch_energy_reduce(const DevView &v, cudaStream_t s, const double *e0, int replica_only)
{
    k_energy_reduce<<<v.R, 256, 0, s>>>(v, e0, replica_only);
}

void launch_volume(const DevView &v, cudaStream_t s, double *e0, double *e1, int *hard, int grid)
{
    launch_volume_propose(v, s);
    launch_volume_finish(v, s, e0, e1, hard, grid);
}

void launch_volume_propose(const DevView &v, cudaStream_t s) { k_volume_propose<<<1, 256, 0, s>>>(v); }

// exact FP64 energies of the current and the scaled configuration (skipped for
// replicas the surrogate screened out), the acceptance test, optional sample
// recording, and the scaling of accepted replicas.
void launch_volume_finish(const DevView &v, cudaStream_t s, double *e0, double *e1, int *hard, int grid)
{
    launch_energy_exact(v, s, e0, e1, hard, 1, grid);
    k_volume_accept<<<v.R, 256, 0, s>>>(v, e0, e1, hard);
    if (v.rec_cap > 0) launch_record_samples(v, s);
    k_volume_scale<<<grid, 256, 0, s>>>(v);
}

void launch_order_sums(const DevView &v, cudaStream_t s, int r, double *out) { k_order_sums<<<1, 256, 0, s>>>(v, r, out); }

void launch_to_id_order(const DevView &v, cudaStream_t s, int r, int grid)
{
    k_to_id_order<<<grid, 256, 0, s>>>(v, r);
}

} // namespace lcmc
