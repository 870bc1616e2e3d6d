// lcmc_misc.cu - per-replica reductions, the NPT volume move, the order
// parameter sums and the id-order copies used by upload/download.
#include <cuda_runtime.h>

#include "lcmc_internal.h"
#include "lcmc_reduce.cuh"
#include "lcmc_rng.cuh"

namespace lcmc {

// Two-level sums over a replica's particles, in a fixed order (results repeat
// bit for bit): blocks (chunk c, replica r) add LCMC_RED_CHUNK particles each
// into red_part[(r * red_nchunk + c) * LCMC_RED_K + k], then one block per replica adds
// its chunks.  One block streaming a whole replica was limited to one SM's
// bandwidth (1.9 ms for 8 MB at N = 2^20).
//   mode 0: k = 0 sum of e0 (total energy)
//   mode 1: k = 0, 1, 2 sums of e0, e1 and hard-core hits (NPT replicas whose
//           volume move was not screened out)
//   mode 2: k = 0..5 Q-tensor sums u_x u_x, u_x u_y, u_x u_z, u_y u_y, u_y u_z,
//           u_z u_z (compute_liquid_crystal_order_parameters,
//           MCnptColloid.c:2149-2167, in FP64)
template <int K, int MODE>
__global__ void __launch_bounds__(256) k_chunk_sums(DevView v, const double *e0, const double *e1, const int *hard)
{
    const int c = blockIdx.x, r = blockIdx.y;
    const Replica &p = v.rep[r];
    const int i0 = c * LCMC_RED_CHUNK;
    if (i0 >= p.n) return;
    if (MODE == 1 && (p.ensemble != 2 || p.vol_stage1 == 0)) return;
    const int i1 = min(p.n, i0 + LCMC_RED_CHUNK);
    double s[K];
#pragma unroll
    for (int k = 0; k < K; k++) s[k] = 0.0;
    for (int i = i0 + (int)threadIdx.x; i < i1; i += blockDim.x) {
        const int g = p.p_off + i;
        if (MODE == 0) {
            s[0] += e0[g];
        } else if (MODE == 1) {
            s[0] += e0[g];
            s[1] += e1[g];
            s[2] += hard[g] ? 1.0 : 0.0;
        } else {
            const double x = v.ox[g], y = v.oy[g], z = v.oz[g];
            s[0] += x * x;
            s[1] += x * y;
            s[2] += x * z;
            s[3] += y * y;
            s[4] += y * z;
            s[5] += z * z;
        }
    }
    __shared__ double sh[K][8];
    block_sums<K>(s, sh);
    if (threadIdx.x == 0)
        for (int k = 0; k < K; k++) v.red_part[((size_t)r * v.red_nchunk + c) * LCMC_RED_K + k] = s[k];
}

// Block per replica: total energy from the chunk sums.  Resets the running
// energy to the recomputed value and records the drift.
__global__ void __launch_bounds__(256) k_energy_reduce(DevView v, int replica_only)
{
    const int r = blockIdx.x;
    if (replica_only >= 0 && r != replica_only) return;
    double s[1];
    finish_sums<1>(v, r, s);
    if (threadIdx.x == 0) {
        const double tot = s[0];
        DevStats &st = v.stats[r];
        st.drift = st.energy - tot;
        st.energy = tot;
        st.last_recompute = tot;
        st.abs_dE = 0.0;
        v.scratch_d[r] = tot;
    }
}

// Periodic FP64 energy check (EnergyCheck, MCnptColloid.c:1343-1362, called
// every statistics interval at 946-955, where it prints the running and the
// recomputed energies): block per replica, the recomputed total from the chunk
// sums; for replicas that are due (all = 1: every replica; else those whose
// sweep counter is a multiple of check_every) drift = running - recomputed
// against the tolerance
//   check_tol (max(|E|, N 4 eps0) + sum of |dE| accepted since the last check)
// (the running sum's rounding grows with the energy changes it carried, which
// near overlaps are many orders above |E|); a breach sets F_DRIFT.  The
// running energy is reset to the recomputed value either way.
__global__ void __launch_bounds__(256) k_energy_check(DevView v, int all)
{
    const int r = blockIdx.x;
    const Replica &p = v.rep[r];
    const bool due = all || (p.check_every > 0 && p.sweep % (unsigned long long)p.check_every == 0ull);
    if (!due) return;
    double s[1];
    finish_sums<1>(v, r, s);
    if (threadIdx.x == 0) {
        const double tot = s[0];
        DevStats &st = v.stats[r];
        const double drift = st.energy - tot;
        const double bound = p.check_tol * (fmax(fabs(tot), (double)p.n * p.k.four_eps0) + st.abs_dE);
        const bool breach = !(fabs(drift) <= bound);
        st.drift = drift;
        st.drift_bound = bound;
        st.checks += 1ull;
        if (breach) {
            st.breaches += 1ull;
            st.flags |= F_DRIFT;
        }
        st.energy = tot;
        st.last_recompute = tot;
        st.abs_dE = 0.0;
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
        p.vol_stage1 = 1; // a screen's stage 1 sets 0 (rejected) or 2 (passed)
        p.vol_dU_sur = 0.0;
    }
}

// NPT: block per replica.  U(V), U(V') and hard-core hits from the chunk sums,
// then the Metropolis test of the ln V walk:
//   ln A = -beta (dU + P dV) + (N + 1) delta,  dV = V (e^delta - 1).
__global__ void __launch_bounds__(256) k_volume_accept(DevView v)
{
    const int r = blockIdx.x;
    Replica &p = v.rep[r];
    if (p.ensemble != 2) return;
    if (p.vol_stage1 == 0) { // rejected by the screen: no exact energy was computed
        if (threadIdx.x == 0) {
            v.stats[r].vol_att += 1ull;
            v.stats[r].vol_s1rej += 1ull;
            p.vol_state = 4;
        }
        return;
    }
    double su[3];
    finish_sums<3>(v, r, su);
    if (threadIdx.x == 0) {
        const double U0 = su[0], U1 = su[1];
        const bool H = su[2] > 0.0;
        DevStats &st = v.stats[r];
        // the exact U(V) doubles as an energy check of the running energy
        // (same tolerance as the periodic check)
        st.drift = st.energy - U0;
        st.drift_bound = p.check_tol * (fmax(fabs(U0), (double)p.n * p.k.four_eps0) + st.abs_dE);
        st.checks += 1ull;
        if (!(fabs(st.drift) <= st.drift_bound)) {
            st.breaches += 1ull;
            st.flags |= F_DRIFT;
        }
        st.abs_dE = 0.0;
        st.last_recompute = U0;
        st.vol_att += 1ull;
        p.vol_U_old = U0;
        p.vol_U_new = U1;
        int state;
        if (H) {
            state = 3;
        } else if (p.vol_stage1 == 2) { // stage 2 of delayed acceptance: exact dU against the screen's
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

// Q-tensor sums of one replica from the chunk sums (mode 2): out[0..5].
__global__ void __launch_bounds__(256) k_order_finish(DevView v, int r, double *out)
{
    double s[6];
    finish_sums<6>(v, r, s);
    if (threadIdx.x == 0)
        for (int k = 0; k < 6; k++) out[k] = s[k];
}

// Checks of an uploaded configuration (check_no_colloid_overlaps,
// MCnptColloid.c:1324-1340, and the box bounds) on the staged arrays; writes
// the identity id map.  flag bits: 1 outside the box, 2 inside the colloid,
// 4 zero or non-finite orientation.
__global__ void k_validate_upload(const double *px, const double *py, const double *pz, const double *ox,
                                  const double *oy, const double *oz, int *id, int n, double L0, double L1, double L2,
                                  double R2, int *flag)
{
    int bad = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double x = px[i], y = py[i], z = pz[i];
        if (!(x >= 0.0 && x <= L0 && y >= 0.0 && y <= L1 && z >= 0.0 && z <= L2)) bad |= 1;
        const double dx = x - 0.5 * L0, dy = y - 0.5 * L1, dz = z - 0.5 * L2;
        if (dx * dx + dy * dy + dz * dz < R2) bad |= 2;
        const double n2 = ox[i] * ox[i] + oy[i] * oy[i] + oz[i] * oz[i];
        if (!(n2 > 0.0) || !(n2 < 1e300)) bad |= 4;
        id[i] = i;
    }
    bad = __reduce_or_sync(0xffffffffu, bad);
    if (bad && (threadIdx.x & 31) == 0) atomicOr(flag, bad);
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

static dim3 chunk_grid(const DevView &v) { return dim3(v.red_nchunk, v.R); }

void launch_energy_reduce(const DevView &v, cudaStream_t s, const double *e0, int replica_only)
{
    k_chunk_sums<1, 0><<<chunk_grid(v), 256, 0, s>>>(v, e0, nullptr, nullptr);
    k_energy_reduce<<<v.R, 256, 0, s>>>(v, replica_only);
}

void launch_energy_check(const DevView &v, cudaStream_t s, const double *e0, int all)
{
    k_chunk_sums<1, 0><<<chunk_grid(v), 256, 0, s>>>(v, e0, nullptr, nullptr);
    k_energy_check<<<v.R, 256, 0, s>>>(v, all);
}

void launch_chunk_sums_volume(const DevView &v, cudaStream_t s, const double *e0, const double *e1, const int *hard)
{
    k_chunk_sums<3, 1><<<chunk_grid(v), 256, 0, s>>>(v, e0, e1, hard);
}

void launch_q_chunk_sums(const DevView &v, cudaStream_t s)
{
    k_chunk_sums<6, 2><<<chunk_grid(v), 256, 0, s>>>(v, nullptr, nullptr, nullptr);
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
    launch_chunk_sums_volume(v, s, e0, e1, hard);
    k_volume_accept<<<v.R, 256, 0, s>>>(v);
    if (v.rec_cap > 0) launch_record_samples(v, s);
    k_volume_scale<<<grid, 256, 0, s>>>(v);
}

void launch_order_sums(const DevView &v, cudaStream_t s, int r, double *out)
{
    launch_q_chunk_sums(v, s);
    k_order_finish<<<1, 256, 0, s>>>(v, r, out);
}

void launch_validate_upload(const double *const x[6], int *id, int n, const double L[3], double R2, int *flag,
                            cudaStream_t s, int grid)
{
    k_validate_upload<<<grid, 256, 0, s>>>(x[0], x[1], x[2], x[3], x[4], x[5], id, n, L[0], L[1], L[2], R2, flag);
}

void launch_to_id_order(const DevView &v, cudaStream_t s, int r, int grid)
{
    k_to_id_order<<<grid, 256, 0, s>>>(v, r);
}

} // namespace lcmc
