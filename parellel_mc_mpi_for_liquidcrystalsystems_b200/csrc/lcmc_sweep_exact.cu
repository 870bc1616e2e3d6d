// lcmc_sweep_exact.cu - FP64 checkerboard phase, bit-identical to the CPU oracle.
//
// Compiled with -fmad=false: every double operation is a single IEEE-rounded
// +, -, *, / or sqrt, in the order of the reference's pij_GB / GBCollRod
// (MCnptColloid.c:2607-2681, 1758-1854), so the accept/reject sequence equals
// the oracle's canonical sweep.
//
// One warp per active cell.  The particles of the cell are attempted one after
// another in ascending id (the reference picks a random particle per cycle,
// MCnptColloid.c:2475; its MPI path loops over an active subcell's particles,
// 683-700).  For each attempt the 32 lanes split the stencil slots q (q mod 32),
// sum the old and new pair energies lane-locally in q order and combine them
// with a xor butterfly: the canonical order the oracle reproduces.
#include <cuda_runtime.h>

#include "lcmc_gb.cuh"
#include "lcmc_internal.h"
#include "lcmc_rng.cuh"
#include "lcmc_trial.cuh"
#include "lcmc_volume_cells.cuh"

namespace lcmc {

__device__ __forceinline__ int find_replica(const int *off, int R, int a)
{
    int lo = 0, hi = R;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (off[mid] <= a) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ double warp_sum_butterfly(double x)
{
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) x = x + __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

__global__ void __launch_bounds__(128) k_phase_exact(DevView v, int ci)
{
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    __shared__ int s_cell[4][27];
    __shared__ int s_base[4][28];
    const int *off = v.act_off + ci * (v.R + 1);
    const int total = off[v.r_hi]; // this launch's replicas: active cells [off[r_lo], off[r_hi])
    for (int a = off[v.r_lo] + blockIdx.x * nw + wib; a < total; a += gridDim.x * nw) {
        const int r = find_replica(off, v.R, a);
        const Replica &p = v.rep[r];
        if (p.use_fast) continue;
        const int col = p.perm[ci];
        const int bx = col % p.kc[0], by = (col / p.kc[0]) % p.kc[1], bz = col / (p.kc[0] * p.kc[1]);
        const int nc0 = p.nc[0], nc1 = p.nc[1], nc2 = p.nc[2];
        const int nax = axis_colour_count(nc0, p.kc[0], bx), nay = axis_colour_count(nc1, p.kc[1], by);
        int loc = a - off[r];
        const int cx = axis_colour_cell(nc0, p.kc[0], bx, loc % nax);
        loc /= nax;
        const int cy = axis_colour_cell(nc1, p.kc[1], by, loc % nay);
        const int cz = axis_colour_cell(nc2, p.kc[2], bz, loc / nay);
        const int cell = p.cell_off + (cz * nc1 + cy) * nc0 + cx;

        // canonical stencil: dz, dy, dx = -1..1, duplicates dropped at first occurrence
        int c = -1;
        if (lane < 27) {
            int dz = lane / 9 - 1, dy = (lane / 3) % 3 - 1, dx = lane % 3 - 1;
            int x = (cx + dx + nc0) % nc0, y = (cy + dy + nc1) % nc1, z = (cz + dz + nc2) % nc2;
            c = p.cell_off + (z * nc1 + y) * nc0 + x;
        }
        unsigned same = __match_any_sync(0xffffffffu, c);
        bool keep = lane < 27 && (__ffs(same) - 1) == lane;
        unsigned kb = __ballot_sync(0xffffffffu, keep);
        int ncell = __popc(kb);
        int slot = __popc(kb & ((1u << lane) - 1u));
        if (keep) s_cell[wib][slot] = c;
        // exclusive prefix of counts over kept cells in slot order
        int cnt_slot = 0;
        __syncwarp();
        if (lane < ncell) cnt_slot = v.cell_start[s_cell[wib][lane] + 1] - v.cell_start[s_cell[wib][lane]];
        int inc = cnt_slot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane < ncell) s_base[wib][lane] = inc - cnt_slot;
        if (lane == 31) s_base[wib][ncell] = inc;
        __syncwarp();

        const int cs = v.cell_start[cell], ce = v.cell_start[cell + 1];
        double dE_sum = 0.0, dE_abs = 0.0;
        int nacc = 0, nhard = 0;
        unsigned long long npairs = 0ull;
        const unsigned long long cands = (unsigned long long)(s_base[wib][ncell] - 1) * (unsigned long long)(ce - cs);
        for (int g = cs; g < ce; g++) {
            const uint32_t id = (uint32_t)v.id[g];
            double ro[3] = {v.px[g], v.py[g], v.pz[g]};
            double eo[3] = {v.ox[g], v.oy[g], v.oz[g]};
            double rn[3], en[3], dsp[3], uacc;
            int ok = make_trial(p, id, ro, eo, rn, en, dsp, &uacc);
            if (ok && leaves_cell(p, cx, cy, cz, ro, dsp)) { // out of its cell: rejected, no energy evaluation
                if (lane == 0) {
                    v.outcome[p.p_off + id] = 0;
                    if (v.rec_dE) {
                        v.rec_dE[p.p_off + id] = 0.0;
                        v.rec_lu[p.p_off + id] = log_unit(uacc);
                    }
                }
                continue;
            }
            if (!ok) {
                if (lane == 0) {
                    v.outcome[p.p_off + id] = 2;
                    if (v.rec_dE) {
                        v.rec_dE[p.p_off + id] = 0.0;
                        v.rec_lu[p.p_off + id] = log_unit(uacc);
                    }
                }
                nhard++;
                continue;
            }
            double po = 0.0, pn = 0.0;
            int np = 0;
            for (int s = 0; s < ncell; s++) {
                const int B = s_base[wib][s], n_s = s_base[wib][s + 1] - B;
                const int g0 = v.cell_start[s_cell[wib][s]];
                for (int q = B + ((lane - B) & 31); q < B + n_s; q += 32) {
                    const int j = g0 + (q - B);
                    if (j == g) continue;
                    double rj[3] = {v.px[j], v.py[j], v.pz[j]};
                    double ej[3] = {v.ox[j], v.oy[j], v.oz[j]};
                    double d[3];
                    double r2 = dist_fold(ro[0], ro[1], ro[2], rj[0], rj[1], rj[2], p.L, d);
                    if (r2 < p.k.rc2) {
                        po += pair_exact(p.k, r2, d, eo, ej);
                        np++;
                    }
                    r2 = dist_fold(rn[0], rn[1], rn[2], rj[0], rj[1], rj[2], p.L, d);
                    if (r2 < p.k.rc2) {
                        pn += pair_exact(p.k, r2, d, en, ej);
                        np++;
                    }
                }
            }
            double Eo = warp_sum_butterfly(po);
            double En = warp_sum_butterfly(pn);
            if (p.k.coll_on) {
                Eo = Eo + colloid_rod(p.k, ro, eo, p.L);
                En = En + colloid_rod(p.k, rn, en, p.L);
            }
            const double dE = En - Eo;
            const bool acc = (dE <= 0.0) || (log_unit(uacc) <= -p.k.beta * dE);
            npairs += (unsigned long long)np;
            if (acc) {
                if (lane == 0) {
                    v.px[g] = rn[0];
                    v.py[g] = rn[1];
                    v.pz[g] = rn[2];
                    v.ox[g] = en[0];
                    v.oy[g] = en[1];
                    v.oz[g] = en[2];
                }
                dE_sum += dE;
                dE_abs += fabs(dE);
                nacc++;
            }
            if (lane == 0) {
                v.outcome[p.p_off + id] = acc ? 1 : 0;
                if (v.rec_dE) {
                    v.rec_dE[p.p_off + id] = dE;
                    v.rec_lu[p.p_off + id] = log_unit(uacc);
                }
            }
            __syncwarp();
        }
        // pair counter: sum over lanes
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) npairs += __shfl_xor_sync(0xffffffffu, npairs, o);
        if (lane == 0) {
            v.cell_e0[cell] = dE_sum;
            v.cell_abs[cell] = dE_abs;
            v.cell_fp64[cell] = 0;
            v.cell_n0[cell] = nacc;
            v.cell_n1[cell] = nhard;
            v.cell_pairs[cell] = npairs;
            v.cell_cands[cell] = cands;
        }
        __syncwarp();
    }
}

// Total energy (tot_ene, MCnptColloid.c:1598-1622) in FP64, warp per particle:
// sum over unordered pairs (r < rc, minimum image) found in the 27-cell
// stencil, plus the colloid term of every particle, with pair_exact (the
// reference-order term).  SCALED: the NPT volume move's energies of the
// current configuration and of the one scaled by lam about the origin
// (colloid at the scaled box centre), with pair_energy64.  Works on any grid,
// including boxes of fewer than 3 cells per axis (the wrapped stencil is
// deduplicated).
//
// Each pair is evaluated once: slots are sorted by cell, so particle i takes
// the rest of its own cell (slots > i) and the whole of every stencil cell
// with a larger index; e0[i] (e1[i] scaled) holds those pair terms plus its
// colloid term, and the slot sums add up to the total.  Only about one
// candidate in eight is inside the cutoff, so pairs are not evaluated where
// they are found: a distance pass over 32 candidates at a time appends the
// in-cutoff (candidate, configuration) items to a per-warp queue, and every
// 32 queued items are evaluated with all lanes busy.  The order of the FP64
// additions is fixed by the data, so results repeat bit for bit.
constexpr int EQ = 96; // queue entries per warp: < 32 pending + 64 from one chunk
#ifndef LCMC_ENERGY_MIN_BLOCKS
#define LCMC_ENERGY_MIN_BLOCKS 8
#endif

template <bool SCALED>
__global__ void __launch_bounds__(128, LCMC_ENERGY_MIN_BLOCKS) k_energy_exact(DevView v, double *e0, double *e1, int *hard)
{
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    __shared__ int s_start[4][28]; // flat index of the first candidate of each cell
    __shared__ int s_base[4][28];  // particle slot minus flat index, per cell
    __shared__ int s_qj[4][EQ];    // queued candidate slot, configuration in bit 31
    if (SCALED) { // nothing to do when the cell kernel serves every NPT replica needing the energies
        bool any = false;
        for (int r = 0; r < v.R && !any; r++) {
            const Replica &p = v.rep[r];
            any = p.ensemble == 2 && !(p.da_on && !p.vol_stage1) && !volume_cells_serves<true>(p);
        }
        if (!any) return;
    }
    for (int i = blockIdx.x * nw + wib; i < v.ntot; i += gridDim.x * nw) {
        const int r = v.p2r[i];
        const Replica &p = v.rep[r];
        const int nc0 = p.nc[0], nc1 = p.nc[1], nc2 = p.nc[2];
        // NVT, screened out, or served by the cell kernel (>= 4 cells per axis)
        if (SCALED && (p.ensemble != 2 || (p.da_on && !p.vol_stage1) || volume_cells_serves<true>(p))) continue;
        const int own = v.scid[i];
        const int cell = own - p.cell_off;
        const int cx = cell % nc0, cy = (cell / nc0) % nc1, cz = cell / (nc0 * nc1);
        int c = -1;
        if (lane < 27) {
            int dz = lane / 9 - 1, dy = (lane / 3) % 3 - 1, dx = lane % 3 - 1;
            int x = (cx + dx + nc0) % nc0, y = (cy + dy + nc1) % nc1, z = (cz + dz + nc2) % nc2;
            c = p.cell_off + (z * nc1 + y) * nc0 + x;
        }
        const unsigned same = __match_any_sync(0xffffffffu, c);
        const bool keep = lane < 27 && (__ffs(same) - 1) == lane && c >= own;
        const unsigned kb = __ballot_sync(0xffffffffu, keep);
        const int ncell = __popc(kb);
        const int slot = __popc(kb & lt);
        int first = 0, cnt = 0;
        if (keep) {
            const int b = v.cell_start[c], e = v.cell_start[c + 1];
            first = c == own ? i + 1 : b;
            cnt = e - first;
        }
        int inc = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (keep) {
            s_start[wib][slot] = inc - cnt;
            s_base[wib][slot] = first - (inc - cnt);
        }
        const int total = __shfl_sync(0xffffffffu, inc, 31);
        if (lane == 0) s_start[wib][ncell] = total;
        __syncwarp();

        const double lam = SCALED ? p.vol_lambda : 1.0;
        const double Ls[3] = {p.L[0] * lam, p.L[1] * lam, p.L[2] * lam};
        const double ri[3] = {v.px[i], v.py[i], v.pz[i]};
        const double ei[3] = {v.ox[i], v.oy[i], v.oz[i]};
        const double rs[3] = {ri[0] * lam, ri[1] * lam, ri[2] * lam};
        // the scaled distance is lam^2 r2 up to a few ulp: decide the scaled
        // cutoff from it unless it lies within 1e-10 of rc^2
        const double lam2 = lam * lam, rc2 = p.k.rc2, band = 1e-10 * rc2;
        double a0 = 0.0, a1 = 0.0;
        int qn = 0;
        int sc = 0; // this lane's current cell (its candidates only move forward)

        for (int t0 = 0; t0 < total; t0 += 32) {
            const int q = t0 + lane;
            bool f0 = false, f1 = false;
            int j = 0;
            if (q < total) {
                while (s_start[wib][sc + 1] <= q) sc++;
                j = s_base[wib][sc] + q;
                const double rj[3] = {v.px[j], v.py[j], v.pz[j]};
                double d[3];
                const double r2 = dist_fold(ri[0], ri[1], ri[2], rj[0], rj[1], rj[2], p.L, d);
                f0 = r2 < rc2;
                if (SCALED) {
                    const double r2s = lam2 * r2;
                    if (fabs(r2s - rc2) > band) f1 = r2s < rc2;
                    else f1 = dist_fold(rs[0], rs[1], rs[2], rj[0] * lam, rj[1] * lam, rj[2] * lam, Ls, d) < rc2;
                }
            }
            const unsigned b0 = __ballot_sync(0xffffffffu, f0);
            const unsigned b1 = __ballot_sync(0xffffffffu, f1);
            if (f0) s_qj[wib][qn + __popc(b0 & lt)] = j;
            if (f1) s_qj[wib][qn + __popc(b0) + __popc(b1 & lt)] = j | (int)0x80000000u;
            qn += __popc(b0) + __popc(b1);
            __syncwarp();
            // evaluate full batches of 32 queued pairs
            while (qn >= 32 || (qn > 0 && t0 + 32 >= total)) {
                const int m = qn < 32 ? qn : 32;
                if (lane < m) {
                    const int e = s_qj[wib][lane];
                    const int jj = e & 0x7fffffff;
                    const double rj[3] = {v.px[jj], v.py[jj], v.pz[jj]};
                    const double ej[3] = {v.ox[jj], v.oy[jj], v.oz[jj]};
                    double d[3], r2;
                    if (e < 0) {
                        r2 = dist_fold(rs[0], rs[1], rs[2], rj[0] * lam, rj[1] * lam, rj[2] * lam, Ls, d);
                        a1 += pair_energy64(p.k, r2, d, ei, ej);
                    } else {
                        r2 = dist_fold(ri[0], ri[1], ri[2], rj[0], rj[1], rj[2], p.L, d);
                        a0 += SCALED ? pair_energy64(p.k, r2, d, ei, ej) : pair_exact(p.k, r2, d, ei, ej);
                    }
                }
                // move entries [m, qn) to the front
                int mv0 = 0, mv1 = 0;
                if (m + lane < qn) mv0 = s_qj[wib][m + lane];
                if (m + 32 + lane < qn) mv1 = s_qj[wib][m + 32 + lane];
                __syncwarp();
                if (m + lane < qn) s_qj[wib][lane] = mv0;
                if (m + 32 + lane < qn) s_qj[wib][32 + lane] = mv1;
                __syncwarp();
                qn -= m;
            }
        }
        a0 = warp_sum_butterfly(a0);
        a1 = warp_sum_butterfly(a1);
        if (lane == 0) {
            double u0 = a0, u1 = a1;
            if (p.k.coll_on) {
                u0 += colloid_rod(p.k, ri, ei, p.L);
                if (SCALED) u1 += colloid_rod(p.k, rs, ei, Ls);
            }
            e0[i] = u0;
            if (SCALED) {
                e1[i] = u1;
                double d[3];
                double r2 = dist_fold(rs[0], rs[1], rs[2], 0.5 * Ls[0], 0.5 * Ls[1], 0.5 * Ls[2], Ls, d);
                hard[i] = !(r2 > p.k.coll_R * p.k.coll_R);
            }
        }
        __syncwarp();
    }
}

} // namespace lcmc

#include "lcmc_launch.h"

namespace lcmc {

void launch_phase_exact(const DevView &v, cudaStream_t s, int ci, int grid)
{
    k_phase_exact<<<grid, 128, 0, s>>>(v, ci);
}

int energy_exact_blocks_per_sm()
{
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_energy_exact<true>, 128, 0) != cudaSuccess || b < 1) {
        cudaGetLastError();
        b = 4;
    }
    return b;
}

// resident blocks of the cell kernel on this device (queried once)
static int volume_cells_grid()
{
    static int grid = 0;
    if (!grid) {
        int dev = 0, sms = 0, b = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_volume_cells<true, false>, 128, 0) != cudaSuccess ||
            b < 1) {
            cudaGetLastError();
            b = 2;
        }
        grid = b * (sms > 0 ? sms : 1);
    }
    return grid;
}

// scaled = 1: the volume move's U(V), U(V') -- the cell kernel for systems with
// >= 4 cells per axis, the per-particle kernel for the rest
void launch_energy_exact(const DevView &v, cudaStream_t s, double *e0, double *e1, int *hard, int scaled, int grid)
{
    if (scaled) {
        k_volume_cells<true, false><<<volume_cells_grid(), 128, 0, s>>>(v, e0, e1, hard);
        k_energy_exact<true><<<grid, 128, 0, s>>>(v, e0, e1, hard);
    } else {
        k_energy_exact<false><<<grid, 128, 0, s>>>(v, e0, e1, hard);
    }
}

} // namespace lcmc
