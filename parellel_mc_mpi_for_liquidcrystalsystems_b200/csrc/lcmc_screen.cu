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

namespace lcmc {

constexpr int SQ = 96; // queue entries per warp: < 32 pending + 64 from one round of two chunks

template <bool SPEC21>
__global__ void __launch_bounds__(128, 6) k_energy_screen(DevView v, double *e0, double *e1, int *hard)
{
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    __shared__ int s_start[4][28];         // flat index of the first candidate of each kept cell
    __shared__ int s_base[4][28];          // particle slot minus flat index, per kept cell
    __shared__ float s_ox[4][28], s_oy[4][28], s_oz[4][28]; // offset of each kept cell's origin
    __shared__ int s_qj[4][SQ];            // queued candidate slot; bit 30: in cutoff at V, bit 31: at V'
    for (int i = blockIdx.x * nw + wib; i < v.ntot; i += gridDim.x * nw) {
        const int r = v.p2r[i];
        const Replica &p = v.rep[r];
        if (p.ensemble != 2 || p.da_kind != 2 || !p.use_fast) continue;
        const int nc0 = p.nc[0], nc1 = p.nc[1], nc2 = p.nc[2]; // >= 4: 27 distinct cells
        const int own = v.scid[i];
        const int cell = own - p.cell_off;
        const int cx = cell % nc0, cy = (cell / nc0) % nc1, cz = cell / (nc0 * nc1);
        int c = -1;
        if (lane < 27) {
            int dz = lane / 9 - 1, dy = (lane / 3) % 3 - 1, dx = lane % 3 - 1;
            int x = (cx + dx + nc0) % nc0, y = (cy + dy + nc1) % nc1, z = (cz + dz + nc2) % nc2;
            c = p.cell_off + (z * nc1 + y) * nc0 + x;
        }
        // each unordered pair once: the rest of the own cell (slots > i) and the
        // stencil cells with a larger index
        const bool keep = lane < 27 && c >= own;
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
            s_ox[wib][slot] = (float)(lane % 3 - 1) * (float)p.w[0];
            s_oy[wib][slot] = (float)((lane / 3) % 3 - 1) * (float)p.w[1];
            s_oz[wib][slot] = (float)(lane / 9 - 1) * (float)p.w[2];
        }
        const int total = __shfl_sync(0xffffffffu, inc, 31);
        if (lane == 0) s_start[wib][ncell] = total;
        __syncwarp();

        const double lam = p.vol_lambda;
        const double Ls[3] = {p.L[0] * lam, p.L[1] * lam, p.L[2] * lam};
        const double ri[3] = {v.px[i], v.py[i], v.pz[i]};
        const double rs[3] = {ri[0] * lam, ri[1] * lam, ri[2] * lam};
        const float4 ci = v.cl4[i];
        const float2 ci2 = v.cl2[i];
        const float eix = ci.w, eiy = ci2.x, eiz = ci2.y; // unit_f32 of the FP64 orientation
        const double rc2 = p.k.rc2;
        const float rc2f = (float)rc2, lam2f = (float)(lam * lam);
        const float lo = rc2f * (1.0f - 1e-5f), hi = rc2f * (1.0f + 1e-5f);
        const FastK K = fast_consts(p.k);
        double a0 = 0.0, a1 = 0.0;
        int qn = 0, sc = 0;
        // two chunks of 32 candidates per round: their loads are independent
        for (int t0 = 0; t0 < total; t0 += 64) {
            bool any[2];
            int ent[2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int q = t0 + 32 * h + lane;
                bool f0 = false, f1 = false;
                int j = 0;
                if (q < total) {
                    while (s_start[wib][sc + 1] <= q) sc++;
                    j = s_base[wib][sc] + q;
                    const float4 cj = v.cl4[j];
                    const float dx = cj.x + s_ox[wib][sc] - ci.x;
                    const float dy = cj.y + s_oy[wib][sc] - ci.y;
                    const float dz = cj.z + s_oz[wib][sc] - ci.z;
                    const float r2 = dx * dx + dy * dy + dz * dz, r2s = lam2f * r2;
                    double d[3];
                    if (r2 < lo) f0 = true;
                    else if (r2 <= hi) f0 = dist_fold(ri[0], ri[1], ri[2], v.px[j], v.py[j], v.pz[j], p.L, d) < rc2;
                    if (r2s < lo) f1 = true;
                    else if (r2s <= hi)
                        f1 = dist_fold(rs[0], rs[1], rs[2], v.px[j] * lam, v.py[j] * lam, v.pz[j] * lam, Ls, d) < rc2;
                }
                any[h] = f0 || f1;
                ent[h] = j | (f0 ? 0x40000000 : 0) | (f1 ? (int)0x80000000u : 0);
            }
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const unsigned b = __ballot_sync(0xffffffffu, any[h]);
                if (any[h]) s_qj[wib][qn + __popc(b & lt)] = ent[h];
                qn += __popc(b);
            }
            __syncwarp();
            while (qn >= 32 || (qn > 0 && t0 + 64 >= total)) {
                const int m = qn < 32 ? qn : 32;
                if (lane < m) {
                    const int e = s_qj[wib][lane];
                    const int jj = e & 0x3fffffff;
                    const double rj[3] = {v.px[jj], v.py[jj], v.pz[jj]};
                    const float ejx = v.cl4[jj].w;
                    const float2 ej2 = v.cl2[jj];
                    const float ejy = ej2.x, ejz = ej2.y;
                    double d[3];
                    if (e & 0x40000000) {
                        dist_fold(ri[0], ri[1], ri[2], rj[0], rj[1], rj[2], p.L, d);
                        const float dx = (float)d[0], dy = (float)d[1], dz = (float)d[2];
                        const float r2 = dx * dx + dy * dy + dz * dz;
                        a0 += (double)pair_fast_t<SPEC21>(K, dx, dy, dz, r2, eix, eiy, eiz, ejx, ejy, ejz);
                    }
                    if (e < 0) {
                        dist_fold(rs[0], rs[1], rs[2], rj[0] * lam, rj[1] * lam, rj[2] * lam, Ls, d);
                        const float dx = (float)d[0], dy = (float)d[1], dz = (float)d[2];
                        const float r2 = dx * dx + dy * dy + dz * dz;
                        a1 += (double)pair_fast_t<SPEC21>(K, dx, dy, dz, r2, eix, eiy, eiz, ejx, ejy, ejz);
                    }
                }
                // move entries [m, qn) (at most 95 - 32) to the front
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
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
            a0 += __shfl_xor_sync(0xffffffffu, a0, o);
            a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        }
        if (lane == 0) {
            double u0 = a0, u1 = a1;
            if (p.k.coll_on) {
                const double ei[3] = {v.ox[i], v.oy[i], v.oz[i]};
                u0 += colloid_rod(p.k, ri, ei, p.L);
                u1 += colloid_rod(p.k, rs, ei, Ls);
            }
            e0[i] = u0;
            e1[i] = u1;
            double d[3];
            const double r2 = dist_fold(rs[0], rs[1], rs[2], 0.5 * Ls[0], 0.5 * Ls[1], 0.5 * Ls[2], Ls, d);
            hard[i] = !(r2 > p.k.coll_R * p.k.coll_R);
        }
        __syncwarp();
    }
}

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
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_energy_screen<true>, 128, 0) != cudaSuccess || b < 1) {
        cudaGetLastError();
        b = 4;
    }
    return b;
}

void launch_screen(const DevView &v, cudaStream_t s, double *e0, double *e1, int *hard, int grid, bool spec21)
{
    if (spec21) k_energy_screen<true><<<grid, 128, 0, s>>>(v, e0, e1, hard);
    else k_energy_screen<false><<<grid, 128, 0, s>>>(v, e0, e1, hard);
    launch_chunk_sums_volume(v, s, e0, e1, hard);
    k_screen_stage1<<<v.R, 256, 0, s>>>(v);
}

} // namespace lcmc
