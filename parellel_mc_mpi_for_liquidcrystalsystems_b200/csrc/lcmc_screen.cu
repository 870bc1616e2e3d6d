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

constexpr int SQ = 96;      // queue entries per warp: < 32 pending + 64 from one round of two chunks
constexpr int SC_CAP = 640; // staged particles per cell: the own cell and its 13 forward neighbours

// replica owning cell slot c (cell ranges are laid out in replica order)
__device__ __forceinline__ int replica_of_cell(const DevView &v, int c)
{
    int lo = 0, hi = v.R;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (v.rep[mid].cell_off <= c) lo = mid;
        else hi = mid;
    }
    return lo;
}

// One block per cell (grid-stride over every cell slot).  The own cell's
// particles and those of its 13 forward neighbours, the stencil slots
// u = 9 (dz + 1) + 3 (dy + 1) + dx + 1 > 13 (each unordered cell pair once under
// periodic wrap, >= 4 cells per axis), are staged in shared memory: FP64
// position, the orientation of the FP32 copy and an FP32 position relative to
// the own cell's origin for the prefilter.
// Own-cell particle k then pairs with staged slots k + 1 .. total - 1, warp by
// warp, through a compacted per-warp queue of in-cutoff pairs.
template <bool SPEC21>
__global__ void __launch_bounds__(128, 5) k_energy_screen(DevView v, double *e0, double *e1, int *hard)
{
    __shared__ double s_px[SC_CAP], s_py[SC_CAP], s_pz[SC_CAP];
    __shared__ float4 s_c4[SC_CAP]; // prefilter position (own cell origin), ux
    __shared__ float2 s_c2[SC_CAP]; // uy, uz
    __shared__ int s_start[14];     // first particle slot of stencil position o (slot 13 + o)
    __shared__ int s_pre[15];       // staged prefix per stencil position
    __shared__ int s_qj[4][SQ];     // queued staged slot; bit 30: in cutoff at V, bit 31: at V'
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const unsigned lt = (1u << lane) - 1u;
    for (int c = blockIdx.x; c < v.ctot; c += gridDim.x) {
        const int r = replica_of_cell(v, c);
        const Replica &p = v.rep[r];
        if (p.ensemble != 2 || p.da_kind != 2 || !p.use_fast) continue; // uniform across the block
        const int nc0 = p.nc[0], nc1 = p.nc[1], nc2 = p.nc[2];
        const int l = c - p.cell_off;
        if (l >= nc0 * nc1 * nc2) continue;
        const int cx = l % nc0, cy = (l / nc0) % nc1, cz = l / (nc0 * nc1);
        // stencil position o = lane: slot 13 + o (the own cell first)
        if (t < 32) {
            int st = 0, cnt = 0;
            if (lane < 14) {
                const int u = 13 + lane;
                int x = cx + u % 3 - 1, y = cy + (u / 3) % 3 - 1, z = cz + u / 9 - 1;
                x += x < 0 ? nc0 : (x >= nc0 ? -nc0 : 0);
                y += y < 0 ? nc1 : (y >= nc1 ? -nc1 : 0);
                z += z < 0 ? nc2 : (z >= nc2 ? -nc2 : 0);
                const int cn = p.cell_off + (z * nc1 + y) * nc0 + x;
                st = v.cell_start[cn];
                cnt = v.cell_start[cn + 1] - st;
            }
            int inc = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += y;
            }
            if (lane < 14) {
                s_start[lane] = st;
                s_pre[lane] = inc - cnt;
            }
            if (lane == 13) s_pre[14] = inc;
        }
        __syncthreads();
        const int na = s_pre[1], total = s_pre[14], g0 = s_start[0];
        if (total > SC_CAP) {
            if (t == 0) atomicOr(&v.stats[r].flags, F_STENCILCAP);
            __syncthreads();
            continue;
        }
        {
            const float wx = (float)p.w[0], wy = (float)p.w[1], wz = (float)p.w[2];
            for (int f = t; f < total; f += blockDim.x) {
                // largest stencil position whose prefix is <= f (empty positions never match)
                int o = 0, hi = 14;
                while (hi - o > 1) {
                    const int mid = (o + hi) >> 1;
                    if (s_pre[mid] <= f) o = mid;
                    else hi = mid;
                }
                const int u = 13 + o;
                const int g = s_start[o] + (f - s_pre[o]);
                s_px[f] = v.px[g];
                s_py[f] = v.py[g];
                s_pz[f] = v.pz[g];
                const float4 c4 = v.cl4[g]; // relative to its own cell's origin
                s_c4[f] = make_float4(c4.x + (float)(u % 3 - 1) * wx, c4.y + (float)((u / 3) % 3 - 1) * wy,
                                      c4.z + (float)(u / 9 - 1) * wz, c4.w);
                s_c2[f] = v.cl2[g];
            }
        }
        __syncthreads();

        const double lam = p.vol_lambda;
        const double Ls[3] = {__dmul_rn(p.L[0], lam), __dmul_rn(p.L[1], lam), __dmul_rn(p.L[2], lam)};
        const double rc2 = p.k.rc2;
        const float rc2f = (float)rc2, lam2f = (float)(lam * lam);
        const float lo = rc2f * (1.0f - 1e-5f), hi = rc2f * (1.0f + 1e-5f);
        const FastK K = fast_consts(p.k);
        for (int k = w; k < na; k += 4) {
            const double ri[3] = {s_px[k], s_py[k], s_pz[k]};
            const double rs[3] = {__dmul_rn(ri[0], lam), __dmul_rn(ri[1], lam), __dmul_rn(ri[2], lam)};
            const float4 ci = s_c4[k];
            const float2 ci2 = s_c2[k];
            const float eix = ci.w, eiy = ci2.x, eiz = ci2.y; // unit_f32 of the FP64 orientation
            double a0 = 0.0, a1 = 0.0;
            int qn = 0;
            // two chunks of 32 candidates per round
            for (int t0 = k + 1; t0 < total; t0 += 64) {
                bool any[2];
                int ent[2];
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int q = t0 + 32 * h + lane;
                    bool f0 = false, f1 = false;
                    if (q < total) {
                        const float4 cj = s_c4[q];
                        const float dx = cj.x - ci.x, dy = cj.y - ci.y, dz = cj.z - ci.z;
                        const float r2 = dx * dx + dy * dy + dz * dz, r2s = lam2f * r2;
                        double d[3];
                        if (r2 < lo) f0 = true;
                        else if (r2 <= hi) f0 = dist_fold(ri[0], ri[1], ri[2], s_px[q], s_py[q], s_pz[q], p.L, d) < rc2;
                        if (r2s < lo) f1 = true;
                        else if (r2s <= hi)
                            f1 = dist_fold(rs[0], rs[1], rs[2], __dmul_rn(s_px[q], lam), __dmul_rn(s_py[q], lam),
                                           __dmul_rn(s_pz[q], lam), Ls, d) < rc2;
                    }
                    any[h] = f0 || f1;
                    ent[h] = q | (f0 ? 0x40000000 : 0) | (f1 ? (int)0x80000000u : 0);
                }
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const unsigned b = __ballot_sync(0xffffffffu, any[h]);
                    if (any[h]) s_qj[w][qn + __popc(b & lt)] = ent[h];
                    qn += __popc(b);
                }
                __syncwarp();
                while (qn >= 32 || (qn > 0 && t0 + 64 >= total)) {
                    const int m = qn < 32 ? qn : 32;
                    if (lane < m) {
                        const int e = s_qj[w][lane];
                        const int jj = e & 0x3fffffff;
                        const double rj[3] = {s_px[jj], s_py[jj], s_pz[jj]};
                        const float ejx = s_c4[jj].w;
                        const float2 ej2 = s_c2[jj];
                        double d[3];
                        if (e & 0x40000000) {
                            dist_fold(ri[0], ri[1], ri[2], rj[0], rj[1], rj[2], p.L, d);
                            const float dx = (float)d[0], dy = (float)d[1], dz = (float)d[2];
                            const float r2 = dx * dx + dy * dy + dz * dz;
                            a0 += (double)pair_fast_t<SPEC21>(K, dx, dy, dz, r2, eix, eiy, eiz, ejx, ej2.x, ej2.y);
                        }
                        if (e < 0) {
                            dist_fold(rs[0], rs[1], rs[2], __dmul_rn(rj[0], lam), __dmul_rn(rj[1], lam),
                                      __dmul_rn(rj[2], lam), Ls, d);
                            const float dx = (float)d[0], dy = (float)d[1], dz = (float)d[2];
                            const float r2 = dx * dx + dy * dy + dz * dz;
                            a1 += (double)pair_fast_t<SPEC21>(K, dx, dy, dz, r2, eix, eiy, eiz, ejx, ej2.x, ej2.y);
                        }
                    }
                    // move entries [m, qn) (at most 95 - 32) to the front
                    int mv0 = 0, mv1 = 0;
                    if (m + lane < qn) mv0 = s_qj[w][m + lane];
                    if (m + 32 + lane < qn) mv1 = s_qj[w][m + 32 + lane];
                    __syncwarp();
                    if (m + lane < qn) s_qj[w][lane] = mv0;
                    if (m + 32 + lane < qn) s_qj[w][32 + lane] = mv1;
                    __syncwarp();
                    qn -= m;
                }
            }
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1) {
                a0 += __shfl_xor_sync(0xffffffffu, a0, o);
                a1 += __shfl_xor_sync(0xffffffffu, a1, o);
            }
            // colloid term at V (lane 0) and at V' with the hard-core test (lane 1)
            const int i = g0 + k;
            double uc = 0.0;
            if (lane < 2 && p.k.coll_on) {
                const double ei[3] = {v.ox[i], v.oy[i], v.oz[i]};
                uc = lane ? colloid_rod(p.k, rs, ei, Ls) : colloid_rod(p.k, ri, ei, p.L);
            }
            const double uc1 = __shfl_sync(0xffffffffu, uc, 1);
            if (lane == 0) {
                e0[i] = a0 + uc;
                e1[i] = a1 + uc1;
            } else if (lane == 1) {
                double d[3];
                const double r2 = dist_fold(rs[0], rs[1], rs[2], __dmul_rn(0.5, Ls[0]), __dmul_rn(0.5, Ls[1]),
                                            __dmul_rn(0.5, Ls[2]), Ls, d);
                hard[i] = !(r2 > __dmul_rn(p.k.coll_R, p.k.coll_R));
            }
            __syncwarp();
        }
        __syncthreads(); // the next cell's staging overwrites the staged particles
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
