// lcmc_volume_cells.cuh - energies U(V) and U(V') of every particle for an NPT
// volume move, one block per cell (no reference counterpart: the reference has
// no NPT move, MCnptColloid.c:3978; the pair term is pij_GB, 2607-2681).
//
// The own cell's particles and those of its 13 forward neighbours, the stencil
// slots u = 9 (dz + 1) + 3 (dy + 1) + dx + 1 > 13 (each unordered cell pair once
// under periodic wrap; >= 4 cells per axis), are staged in shared memory: FP64
// position, the orientation, and an FP32 position relative to the own cell's
// origin for the cutoff prefilter.  Own-cell particle k pairs with staged slots
// k + 1 .. total - 1, warp by warp (forward neighbours beyond the staging
// capacity are taken in further chunks, own-cell sums carried across); a pair is in the cutoff at V (V') when its
// FP32 distance is below rc^2 (1 - 1e-5) or, inside that band, when the FP64
// minimum-image distance of the (scaled) FP64 positions is below rc^2 -- the FP64
// kernel's pair set exactly.  In-cutoff pairs go through a compacted per-warp
// queue and are evaluated on the FP64 minimum-image vector:
//   EXACT = true   FP64 pair term (pair_energy64), FP64 orientations: the
//                  volume move's exact energies, any kernel's systems;
//   EXACT = false  FP32 pair term on that vector rounded to FP32 with the FP32
//                  copy's orientations: the delayed-acceptance screen U32
//                  (FP32-kernel systems, whose FP32 state copy exists).
// The scaled configuration is formed as the volume scaling forms it (positions
// r lambda, box L lambda, rounded products).  Sums are FP64 in a fixed order.
#pragma once
#include <cuda_runtime.h>

#include "lcmc_gb.cuh"
#include "lcmc_internal.h"
#include "lcmc_trial.cuh"

namespace lcmc {

constexpr int VC_Q = 96;    // queue entries per warp: < 32 pending + 64 from one round of two chunks
constexpr int VC_CAP = 576; // staged particles per chunk: the own cell and (part of) its forward neighbours
constexpr int VC_OWN = 256; // own-cell particles (more: F_CELLCAP)
constexpr int VC_REP = 64;  // replicas whose used cells are enumerated directly (more: every allocated cell)

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

// replicas whose volume energies this kernel computes this sweep
template <bool EXACT>
__device__ __forceinline__ bool volume_cells_serves(const Replica &p)
{
    if (p.ensemble != 2) return false;
    if (!EXACT) return p.da_kind == 2 && p.use_fast;
    if (p.da_on && !p.vol_stage1) return false; // screened out: no exact recompute
    return p.vol_cells && p.nc[0] >= 4 && p.nc[1] >= 4 && p.nc[2] >= 4;
}

template <bool EXACT>
struct VolCellsSmem {
    double px[VC_CAP], py[VC_CAP], pz[VC_CAP];
    float4 pre[VC_CAP];                                    // prefilter position (own cell origin); .w = FP32 ux
    float2 u2[EXACT ? 1 : VC_CAP];                         // FP32 uy, uz
    double ox[EXACT ? VC_CAP : 1], oy[EXACT ? VC_CAP : 1], oz[EXACT ? VC_CAP : 1]; // FP64 orientation
    double acc0[VC_OWN], acc1[VC_OWN];                     // own-cell sums carried between chunks
    double cu0[VC_OWN], cu1[VC_OWN];                       // own-cell colloid terms at V, V'
    int ucell[VC_REP + 1];                                 // used-cell prefix over the replicas
    int start[14];                                         // first particle slot of stencil position o (slot 13 + o)
    int pre_n[15];                                         // particle prefix per stencil position
    int qj[4][VC_Q]; // queued staged slot; bit 30: in cutoff at V, bit 31: at V'
};

template <bool EXACT, bool SPEC21>
__global__ void __launch_bounds__(128, EXACT ? 4 : 5) k_volume_cells(DevView v, double *e0, double *e1, int *hard)
{
    __shared__ VolCellsSmem<EXACT> sm;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const unsigned lt = (1u << lane) - 1u;
    // the cells this kernel serves: the used cells (nc0 nc1 nc2 of the nc_max^3
    // allocated) of the replicas it serves, enumerated through a prefix
    const bool direct = v.R <= VC_REP;
    if (direct && t == 0) {
        int acc = 0;
        for (int r = 0; r < v.R; r++) {
            sm.ucell[r] = acc;
            const Replica &p = v.rep[r];
            if (volume_cells_serves<EXACT>(p)) acc += p.nc[0] * p.nc[1] * p.nc[2];
        }
        sm.ucell[v.R] = acc;
    }
    __syncthreads();
    const int ncells = direct ? sm.ucell[v.R] : v.ctot;
    for (int e = blockIdx.x; e < ncells; e += gridDim.x) {
        int r, l;
        if (direct) { // replica: the largest r with ucell[r] <= e (replicas it does not serve are empty)
            int lo_ = 0, hi_ = v.R;
            while (hi_ - lo_ > 1) {
                const int mid = (lo_ + hi_) >> 1;
                if (sm.ucell[mid] <= e) lo_ = mid;
                else hi_ = mid;
            }
            r = lo_;
            l = e - sm.ucell[r];
        } else {
            r = replica_of_cell(v, e);
            l = e - v.rep[r].cell_off;
        }
        const Replica &p = v.rep[r];
        if (!volume_cells_serves<EXACT>(p)) continue; // uniform across the block
        const int nc0 = p.nc[0], nc1 = p.nc[1], nc2 = p.nc[2];
        if (l >= nc0 * nc1 * nc2) continue;
        const int c = p.cell_off + l;
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
                sm.start[lane] = st;
                sm.pre_n[lane] = inc - cnt;
            }
            if (lane == 13) sm.pre_n[14] = inc;
        }
        __syncthreads();
        const int na = sm.pre_n[1], nall = sm.pre_n[14], g0 = sm.start[0];
        if (na > VC_OWN) {
            if (t == 0) atomicOr(&v.stats[r].flags, F_CELLCAP);
            __syncthreads();
            continue;
        }
        const int fcap = VC_CAP - na; // forward particles per chunk
        const double lam = p.vol_lambda;
        const double Ls[3] = {__dmul_rn(p.L[0], lam), __dmul_rn(p.L[1], lam), __dmul_rn(p.L[2], lam)};
        const double rc2 = p.k.rc2;
        const float rc2f = (float)rc2, lam2f = (float)(lam * lam);
        const float lo = rc2f * (1.0f - 1e-5f), hi = rc2f * (1.0f + 1e-5f);
        const FastK K = fast_consts(p.k);
        const float wx = (float)p.w[0], wy = (float)p.w[1], wz = (float)p.w[2];
        // colloid term of own-cell particle k at V (thread 2k) and at V' with the
        // hard-core test (thread 2k + 1)
        if (t < 2 * na) {
            const int k = t >> 1, i = g0 + k;
            const double ri[3] = {v.px[i], v.py[i], v.pz[i]};
            double uc = 0.0;
            if (t & 1) {
                const double rs[3] = {__dmul_rn(ri[0], lam), __dmul_rn(ri[1], lam), __dmul_rn(ri[2], lam)};
                if (p.k.coll_on) {
                    const double ei[3] = {v.ox[i], v.oy[i], v.oz[i]};
                    uc = colloid_rod(p.k, rs, ei, Ls);
                }
                double d[3];
                const double r2 = dist_fold(rs[0], rs[1], rs[2], __dmul_rn(0.5, Ls[0]), __dmul_rn(0.5, Ls[1]),
                                            __dmul_rn(0.5, Ls[2]), Ls, d);
                hard[i] = !(r2 > __dmul_rn(p.k.coll_R, p.k.coll_R));
                sm.cu1[k] = uc;
            } else {
                if (p.k.coll_on) {
                    const double ei[3] = {v.ox[i], v.oy[i], v.oz[i]};
                    uc = colloid_rod(p.k, ri, ei, p.L);
                }
                sm.cu0[k] = uc;
            }
        }
        for (int cs = na; cs == na || cs < nall; cs += fcap) {
            const bool first = cs == na, last = cs + fcap >= nall;
            const int total = na + min(fcap, nall - cs); // staged slots of this chunk
            // own cell (first chunk) at slots [0, na), forward particles [cs, cs + fcap) after it
            for (int s_ = first ? t : na + t; s_ < total; s_ += blockDim.x) {
                const int f = s_ < na ? s_ : cs + (s_ - na); // particle index over the stencil positions
                // largest stencil position whose prefix is <= f (empty positions never match)
                int o = 0, hi_ = 14;
                while (hi_ - o > 1) {
                    const int mid = (o + hi_) >> 1;
                    if (sm.pre_n[mid] <= f) o = mid;
                    else hi_ = mid;
                }
                const int u = 13 + o;
                const int g = sm.start[o] + (f - sm.pre_n[o]);
                const double x = v.px[g], y = v.py[g], z = v.pz[g];
                sm.px[s_] = x;
                sm.py[s_] = y;
                sm.pz[s_] = z;
                const float ox_ = (float)(u % 3 - 1) * wx, oy_ = (float)((u / 3) % 3 - 1) * wy,
                            oz_ = (float)(u / 9 - 1) * wz;
                if (EXACT) {
                    // position relative to the particle's own cell origin, as the FP32
                    // state copy forms it, plus the stencil offset
                    int ux_ = cx + u % 3 - 1, uy_ = cy + (u / 3) % 3 - 1, uz_ = cz + u / 9 - 1;
                    ux_ += ux_ < 0 ? nc0 : (ux_ >= nc0 ? -nc0 : 0);
                    uy_ += uy_ < 0 ? nc1 : (uy_ >= nc1 ? -nc1 : 0);
                    uz_ += uz_ < 0 ? nc2 : (uz_ >= nc2 ? -nc2 : 0);
                    const double lx = fold_rel(x, p.shift[0] + (double)ux_ * p.w[0], 0.5 * p.w[0], p.L[0], 1.0 / p.L[0]);
                    const double ly = fold_rel(y, p.shift[1] + (double)uy_ * p.w[1], 0.5 * p.w[1], p.L[1], 1.0 / p.L[1]);
                    const double lz = fold_rel(z, p.shift[2] + (double)uz_ * p.w[2], 0.5 * p.w[2], p.L[2], 1.0 / p.L[2]);
                    sm.pre[s_] = make_float4((float)lx + ox_, (float)ly + oy_, (float)lz + oz_, 0.0f);
                    sm.ox[s_] = v.ox[g];
                    sm.oy[s_] = v.oy[g];
                    sm.oz[s_] = v.oz[g];
                } else {
                    const float4 c4 = v.cl4[g]; // relative to its own cell's origin
                    sm.pre[s_] = make_float4(c4.x + ox_, c4.y + oy_, c4.z + oz_, c4.w);
                    sm.u2[s_] = v.cl2[g];
                }
            }
            __syncthreads();

            for (int k = w; k < na; k += 4) {
                const double ri[3] = {sm.px[k], sm.py[k], sm.pz[k]};
                const double rs[3] = {__dmul_rn(ri[0], lam), __dmul_rn(ri[1], lam), __dmul_rn(ri[2], lam)};
                const float4 ci = sm.pre[k];
                double a0 = 0.0, a1 = 0.0;
                int qn = 0;
                // two chunks of 32 candidates per round
                for (int t0 = first ? k + 1 : na; t0 < total; t0 += 64) {
                    bool any[2];
                    int ent[2];
    #pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const int q = t0 + 32 * h + lane;
                        bool f0 = false, f1 = false, b0 = false, b1 = false;
                        if (q < total) {
                            const float4 cj = sm.pre[q];
                            const float dx = cj.x - ci.x, dy = cj.y - ci.y, dz = cj.z - ci.z;
                            const float r2 = dx * dx + dy * dy + dz * dz, r2s = lam2f * r2;
                            f0 = r2 < lo;
                            f1 = r2s < lo;
                            b0 = !f0 && r2 <= hi;
                            b1 = !f1 && r2s <= hi;
                        }
                        // within 1e-5 of rc^2: the FP64 distance decides (rare; warp-uniform branch)
                        if (__any_sync(0xffffffffu, b0 || b1)) {
                            double d[3];
                            if (b0) f0 = dist_fold(ri[0], ri[1], ri[2], sm.px[q], sm.py[q], sm.pz[q], p.L, d) < rc2;
                            if (b1)
                                f1 = dist_fold(rs[0], rs[1], rs[2], __dmul_rn(sm.px[q], lam), __dmul_rn(sm.py[q], lam),
                                               __dmul_rn(sm.pz[q], lam), Ls, d) < rc2;
                        }
                        any[h] = f0 || f1;
                        ent[h] = q | (f0 ? 0x40000000 : 0) | (f1 ? (int)0x80000000u : 0);
                    }
    #pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const unsigned b = __ballot_sync(0xffffffffu, any[h]);
                        if (any[h]) sm.qj[w][qn + __popc(b & lt)] = ent[h];
                        qn += __popc(b);
                    }
                    __syncwarp();
                    while (qn >= 32 || (qn > 0 && t0 + 64 >= total)) {
                        const int m = qn < 32 ? qn : 32;
                        if (lane < m) {
                            const int e = sm.qj[w][lane];
                            const int jj = e & 0x3fffffff;
                            const double rj[3] = {sm.px[jj], sm.py[jj], sm.pz[jj]};
                            double d[3];
                            if (EXACT) {
                                const double ei[3] = {sm.ox[k], sm.oy[k], sm.oz[k]};
                                const double ej[3] = {sm.ox[jj], sm.oy[jj], sm.oz[jj]};
                                if (e & 0x40000000) {
                                    const double r2 = dist_fold(ri[0], ri[1], ri[2], rj[0], rj[1], rj[2], p.L, d);
                                    a0 += pair_energy64(p.k, r2, d, ei, ej);
                                }
                                if (e < 0) {
                                    const double r2 = dist_fold(rs[0], rs[1], rs[2], __dmul_rn(rj[0], lam),
                                                                __dmul_rn(rj[1], lam), __dmul_rn(rj[2], lam), Ls, d);
                                    a1 += pair_energy64(p.k, r2, d, ei, ej);
                                }
                            } else {
                                const float eix = ci.w, eiy = sm.u2[k].x, eiz = sm.u2[k].y;
                                const float ejx = sm.pre[jj].w;
                                const float2 ej2 = sm.u2[jj];
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
                        }
                        // move entries [m, qn) (at most 95 - 32) to the front
                        int mv0 = 0, mv1 = 0;
                        if (m + lane < qn) mv0 = sm.qj[w][m + lane];
                        if (m + 32 + lane < qn) mv1 = sm.qj[w][m + 32 + lane];
                        __syncwarp();
                        if (m + lane < qn) sm.qj[w][lane] = mv0;
                        if (m + 32 + lane < qn) sm.qj[w][32 + lane] = mv1;
                        __syncwarp();
                        qn -= m;
                    }
                }
#pragma unroll
                for (int o = 16; o >= 1; o >>= 1) {
                    a0 += __shfl_xor_sync(0xffffffffu, a0, o);
                    a1 += __shfl_xor_sync(0xffffffffu, a1, o);
                }
                if (!first) {
                    a0 = sm.acc0[k] + a0;
                    a1 = sm.acc1[k] + a1;
                }
                if (!last) {
                    if (lane == 0) {
                        sm.acc0[k] = a0;
                        sm.acc1[k] = a1;
                    }
                    continue;
                }
                if (lane == 0) {
                    const int i = g0 + k;
                    e0[i] = a0 + sm.cu0[k];
                    e1[i] = a1 + sm.cu1[k];
                }
            }
            __syncthreads(); // the next chunk or cell overwrites the staged particles
        }
    }
}

} // namespace lcmc
