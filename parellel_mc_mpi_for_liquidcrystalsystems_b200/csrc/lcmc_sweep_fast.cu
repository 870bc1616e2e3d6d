// lcmc_sweep_fast.cu - FP32 checkerboard phase (production path).
//
// One CTA per active cell (grid-stride over all active cells of all replicas).
// Within a colour phase the 26 neighbour cells of an active cell do not move
// (they have other colours), and each particle of the active cell is attempted
// exactly once, from its phase-start state, with a trial state that depends
// only on its own Philox draws (precomputed for the whole sweep by the rebin
// gather, k_gather).  So for every particle k the energy against the 26 static
// cells, old and new, is independent of the other attempts:
//
//   dE_k = [S_new(k) - S_old(k)]                            static cells
//        + sum_{m != k} [phi(n_k, o_m) - phi(o_k, o_m)]     in-cell, old states
//        + sum_{m < k, m accepted} c(k, m)                  in-cell corrections
//        + U_coll(n_k) - U_coll(o_k)
//   c(k, m) = [phi(n_k, n_m) - phi(o_k, n_m)] - [phi(n_k, o_m) - phi(o_k, o_m)]
//
// which is exactly E_new - E_old of attempt_monte_carlo_move (MCnptColloid.c:
// 2491-2563) for the sequential in-cell order (ascending id).  Only the short
// scan over the accept decisions is sequential.
//
// Phases per cell:
//   1 stencil  27 cells (>= 4 cells per axis, no duplicates)
//   2 active   phase-start state and precomputed trial of each particle of the
//              cell, coordinates relative to the cell origin (FP32)
//   3 staging  the 26 static cells -> shared memory (float4 x,y,z,ux + float2
//              uy,uz), folded across the periodic seam, pruned to the cell box
//              grown by rc + max_displacement/2; warp w compacts its quarter of
//              the candidates into its own segment (no block barrier per round)
//   4 tasks    warps take tasks from a shared queue:
//              particle task k: cutoff test of all staged candidates against
//                k's old position with radius rc + |displacement| (covers old
//                and new state), ballot compaction into the warp's list, then
//                FP32 Gay-Berne for old and new state over the list, lane sums
//                in FP64
//              pair task: 32 unordered in-cell pairs, 4 terms each
//              (old/new x old/new), differences formed in FP64
//   5 sums     warp per particle: in-cell row sums -> dE before corrections
//   6 scan     warp 0: Metropolis decisions in id order with the corrections
//   7 write    accepted trial states to the FP64 master arrays
#include <cuda_runtime.h>

#include "lcmc_gb.cuh"
#include "lcmc_internal.h"
#include "lcmc_rng.cuh"

namespace lcmc {

__device__ __forceinline__ int find_replica_f(const int *off, int R, int a)
{
    int lo = 0, hi = R;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (off[mid] <= a) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ int tri(int p, int q) { return (q * (q - 1)) / 2 + p; } // p < q

// Coordinate relative to the active cell's origin o, folded by whole periods
// into the window of the stencil cell it belongs to (centre cexp = (d + 1/2) w
// for stencil offset d).  A stored coordinate may lie on either side of the
// shifted periodic seam (cells that straddle it, or particles that crossed it
// earlier in the sweep); the fold is exact because every particle stays within
// w/2 + max_displacement/2 of its cell centre and w <= L/4.
__device__ __forceinline__ double fold_rel(double x, double o, double cexp, double L, double invL)
{
    const double r = x - o;
    return r - L * rint((r - cexp) * invL);
}

template <int NT, int AMAX, int SEG, int LW>
struct FastSmem {
    static constexpr int NW = NT / 32;
    static constexpr int NPAIR = AMAX * (AMAX - 1) / 2;
    float4 cpos[NW * SEG];     // x, y, z, ux of the static candidates (segment per warp)
    float2 cori[NW * SEG];     // uy, uz
    float pCA[NPAIR], pBA[NPAIR], pcm[NPAIR]; // in-cell: C-A, B-A, (D-C)-(B-A)
    float ax[AMAX], ay[AMAX], az[AMAX], aux[AMAX], auy[AMAX], auz[AMAX]; // old, relative
    float bx[AMAX], by[AMAX], bz[AMAX], bux[AMAX], buy[AMAX], buz[AMAX]; // new, relative
    float rad2[AMAX];
    double Sold[AMAX], Snew[AMAX], dEk[AMAX];
    int acc[AMAX];
    unsigned short wlist[NW][LW];
    int st_start[27], st_cnt[27], st_pre[28];
    int segcnt[NW];
    int task;
    int overflow;
    unsigned long long pairs;
};

__device__ __forceinline__ FastK fast_consts(const GBConsts &k)
{
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
    return K;
}

__device__ __forceinline__ void cell_failed(const DevView &v, int r, int cell, int flag)
{
    atomicOr(&v.stats[r].flags, flag);
    v.cell_e0[cell] = 0.0;
    v.cell_n0[cell] = 0;
    v.cell_n1[cell] = 0;
    v.cell_pairs[cell] = 0ull;
    v.cell_cands[cell] = 0ull;
}

template <int NT, int AMAX, int SEG, int LW, bool SPEC21>
__global__ void __launch_bounds__(NT, 5) k_phase_fast(DevView v, int ci)
{
    using SM = FastSmem<NT, AMAX, SEG, LW>;
    constexpr int NW = SM::NW;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SM &sm = *reinterpret_cast<SM *>(smem_raw);
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const int *off = v.act_off + ci * (v.R + 1);
    const int total = off[v.R];

    for (int a = blockIdx.x; a < total; a += gridDim.x) {
        const int r = find_replica_f(off, v.R, a);
        const Replica &p = v.rep[r];
        if (!p.use_fast) continue; // uniform across the block
        const int col = p.perm[ci];
        const int nc0 = p.nc[0], nc1 = p.nc[1], nc2 = p.nc[2];
        const int nax = nc0 >> 1, nay = nc1 >> 1;
        int loc = a - off[r];
        const int cx = 2 * (loc % nax) + (col & 1);
        loc /= nax;
        const int cy = 2 * (loc % nay) + ((col >> 1) & 1);
        const int cz = 2 * (loc / nay) + ((col >> 2) & 1);
        const int cell = p.cell_off + (cz * nc1 + cy) * nc0 + cx;
        const double w0 = p.w[0], w1 = p.w[1], w2 = p.w[2];
        const double L0 = p.L[0], L1 = p.L[1], L2 = p.L[2];
        const double iL0 = 1.0 / L0, iL1 = 1.0 / L1, iL2 = 1.0 / L2;
        const double o0 = p.shift[0] + (double)cx * w0;
        const double o1 = p.shift[1] + (double)cy * w1;
        const double o2 = p.shift[2] + (double)cz * w2;
        const FastK K = fast_consts(p.k);

        // ---- 1 stencil ----
        if (t < 27) {
            int x = cx + t % 3 - 1, y = cy + (t / 3) % 3 - 1, z = cz + t / 9 - 1;
            x += x < 0 ? nc0 : (x >= nc0 ? -nc0 : 0);
            y += y < 0 ? nc1 : (y >= nc1 ? -nc1 : 0);
            z += z < 0 ? nc2 : (z >= nc2 ? -nc2 : 0);
            const int c = p.cell_off + (z * nc1 + y) * nc0 + x;
            const int s = v.cell_start[c];
            sm.st_start[t] = s;
            sm.st_cnt[t] = v.cell_start[c + 1] - s;
        }
        if (t == 0) {
            sm.overflow = 0;
            sm.pairs = 0ull;
            sm.task = 0;
        }
        __syncthreads();
        if (t < 32) { // prefix over the 26 static cells (slot 13 = the active cell excluded)
            int c = (t < 27 && t != 13) ? sm.st_cnt[t] : 0;
            int inc = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += y;
            }
            if (t < 27) sm.st_pre[t] = inc - c;
            if (t == 26) sm.st_pre[27] = inc;
        }
        __syncthreads();
        const int na = sm.st_cnt[13];
        const int g0 = sm.st_start[13];
        const int S26 = sm.st_pre[27];
        if (na > AMAX) {
            if (t == 0) cell_failed(v, r, cell, F_CELLCAP);
            for (int k = t; k < na; k += NT) v.outcome[p.p_off + v.id[g0 + k]] = 0;
            __syncthreads();
            continue;
        }

        // ---- 2 active particles: phase-start state and precomputed trial ----
        const float rcf = (float)p.k.rc;
        for (int k = t; k < na; k += NT) {
            const int g = g0 + k;
            const double qx = fold_rel(v.px[g], o0, 0.5 * w0, L0, iL0);
            const double qy = fold_rel(v.py[g], o1, 0.5 * w1, L1, iL1);
            const double qz = fold_rel(v.pz[g], o2, 0.5 * w2, L2, iL2);
            const double ex = v.ox[g], ey = v.oy[g], ez = v.oz[g];
            const float en = rsqrtf((float)(ex * ex + ey * ey + ez * ez));
            const float dx = v.tdx[g], dy = v.tdy[g], dz = v.tdz[g];
            sm.ax[k] = (float)qx;
            sm.ay[k] = (float)qy;
            sm.az[k] = (float)qz;
            sm.aux[k] = (float)ex * en;
            sm.auy[k] = (float)ey * en;
            sm.auz[k] = (float)ez * en;
            sm.bx[k] = (float)qx + dx;
            sm.by[k] = (float)qy + dy;
            sm.bz[k] = (float)qz + dz;
            sm.bux[k] = (float)v.tux[g];
            sm.buy[k] = (float)v.tuy[g];
            sm.buz[k] = (float)v.tuz[g];
            const float rr = rcf + sqrtf(dx * dx + dy * dy + dz * dz) + 1e-3f;
            sm.rad2[k] = v.thard[g] ? -1.0f : rr * rr;
        }

        // ---- 3 staging: warp w takes a contiguous quarter of the 26 static cells'
        //      particles and compacts the kept ones into its own segment ----
        {
            const float wx = (float)w0, wy = (float)w1, wz = (float)w2;
            const float hb = 0.5f * (float)p.k.max_disp + 1e-3f;
            const float prune2 = K.rc2 * 1.0002f + 1e-3f;
            const int fb = (int)(((long long)S26 * w) / NW), fe = (int)(((long long)S26 * (w + 1)) / NW);
            int cnt = 0;
            for (int base = fb; base < fe; base += 32) {
                const int f = base + lane;
                bool keep = false;
                float x = 0, y = 0, z = 0, ux = 0, uy = 0, uz = 0;
                if (f < fe) {
                    // largest stencil slot whose prefix is <= f (slot 13 has an empty range;
                    // an empty slot's prefix is the end of the previous range, so it is never picked)
                    int s = 0, hi = 27;
                    while (hi - s > 1) {
                        const int mid = (s + hi) >> 1;
                        if (sm.st_pre[mid] <= f) s = mid;
                        else hi = mid;
                    }
                    const int g = sm.st_start[s] + (f - sm.st_pre[s]);
                    // stencil offset of slot s is (s % 3, s / 3 % 3, s / 9) - 1
                    x = (float)fold_rel(v.px[g], o0, ((double)(s % 3) - 0.5) * w0, L0, iL0);
                    y = (float)fold_rel(v.py[g], o1, ((double)((s / 3) % 3) - 0.5) * w1, L1, iL1);
                    z = (float)fold_rel(v.pz[g], o2, ((double)(s / 9) - 0.5) * w2, L2, iL2);
                    const float qx = fmaxf(fmaxf(-hb - x, x - (wx + hb)), 0.0f);
                    const float qy = fmaxf(fmaxf(-hb - y, y - (wy + hb)), 0.0f);
                    const float qz = fmaxf(fmaxf(-hb - z, z - (wz + hb)), 0.0f);
                    keep = qx * qx + qy * qy + qz * qz < prune2;
                    if (keep) {
                        const double ex = v.ox[g], ey = v.oy[g], ez = v.oz[g];
                        const float in = rsqrtf((float)(ex * ex + ey * ey + ez * ez));
                        ux = (float)ex * in;
                        uy = (float)ey * in;
                        uz = (float)ez * in;
                    }
                }
                const unsigned bal = __ballot_sync(0xffffffffu, keep);
                const int pos = cnt + __popc(bal & lt);
                if (keep && pos < SEG) {
                    sm.cpos[w * SEG + pos] = make_float4(x, y, z, ux);
                    sm.cori[w * SEG + pos] = make_float2(uy, uz);
                }
                cnt += __popc(bal);
            }
            if (lane == 0) {
                sm.segcnt[w] = cnt < SEG ? cnt : SEG;
                if (cnt > SEG) sm.overflow = 2;
            }
        }
        __syncthreads();
        if (sm.overflow) {
            if (t == 0) cell_failed(v, r, cell, F_STENCILCAP);
            for (int k = t; k < na; k += NT) v.outcome[p.p_off + v.id[g0 + k]] = 0;
            __syncthreads();
            continue;
        }
        int segc[NW];
#pragma unroll
        for (int i = 0; i < NW; i++) segc[i] = sm.segcnt[i];

        // ---- 4 task queue: particle tasks (test + pair sums) and in-cell pair tasks ----
        const int npair = na * (na - 1) / 2;
        const int ntask = na + (npair + 31) / 32;
        unsigned long long npairs = 0ull;
        for (;;) {
            int task = 0;
            if (lane == 0) task = atomicAdd(&sm.task, 1);
            task = __shfl_sync(0xffffffffu, task, 0);
            if (task >= ntask) break;
            if (task < na) {
                const int k = task;
                const float R2 = sm.rad2[k];
                double so = 0.0, sn = 0.0;
                int np = 0;
                if (R2 > 0.0f) {
                    const float xo = sm.ax[k], yo = sm.ay[k], zo = sm.az[k];
                    int cnt = 0;
#pragma unroll
                    for (int sg = 0; sg < NW; sg++) {
                        const int n = segc[sg];
                        for (int base = 0; base < n; base += 32) {
                            const int j = base + lane;
                            bool pass = false;
                            if (j < n) {
                                const float4 c = sm.cpos[sg * SEG + j];
                                const float dx = c.x - xo, dy = c.y - yo, dz = c.z - zo;
                                pass = dx * dx + dy * dy + dz * dz < R2;
                            }
                            const unsigned bal = __ballot_sync(0xffffffffu, pass);
                            const int pos = cnt + __popc(bal & lt);
                            if (pass && pos < LW) sm.wlist[w][pos] = (unsigned short)(sg * SEG + j);
                            cnt += __popc(bal);
                        }
                    }
                    if (cnt > LW) {
                        if (lane == 0) sm.overflow = 1;
                        cnt = LW;
                    }
                    __syncwarp();
                    const float uox = sm.aux[k], uoy = sm.auy[k], uoz = sm.auz[k];
                    const float xn = sm.bx[k], yn = sm.by[k], zn = sm.bz[k];
                    const float unx = sm.bux[k], uny = sm.buy[k], unz = sm.buz[k];
                    // FP64 lane sums: the 1e9 overlap clamp is exact in FP32 and
                    // must cancel exactly between the old and the new sum
                    for (int q = lane; q < cnt; q += 32) {
                        const int j = sm.wlist[w][q];
                        const float4 c = sm.cpos[j];
                        const float2 u = sm.cori[j];
                        float dx = c.x - xo, dy = c.y - yo, dz = c.z - zo;
                        float r2 = dx * dx + dy * dy + dz * dz;
                        const float e0 = pair_fast_t<SPEC21>(K, dx, dy, dz, r2, uox, uoy, uoz, c.w, u.x, u.y);
                        const bool in0 = r2 < K.rc2;
                        dx = c.x - xn;
                        dy = c.y - yn;
                        dz = c.z - zn;
                        r2 = dx * dx + dy * dy + dz * dz;
                        const float e1 = pair_fast_t<SPEC21>(K, dx, dy, dz, r2, unx, uny, unz, c.w, u.x, u.y);
                        const bool in1 = r2 < K.rc2;
                        so += in0 ? (double)e0 : 0.0;
                        sn += in1 ? (double)e1 : 0.0;
                        np += (int)in0 + (int)in1;
                    }
                    __syncwarp();
                }
#pragma unroll
                for (int o = 16; o >= 1; o >>= 1) {
                    so += __shfl_xor_sync(0xffffffffu, so, o);
                    sn += __shfl_xor_sync(0xffffffffu, sn, o);
                    np += __shfl_xor_sync(0xffffffffu, np, o);
                }
                if (lane == 0) {
                    sm.Sold[k] = so;
                    sm.Snew[k] = sn;
                }
                npairs += (unsigned long long)np;
            } else {
                const int idx = (task - na) * 32 + lane;
                int npin = 0;
                if (idx < npair) {
                    int q = (int)((1.0f + sqrtf(1.0f + 8.0f * (float)idx)) * 0.5f);
                    while (q * (q - 1) / 2 > idx) q--;
                    while ((q + 1) * q / 2 <= idx) q++;
                    const int pp = idx - q * (q - 1) / 2;
                    float A, B, Cc, D;
                    {
                        float dx = sm.ax[q] - sm.ax[pp], dy = sm.ay[q] - sm.ay[pp], dz = sm.az[q] - sm.az[pp];
                        float r2 = dx * dx + dy * dy + dz * dz;
                        A = pair_fast_t<SPEC21>(K, dx, dy, dz, r2, sm.aux[pp], sm.auy[pp], sm.auz[pp], sm.aux[q],
                                                sm.auy[q], sm.auz[q]);
                        A = r2 < K.rc2 ? A : 0.0f;
                        npin += 2 * (r2 < K.rc2);
                    }
                    {
                        float dx = sm.bx[q] - sm.ax[pp], dy = sm.by[q] - sm.ay[pp], dz = sm.bz[q] - sm.az[pp];
                        float r2 = dx * dx + dy * dy + dz * dz;
                        B = pair_fast_t<SPEC21>(K, dx, dy, dz, r2, sm.aux[pp], sm.auy[pp], sm.auz[pp], sm.bux[q],
                                                sm.buy[q], sm.buz[q]);
                        B = r2 < K.rc2 ? B : 0.0f;
                        npin += (r2 < K.rc2);
                    }
                    {
                        float dx = sm.ax[q] - sm.bx[pp], dy = sm.ay[q] - sm.by[pp], dz = sm.az[q] - sm.bz[pp];
                        float r2 = dx * dx + dy * dy + dz * dz;
                        Cc = pair_fast_t<SPEC21>(K, dx, dy, dz, r2, sm.bux[pp], sm.buy[pp], sm.buz[pp], sm.aux[q],
                                                 sm.auy[q], sm.auz[q]);
                        Cc = r2 < K.rc2 ? Cc : 0.0f;
                        npin += (r2 < K.rc2);
                    }
                    {
                        float dx = sm.bx[q] - sm.bx[pp], dy = sm.by[q] - sm.by[pp], dz = sm.bz[q] - sm.bz[pp];
                        float r2 = dx * dx + dy * dy + dz * dz;
                        D = pair_fast_t<SPEC21>(K, dx, dy, dz, r2, sm.bux[pp], sm.buy[pp], sm.buz[pp], sm.bux[q],
                                                sm.buy[q], sm.buz[q]);
                        D = r2 < K.rc2 ? D : 0.0f;
                    }
                    // differences in FP64 (exact cancellation of the overlap clamp), then rounded
                    const double a = A, b = B, c = Cc, d = D;
                    sm.pCA[idx] = (float)(c - a);
                    sm.pBA[idx] = (float)(b - a);
                    sm.pcm[idx] = (float)((d - c) - (b - a));
                }
#pragma unroll
                for (int o = 16; o >= 1; o >>= 1) npin += __shfl_xor_sync(0xffffffffu, npin, o);
                npairs += (unsigned long long)npin;
            }
        }
        if (lane == 0 && npairs) atomicAdd(&sm.pairs, npairs);
        __syncthreads();
        if (sm.overflow) {
            if (t == 0) cell_failed(v, r, cell, F_LISTCAP);
            for (int k = t; k < na; k += NT) v.outcome[p.p_off + v.id[g0 + k]] = 0;
            __syncthreads();
            continue;
        }

        // ---- 5 warp per particle: in-cell row sums -> dE before the corrections ----
        for (int k = w; k < na; k += NW) {
            double s = 0.0;
            for (int m = lane; m < na; m += 32) {
                if (m < k) s += (double)sm.pBA[tri(m, k)];     // phi(n_k, o_m) - phi(o_k, o_m), k later
                else if (m > k) s += (double)sm.pCA[tri(k, m)]; // k earlier in the pair
            }
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) sm.dEk[k] = (sm.Snew[k] - sm.Sold[k]) + s + v.tdU[g0 + k];
        }
        __syncthreads();

        // ---- 6 sequential Metropolis scan (warp 0) ----
        if (w == 0) {
            double e0 = lane < na ? sm.dEk[lane] : 0.0;
            double e1 = lane + 32 < na ? sm.dEk[lane + 32] : 0.0;
            const double lu0 = lane < na ? v.tlu[g0 + lane] : 0.0;
            const double lu1 = lane + 32 < na ? v.tlu[g0 + lane + 32] : 0.0;
            const double beta = p.k.beta;
            double dsum = 0.0;
            int nacc = 0, nhard = 0;
            for (int m = 0; m < na; m++) {
                const int own = m & 31;
                const double val = __shfl_sync(0xffffffffu, m < 32 ? e0 : e1, own);
                const double lum = __shfl_sync(0xffffffffu, m < 32 ? lu0 : lu1, own);
                const int hd = sm.rad2[m] < 0.0f;
                const bool acc = !hd && ((val <= 0.0) || (lum <= -beta * val));
                nhard += hd;
                if (acc) {
                    dsum += val;
                    nacc++;
                    if (lane > m && lane < na) e0 += (double)sm.pcm[tri(m, lane)];
                    if (lane + 32 > m && lane + 32 < na) e1 += (double)sm.pcm[tri(m, lane + 32)];
                }
                if (lane == 0) sm.acc[m] = acc;
            }
            if (lane == 0) {
                if (!(dsum - dsum == 0.0)) atomicOr(&v.stats[r].flags, F_NONFINITE);
                v.cell_e0[cell] = dsum;
                v.cell_n0[cell] = nacc;
                v.cell_n1[cell] = nhard;
                v.cell_pairs[cell] = sm.pairs;
                v.cell_cands[cell] = (unsigned long long)na * (unsigned long long)(S26 + na - 1);
            }
        }
        __syncthreads();

        // ---- 7 write-back ----
        for (int k = t; k < na; k += NT) {
            const int g = g0 + k;
            const int acc = sm.acc[k];
            if (acc) {
                v.px[g] = v.tnx[g];
                v.py[g] = v.tny[g];
                v.pz[g] = v.tnz[g];
                v.ox[g] = v.tux[g];
                v.oy[g] = v.tuy[g];
                v.oz[g] = v.tuz[g];
            }
            v.outcome[p.p_off + v.id[g]] = v.thard[g] ? 2 : acc;
        }
        __syncthreads();
    }
}

} // namespace lcmc

#include "lcmc_launch.h"

namespace lcmc {

// (threads, active capacity, staged candidates per warp segment, per-warp list capacity)
static const FastVariant kVariants[] = {{128, 48, 192, 256}, {128, 64, 288, 384}};

int fast_variant_count() { return (int)(sizeof(kVariants) / sizeof(kVariants[0])); }
FastVariant fast_variant(int i) { return kVariants[i]; }

template <int NT, int AMAX, int SEG, int LW, bool S21>
static void launch_v(const DevView &v, cudaStream_t s, int ci, int grid)
{
    const int bytes = (int)sizeof(FastSmem<NT, AMAX, SEG, LW>);
    k_phase_fast<NT, AMAX, SEG, LW, S21><<<grid, NT, bytes, s>>>(v, ci);
}

template <int NT, int AMAX, int SEG, int LW, bool S21>
static int occupancy_v()
{
    const int bytes = (int)sizeof(FastSmem<NT, AMAX, SEG, LW>);
    cudaFuncSetAttribute(k_phase_fast<NT, AMAX, SEG, LW, S21>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_phase_fast<NT, AMAX, SEG, LW, S21>, NT, bytes);
    return n > 0 ? n : 1;
}

// variant = 2 * capacity class + (mu = 2, nu = 1, sigma0 = 1 specialisation)
void launch_phase_fast(int variant, const DevView &v, cudaStream_t s, int ci, int grid)
{
    switch (variant) {
    case 0: launch_v<128, 48, 192, 256, false>(v, s, ci, grid); break;
    case 1: launch_v<128, 48, 192, 256, true>(v, s, ci, grid); break;
    case 2: launch_v<128, 64, 288, 384, false>(v, s, ci, grid); break;
    default: launch_v<128, 64, 288, 384, true>(v, s, ci, grid); break;
    }
}

// Also opts the variant in to its dynamic shared memory size: call once
// before the first launch of a variant.
int fast_blocks_per_sm(int variant)
{
    switch (variant) {
    case 0: return occupancy_v<128, 48, 192, 256, false>();
    case 1: return occupancy_v<128, 48, 192, 256, true>();
    case 2: return occupancy_v<128, 64, 288, 384, false>();
    default: return occupancy_v<128, 64, 288, 384, true>();
    }
}

} // namespace lcmc
