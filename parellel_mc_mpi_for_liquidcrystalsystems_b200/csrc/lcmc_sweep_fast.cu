// lcmc_sweep_fast.cu - FP32 checkerboard phase (production path).
//
// One CTA per active cell (grid-stride over all active cells of all replicas).
// Within a colour phase the 26 neighbour cells of an active cell do not move
// (they have other colours), and each particle of the active cell is attempted
// exactly once, from its phase-start state, with a trial state that depends
// only on its own Philox draws.  So for every particle k the energy against
// the 26 static cells, old and new, is independent of the other attempts:
//
//   dE_k = [S_new(k) - S_old(k)]                 static cells, all k in parallel
//        + sum_{m != k} [phi(n_k, o_m) - phi(o_k, o_m)]   in-cell, old states
//        + sum_{m < k, m accepted} c(k, m)          in-cell corrections
//        + U_coll(n_k) - U_coll(o_k)
//   c(k, m) = [phi(n_k, n_m) - phi(o_k, n_m)] - [phi(n_k, o_m) - phi(o_k, o_m)]
//
// which is exactly E_new - E_old of attempt_monte_carlo_move (MCnptColloid.c:
// 2491-2563) for the sequential in-cell order (ascending id).  Only the short
// scan over the accept decisions is sequential.
//
// Phases per cell:
//   1 stencil  27 cells, periodic image offsets (>= 4 cells per axis)
//   2 active   trial moves (FP64, Philox), colloid hard core and colloid term
//   3 staging  26 static cells -> shared memory, coordinates relative to the
//              active cell's origin in FP32, pruned to the cell box grown by
//              rc + max_displacement/2 (ordered block compaction)
//   4 test     candidates held in registers; for each k one cutoff test
//              against its old position with radius rc + |trial displacement|
//              (covers the old and the new state); passes appended to a
//              per-warp list (ballot compaction)
//   5 pairs    warp per k over its list: FP32 Gay-Berne for old and new state,
//              lane sums combined in FP64
//   6 in-cell  4 pair terms per unordered in-cell pair (old/new x old/new)
//   7 scan     warp 0: Metropolis decisions in id order with the corrections
//   8 write    accepted states back to the FP64 master arrays
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
__device__ __forceinline__ double fold_rel(double x, double o, double cexp, double L)
{
    const double r = x - o;
    return r - L * rint((r - cexp) / L);
}

template <int NT, int CPL, int AMAX, int LCAP>
struct FastSmem {
    static constexpr int NW = NT / 32;
    static constexpr int SMAX = NT * CPL;
    static constexpr int NPAIR = AMAX * (AMAX - 1) / 2;
    static constexpr int CAND = 6 * SMAX > 4 * NPAIR ? 6 * SMAX : 4 * NPAIR;
    float cand[CAND]; // x | y | z | ux | uy | uz ; later the in-cell terms A | B | C | D
    float ax[AMAX], ay[AMAX], az[AMAX], aux[AMAX], auy[AMAX], auz[AMAX]; // old, relative
    float bx[AMAX], by[AMAX], bz[AMAX], bux[AMAX], buy[AMAX], buz[AMAX]; // new, relative
    float rad2[AMAX];
    double rn[3][AMAX], en[3][AMAX]; // new state, FP64, wrapped
    double dUc[AMAX], Sold[AMAX], Snew[AMAX], dEk[AMAX], lu[AMAX];
    int hard[AMAX];
    int acc[AMAX];
    unsigned short list[NW][LCAP];
    unsigned short loff[NW][AMAX], lcnt[NW][AMAX];
    int st_start[27], st_cnt[27], st_pre[28];
    int wcnt[NW];
    int overflow;
    unsigned long long pairs;
};

template <int NT, int CPL, int AMAX, int LCAP>
__global__ void __launch_bounds__(NT) k_phase_fast(DevView v, int ci)
{
    using SM = FastSmem<NT, CPL, AMAX, LCAP>;
    constexpr int NW = SM::NW;
    constexpr int SMAX = SM::SMAX;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SM &sm = *reinterpret_cast<SM *>(smem_raw);
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    float *cx_ = sm.cand, *cy_ = sm.cand + SMAX, *cz_ = sm.cand + 2 * SMAX;
    float *cux = sm.cand + 3 * SMAX, *cuy = sm.cand + 4 * SMAX, *cuz = sm.cand + 5 * SMAX;
    const int *off = v.act_off + ci * (v.R + 1);
    const int total = off[v.R];

    for (int a = blockIdx.x; a < total; a += gridDim.x) {
        const int r = find_replica_f(off, v.R, a);
        const Replica &p = v.rep[r];
        if (!p.use_fast) continue; // uniform across the block
        const int col = p.perm[ci];
        const int bxo = col & 1, byo = (col >> 1) & 1, bzo = (col >> 2) & 1;
        const int nc0 = p.nc[0], nc1 = p.nc[1], nc2 = p.nc[2];
        const int nax = nc0 >> 1, nay = nc1 >> 1;
        int loc = a - off[r];
        const int cx = 2 * (loc % nax) + bxo;
        loc /= nax;
        const int cy = 2 * (loc % nay) + byo;
        const int cz = 2 * (loc / nay) + bzo;
        const int cell = p.cell_off + (cz * nc1 + cy) * nc0 + cx;
        const double o0 = p.shift[0] + (double)cx * p.w[0];
        const double o1 = p.shift[1] + (double)cy * p.w[1];
        const double o2 = p.shift[2] + (double)cz * p.w[2];
        FastK K;
        K.rc2 = p.k.f_rc2;
        K.chi = p.k.f_chi;
        K.chi_sq = p.k.f_chi_sq;
        K.chip = p.k.f_chip;
        K.chip_sq = p.k.f_chip_sq;
        K.sigma0 = p.k.f_sigma0;
        K.four_eps0 = p.k.f_4eps0;
        K.half_chi = p.k.f_half_chi;
        K.half_chip = p.k.f_half_chip;
        K.mu_code = p.k.mu_code;
        K.nu_code = p.k.nu_code;
        K.mu = (float)p.k.mu;
        K.nu = (float)p.k.nu;

        // ---- 1 stencil ----
        if (t < 27) {
            int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
            int x = cx + dx, y = cy + dy, z = cz + dz;
            int ix = x < 0 ? -1 : (x >= nc0 ? 1 : 0);
            int iy = y < 0 ? -1 : (y >= nc1 ? 1 : 0);
            int iz = z < 0 ? -1 : (z >= nc2 ? 1 : 0);
            x -= ix * nc0;
            y -= iy * nc1;
            z -= iz * nc2;
            int c = p.cell_off + (z * nc1 + y) * nc0 + x;
            int s = v.cell_start[c];
            sm.st_start[t] = s;
            sm.st_cnt[t] = v.cell_start[c + 1] - s;
        }
        if (t == 0) {
            sm.overflow = 0;
            sm.pairs = 0ull;
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
            if (t == 0) {
                atomicOr(&v.stats[r].flags, F_CELLCAP);
                v.cell_e0[cell] = 0.0;
                v.cell_n0[cell] = 0;
                v.cell_n1[cell] = 0;
                v.cell_pairs[cell] = 0ull;
                v.cell_cands[cell] = 0ull;
            }
            for (int k = t; k < na; k += NT) v.outcome[p.p_off + v.id[g0 + k]] = 0;
            __syncthreads();
            continue;
        }

        // ---- 2 active particles: trial moves ----
        const double dmax = p.k.max_disp;
        for (int k = t; k < na; k += NT) {
            const int g = g0 + k;
            const uint32_t id = (uint32_t)v.id[g];
            double ro[3] = {v.px[g], v.py[g], v.pz[g]};
            double eo[3] = {v.ox[g], v.oy[g], v.oz[g]};
            U4 m = draw(p.key, id, p.sweep, TAG_MOVE);
            double dsp[3] = {dmax * (u01(m.x) - 0.5), dmax * (u01(m.y) - 0.5), dmax * (u01(m.z) - 0.5)};
            double rn[3] = {ro[0] + dsp[0], ro[1] + dsp[1], ro[2] + dsp[2]};
            // coordinates relative to the cell origin (unwrapped) for the pair terms
            const double qx = fold_rel(ro[0], o0, 0.5 * p.w[0], p.L[0]);
            const double qy = fold_rel(ro[1], o1, 0.5 * p.w[1], p.L[1]);
            const double qz = fold_rel(ro[2], o2, 0.5 * p.w[2], p.L[2]);
            float xo = (float)qx, yo = (float)qy, zo = (float)qz;
            float xn = (float)(qx + dsp[0]), yn = (float)(qy + dsp[1]), zn = (float)(qz + dsp[2]);
            for (int a3 = 0; a3 < 3; a3++) { // apply_pbc (MCnptColloid.c:2420-2430)
                if (rn[a3] > p.L[a3]) rn[a3] -= p.L[a3];
                else if (rn[a3] < 0.0) rn[a3] += p.L[a3];
            }
            double cdist[3];
            double r2c = dist_fold(rn[0], rn[1], rn[2], 0.5 * p.L[0], 0.5 * p.L[1], 0.5 * p.L[2], p.L, cdist);
            int hard = !(r2c > p.k.coll_R * p.k.coll_R);
            double en[3] = {eo[0], eo[1], eo[2]};
            double dU = 0.0;
            if (!hard) {
                double vv[3];
                sphere_point(p.key, id, p.sweep, vv);
                const double ar = p.k.max_rot;
                en[0] = ar * vv[0] + eo[0];
                en[1] = ar * vv[1] + eo[1];
                en[2] = ar * vv[2] + eo[2];
                double n2 = en[0] * en[0] + en[1] * en[1] + en[2] * en[2];
                if (n2 <= 1e-12) {
                    en[0] = eo[0];
                    en[1] = eo[1];
                    en[2] = eo[2];
                } else {
                    double nr = sqrt(n2);
                    en[0] /= nr;
                    en[1] /= nr;
                    en[2] /= nr;
                }
                if (p.k.coll_on) dU = colloid_rod(p.k, rn, en, p.L) - colloid_rod(p.k, ro, eo, p.L);
            }
            float eon = rsqrtf((float)(eo[0] * eo[0] + eo[1] * eo[1] + eo[2] * eo[2]));
            sm.ax[k] = xo;
            sm.ay[k] = yo;
            sm.az[k] = zo;
            sm.aux[k] = (float)eo[0] * eon;
            sm.auy[k] = (float)eo[1] * eon;
            sm.auz[k] = (float)eo[2] * eon;
            sm.bx[k] = xn;
            sm.by[k] = yn;
            sm.bz[k] = zn;
            sm.bux[k] = (float)en[0];
            sm.buy[k] = (float)en[1];
            sm.buz[k] = (float)en[2];
            float dl = (float)sqrt(dsp[0] * dsp[0] + dsp[1] * dsp[1] + dsp[2] * dsp[2]);
            float rr = (float)p.k.rc + dl + 1e-3f;
            sm.rad2[k] = hard ? -1.0f : rr * rr;
            for (int a3 = 0; a3 < 3; a3++) {
                sm.rn[a3][k] = rn[a3];
                sm.en[a3][k] = en[a3];
            }
            sm.dUc[k] = dU;
            sm.hard[k] = hard;
            sm.lu[k] = log_unit(u01(m.w));
        }

        // ---- 3 staging of the 26 static cells, pruned ----
        const float wx = (float)p.w[0], wy = (float)p.w[1], wz = (float)p.w[2];
        const float hb = 0.5f * (float)dmax + 1e-3f;
        const float prune2 = (float)(p.k.rc * p.k.rc) * 1.0002f + 1e-3f;
        int S = 0;
        for (int base = 0; base < S26; base += NT) {
            const int f = base + t;
            bool keep = false;
            float x = 0, y = 0, z = 0, ux = 0, uy = 0, uz = 0;
            if (f < S26) {
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
                x = (float)fold_rel(v.px[g], o0, ((double)(s % 3) - 0.5) * p.w[0], p.L[0]);
                y = (float)fold_rel(v.py[g], o1, ((double)((s / 3) % 3) - 0.5) * p.w[1], p.L[1]);
                z = (float)fold_rel(v.pz[g], o2, ((double)(s / 9) - 0.5) * p.w[2], p.L[2]);
                float qx = fmaxf(fmaxf(-hb - x, x - (wx + hb)), 0.0f);
                float qy = fmaxf(fmaxf(-hb - y, y - (wy + hb)), 0.0f);
                float qz = fmaxf(fmaxf(-hb - z, z - (wz + hb)), 0.0f);
                keep = qx * qx + qy * qy + qz * qz < prune2;
                if (keep) {
                    double ex = v.ox[g], ey = v.oy[g], ez = v.oz[g];
                    float in = rsqrtf((float)(ex * ex + ey * ey + ez * ez));
                    ux = (float)ex * in;
                    uy = (float)ey * in;
                    uz = (float)ez * in;
                }
            }
            unsigned bal = __ballot_sync(0xffffffffu, keep);
            if (lane == 0) sm.wcnt[w] = __popc(bal);
            __syncthreads();
            int woff = 0, tot = 0;
#pragma unroll
            for (int i = 0; i < NW; i++) {
                int c = sm.wcnt[i];
                woff += i < w ? c : 0;
                tot += c;
            }
            const int pos = S + woff + __popc(bal & ((1u << lane) - 1u));
            if (keep && pos < SMAX) {
                cx_[pos] = x;
                cy_[pos] = y;
                cz_[pos] = z;
                cux[pos] = ux;
                cuy[pos] = uy;
                cuz[pos] = uz;
            }
            S += tot;
            __syncthreads();
        }
        if (S > SMAX) {
            if (t == 0) {
                atomicOr(&v.stats[r].flags, F_STENCILCAP);
                v.cell_e0[cell] = 0.0;
                v.cell_n0[cell] = 0;
                v.cell_n1[cell] = 0;
                v.cell_pairs[cell] = 0ull;
                v.cell_cands[cell] = 0ull;
            }
            for (int k = t; k < na; k += NT) v.outcome[p.p_off + v.id[g0 + k]] = 0;
            __syncthreads();
            continue;
        }

        // ---- 4 cutoff test: candidates in registers, per-warp compacted lists ----
        {
            float rx[CPL], ry[CPL], rz[CPL];
#pragma unroll
            for (int c = 0; c < CPL; c++) {
                const int j = t + NT * c;
                const bool ok = j < S;
                rx[c] = ok ? cx_[j] : 1.0e30f;
                ry[c] = ok ? cy_[j] : 1.0e30f;
                rz[c] = ok ? cz_[j] : 1.0e30f;
            }
            int base = 0;
            const unsigned lt = (1u << lane) - 1u;
            for (int k = 0; k < na; k++) {
                const float xk = sm.ax[k], yk = sm.ay[k], zk = sm.az[k], R2 = sm.rad2[k];
                const int b0 = base;
#pragma unroll
                for (int c = 0; c < CPL; c++) {
                    const float dx = rx[c] - xk, dy = ry[c] - yk, dz = rz[c] - zk;
                    const float r2 = dx * dx + dy * dy + dz * dz;
                    const bool pass = r2 < R2;
                    const unsigned bal = __ballot_sync(0xffffffffu, pass);
                    const int pos = base + __popc(bal & lt);
                    if (pass && pos < LCAP) sm.list[w][pos] = (unsigned short)(t + NT * c);
                    base += __popc(bal);
                }
                if (lane == 0) { // on overflow the cell is skipped below, so no clamping here
                    sm.loff[w][k] = (unsigned short)b0;
                    sm.lcnt[w][k] = (unsigned short)(base - b0);
                }
            }
            if (lane == 0 && base > LCAP) sm.overflow = 1;
        }
        __syncthreads();
        if (sm.overflow) {
            if (t == 0) {
                atomicOr(&v.stats[r].flags, F_LISTCAP);
                v.cell_e0[cell] = 0.0;
                v.cell_n0[cell] = 0;
                v.cell_n1[cell] = 0;
                v.cell_pairs[cell] = 0ull;
                v.cell_cands[cell] = 0ull;
            }
            for (int k = t; k < na; k += NT) v.outcome[p.p_off + v.id[g0 + k]] = 0;
            __syncthreads();
            continue;
        }

        // ---- 5 static pair sums: warp per active particle ----
        for (int k = w; k < na; k += NW) {
            const float xo = sm.ax[k], yo = sm.ay[k], zo = sm.az[k];
            const float uox = sm.aux[k], uoy = sm.auy[k], uoz = sm.auz[k];
            const float xn = sm.bx[k], yn = sm.by[k], zn = sm.bz[k];
            const float unx = sm.bux[k], uny = sm.buy[k], unz = sm.buz[k];
            int pre[NW + 1];
            pre[0] = 0;
#pragma unroll
            for (int i = 0; i < NW; i++) pre[i + 1] = pre[i] + sm.lcnt[i][k];
            const int T = pre[NW];
            // FP64 lane sums: the 1e9 overlap clamp is exact in FP32 and must
            // cancel exactly between the old and the new sum
            double so = 0.0, sn = 0.0;
            int np = 0;
            for (int q = lane; q < T; q += 32) {
                int ww = 0;
#pragma unroll
                for (int i = 1; i < NW; i++) ww += q >= pre[i];
                const int j = sm.list[ww][sm.loff[ww][k] + (q - pre[ww])];
                const float xj = cx_[j], yj = cy_[j], zj = cz_[j];
                const float ujx = cux[j], ujy = cuy[j], ujz = cuz[j];
                float dx = xj - xo, dy = yj - yo, dz = zj - zo;
                float r2 = dx * dx + dy * dy + dz * dz;
                float e = pair_fast(K, dx, dy, dz, r2, uox, uoy, uoz, ujx, ujy, ujz);
                bool in = r2 < K.rc2;
                so += in ? (double)e : 0.0;
                np += in;
                dx = xj - xn;
                dy = yj - yn;
                dz = zj - zn;
                r2 = dx * dx + dy * dy + dz * dz;
                e = pair_fast(K, dx, dy, dz, r2, unx, uny, unz, ujx, ujy, ujz);
                in = r2 < K.rc2;
                sn += in ? (double)e : 0.0;
                np += in;
            }
            double dso = so, dsn = sn;
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1) {
                dso += __shfl_xor_sync(0xffffffffu, dso, o);
                dsn += __shfl_xor_sync(0xffffffffu, dsn, o);
                np += __shfl_xor_sync(0xffffffffu, np, o);
            }
            if (lane == 0) {
                sm.Sold[k] = dso;
                sm.Snew[k] = dsn;
                atomicAdd(&sm.pairs, (unsigned long long)np);
            }
        }
        __syncthreads();

        // ---- 6 in-cell pairs: 4 terms per unordered pair (reuses the candidate region) ----
        float *tA = sm.cand, *tB = sm.cand + SM::NPAIR, *tC = sm.cand + 2 * SM::NPAIR, *tD = sm.cand + 3 * SM::NPAIR;
        const int npair = na * (na - 1) / 2;
        int npin = 0;
        for (int idx = t; idx < npair; idx += NT) {
            int q = (int)((1.0f + sqrtf(1.0f + 8.0f * (float)idx)) * 0.5f);
            while (q * (q - 1) / 2 > idx) q--;
            while ((q + 1) * q / 2 <= idx) q++;
            const int pp = idx - q * (q - 1) / 2;
            float A, B, C, D;
            {
                float dx = sm.ax[q] - sm.ax[pp], dy = sm.ay[q] - sm.ay[pp], dz = sm.az[q] - sm.az[pp];
                float r2 = dx * dx + dy * dy + dz * dz;
                A = r2 < K.rc2 ? pair_fast(K, dx, dy, dz, r2, sm.aux[pp], sm.auy[pp], sm.auz[pp], sm.aux[q],
                                           sm.auy[q], sm.auz[q])
                               : 0.0f;
                npin += 2 * (r2 < K.rc2);
            }
            {
                float dx = sm.bx[q] - sm.ax[pp], dy = sm.by[q] - sm.ay[pp], dz = sm.bz[q] - sm.az[pp];
                float r2 = dx * dx + dy * dy + dz * dz;
                B = r2 < K.rc2 ? pair_fast(K, dx, dy, dz, r2, sm.aux[pp], sm.auy[pp], sm.auz[pp], sm.bux[q],
                                           sm.buy[q], sm.buz[q])
                               : 0.0f;
                npin += (r2 < K.rc2);
            }
            {
                float dx = sm.ax[q] - sm.bx[pp], dy = sm.ay[q] - sm.by[pp], dz = sm.az[q] - sm.bz[pp];
                float r2 = dx * dx + dy * dy + dz * dz;
                C = r2 < K.rc2 ? pair_fast(K, dx, dy, dz, r2, sm.bux[pp], sm.buy[pp], sm.buz[pp], sm.aux[q],
                                           sm.auy[q], sm.auz[q])
                               : 0.0f;
                npin += (r2 < K.rc2);
            }
            {
                float dx = sm.bx[q] - sm.bx[pp], dy = sm.by[q] - sm.by[pp], dz = sm.bz[q] - sm.bz[pp];
                float r2 = dx * dx + dy * dy + dz * dz;
                D = r2 < K.rc2 ? pair_fast(K, dx, dy, dz, r2, sm.bux[pp], sm.buy[pp], sm.buz[pp], sm.bux[q],
                                           sm.buy[q], sm.buz[q])
                               : 0.0f;
            }
            // the four terms as computed (the 1e9 clamp is exact); differences are taken in FP64
            tA[idx] = A;
            tB[idx] = B;
            tC[idx] = C;
            tD[idx] = D;
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) npin += __shfl_xor_sync(0xffffffffu, npin, o);
        if (lane == 0 && npin) atomicAdd(&sm.pairs, (unsigned long long)npin);
        __syncthreads();
        for (int k = t; k < na; k += NT) {
            double dsum = 0.0;
            for (int m = 0; m < na; m++) {
                if (m < k) {
                    const int i2 = tri(m, k); // k is the later particle: phi(n_k, o_m) - phi(o_k, o_m)
                    dsum += (double)tB[i2] - (double)tA[i2];
                } else if (m > k) {
                    const int i2 = tri(k, m); // k is the earlier particle
                    dsum += (double)tC[i2] - (double)tA[i2];
                }
            }
            sm.dEk[k] = (sm.Snew[k] - sm.Sold[k]) + dsum + sm.dUc[k];
        }
        __syncthreads();

        // ---- 7 sequential Metropolis scan (warp 0) ----
        if (w == 0) {
            double e0 = lane < na ? sm.dEk[lane] : 0.0;
            double e1 = lane + 32 < na ? sm.dEk[lane + 32] : 0.0;
            const double beta = p.k.beta;
            double dsum = 0.0;
            int nacc = 0, nhard = 0;
            for (int m = 0; m < na; m++) {
                const int own = m & 31;
                const double val = __shfl_sync(0xffffffffu, m < 32 ? e0 : e1, own);
                const int hd = sm.hard[m];
                const bool acc = !hd && ((val <= 0.0) || (sm.lu[m] <= -beta * val));
                nhard += hd;
                if (acc) {
                    dsum += val;
                    nacc++;
                    // c(k, m) = [phi(n_k, n_m) - phi(o_k, n_m)] - [phi(n_k, o_m) - phi(o_k, o_m)]
                    if (lane > m && lane < na) {
                        const int i2 = tri(m, lane);
                        e0 += ((double)tD[i2] - (double)tC[i2]) - ((double)tB[i2] - (double)tA[i2]);
                    }
                    if (lane + 32 > m && lane + 32 < na) {
                        const int i2 = tri(m, lane + 32);
                        e1 += ((double)tD[i2] - (double)tC[i2]) - ((double)tB[i2] - (double)tA[i2]);
                    }
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

        // ---- 8 write-back ----
        for (int k = t; k < na; k += NT) {
            const int g = g0 + k;
            const int acc = sm.acc[k];
            if (acc) {
                v.px[g] = sm.rn[0][k];
                v.py[g] = sm.rn[1][k];
                v.pz[g] = sm.rn[2][k];
                v.ox[g] = sm.en[0][k];
                v.oy[g] = sm.en[1][k];
                v.oz[g] = sm.en[2][k];
            }
            v.outcome[p.p_off + v.id[g]] = sm.hard[k] ? 2 : acc;
        }
        __syncthreads();
    }
}

// Instantiations: (threads, candidates per thread, active capacity, list capacity per warp).
template __global__ void k_phase_fast<128, 6, 48, 1024>(DevView, int);
template __global__ void k_phase_fast<128, 8, 64, 1536>(DevView, int);
template __global__ void k_phase_fast<256, 4, 64, 768>(DevView, int);

} // namespace lcmc

#include "lcmc_launch.h"

namespace lcmc {

static const FastVariant kVariants[] = {{128, 6, 48, 1024}, {128, 8, 64, 1536}, {256, 4, 64, 768}};

int fast_variant_count() { return (int)(sizeof(kVariants) / sizeof(kVariants[0])); }
FastVariant fast_variant(int i) { return kVariants[i]; }

template <int NT, int CPL, int AMAX, int LCAP>
static void launch_v(const DevView &v, cudaStream_t s, int ci, int grid)
{
    const int bytes = (int)sizeof(FastSmem<NT, CPL, AMAX, LCAP>);
    k_phase_fast<NT, CPL, AMAX, LCAP><<<grid, NT, bytes, s>>>(v, ci);
}

template <int NT, int CPL, int AMAX, int LCAP>
static int occupancy_v()
{
    const int bytes = (int)sizeof(FastSmem<NT, CPL, AMAX, LCAP>);
    cudaFuncSetAttribute(k_phase_fast<NT, CPL, AMAX, LCAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_phase_fast<NT, CPL, AMAX, LCAP>, NT, bytes);
    return n > 0 ? n : 1;
}

void launch_phase_fast(int variant, const DevView &v, cudaStream_t s, int ci, int grid)
{
    switch (variant) {
    case 0: launch_v<128, 6, 48, 1024>(v, s, ci, grid); break;
    case 1: launch_v<128, 8, 64, 1536>(v, s, ci, grid); break;
    default: launch_v<256, 4, 64, 768>(v, s, ci, grid); break;
    }
}

// Also opts the variant in to its dynamic shared memory size: call once
// before the first launch of a variant.
int fast_blocks_per_sm(int variant)
{
    switch (variant) {
    case 0: return occupancy_v<128, 6, 48, 1024>();
    case 1: return occupancy_v<128, 8, 64, 1536>();
    default: return occupancy_v<256, 4, 64, 768>();
    }
}

} // namespace lcmc
