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
//   dE_k = [S_new(k) - S_old(k)]                               static cells
//        + sum_{m > k} [phi(n_k, o_m) - phi(o_k, o_m)]          later in-cell partners
//        + sum_{m < k} [phi(n_k, n_m) - phi(o_k, n_m)]  if m was accepted,
//                      [phi(n_k, o_m) - phi(o_k, o_m)]  if not  earlier partners
//        + U_coll(n_k) - U_coll(o_k)
//
// Each earlier partner contributes exactly one of its two terms, never one and
// then a correction: a near-overlap term of 1e20 or more that would cancel must
// not pass through the FP64 sum, whose rounding at that size (1e4 and up) would
// swamp dE_k.  This is exactly E_new - E_old of attempt_monte_carlo_move
// (MCnptColloid.c:2491-2563) for the sequential in-cell order (ascending id);
// only the decisions depend on each other, through a triangular system.
//
// Phases per cell:
//   1 stencil  27 cells (>= 4 cells per axis, no duplicates)
//   2 active   phase-start state and precomputed trial of each particle of the
//              cell, coordinates relative to the cell origin (FP32)
//   3 staging  the 26 static cells -> shared memory (float4 x,y,z,ux + float2
//              uy,uz), read from the FP32 copy of the state (coordinates
//              relative to each particle's own cell origin, folded across the
//              periodic seam by the gather) plus the stencil offset, pruned to
//              the cell box grown by rc + max_displacement/2; warp w compacts its
//              quarter of the candidates into its own segment (no block barrier
//              per round)
//   4 tasks    warps take tasks from a shared queue:
//              particle task (two particles k, k + 1): cutoff test of every
//                staged candidate, loaded once, against both old positions
//                with radius rc + |displacement| (covers old and new state),
//                warp segment by warp segment, ballot compaction into two
//                lists, then FP32 Gay-Berne for old and new state over both
//                lists together, lane sums in FP64
//              pair task: 32 unordered in-cell pairs, 4 terms each
//              (old/new x old/new), differences formed in FP64
//   5 sums     warp 0, thread per particle: static + colloid + later in-cell
//              partners (per-particle trial data was prefetched into shared
//              memory in step 2)
//   6 decide   warp 0: Metropolis decisions in id order (fixed-point passes
//              over the triangular system the sequential order defines)
//   7 write    accepted trial states to the FP64 master arrays
//
// FP64 for overlaps: FP32 rounding of a pair term is relative to the term,
// and near an overlap (R^12 up to 1e36 just above the 1e9 clamp) it exceeds
// any energy scale, so a decision or a running energy built from such terms
// is meaningless.  A static pair whose FP32 term (old or new state) exceeds
// f_big in magnitude, hits the overlap clamp or is not finite is evaluated
// again in FP64 from the master arrays (its flat stencil index is kept with
// the staged candidate), both states, on the one-fold minimum image; the lane
// sums are FP64, so such terms carry FP64 rounding only.  A cell with such an
// in-cell term (whose pair differences are kept in FP32), or above the
// kernel's capacity (particles, staged candidates or list entries), makes no
// move here and is handed over to k_phase_rescue, which attempts it from the
// same phase-start state in FP64.  Below f_big the FP32 terms carry an absolute
// error of at most about 2e-4 f_big / 100 (1.9e-4 relative, stated per pair),
// so decisions differ from FP64 only at near-ties.
#include <cuda_runtime.h>

#include "lcmc_gb.cuh"
#include "lcmc_internal.h"
#include "lcmc_rng.cuh"
#include "lcmc_trial.cuh"

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

// FP64 pair term for a pair the FP32 term cannot carry: pair_energy64's
// form for mu = 2, nu = 1, sigma0 = 1, else the reference-order pair_exact.
template <bool SPEC21>
__device__ __forceinline__ double pair64_t(const GBConsts &k, double r2, const double d[3], const double ei[3],
                                           const double ej[3])
{
    return SPEC21 ? pair_energy64_21(k, r2, d, ei, ej) : pair_exact(k, r2, d, ei, ej);
}

struct BigPair {
    double e0, e1; // FP64 terms of the old and the new state (0 beyond the cutoff)
    int n;         // in-cutoff states (0, 1 or 2)
};

// Both states of one static pair (active particle at slot gk, its trial
// state, candidate at slot gj) in FP64 from the master arrays, on the one-fold
// minimum image, the cutoff decided in FP64.  Not inlined: the rare path keeps
// its registers out of the hot loop's allocation.
template <bool SPEC21>
__device__ __forceinline__ BigPair big_pair64(const double *__restrict__ px, const double *__restrict__ py,
                                           const double *__restrict__ pz, const double *__restrict__ ox,
                                           const double *__restrict__ oy, const double *__restrict__ oz,
                                           const double *__restrict__ tnx, const double *__restrict__ tny,
                                           const double *__restrict__ tnz, const double *__restrict__ tux,
                                           const double *__restrict__ tuy, const double *__restrict__ tuz,
                                           const Replica *__restrict__ rp, int gk, int gj)
{
    const Replica &p = *rp;
    const double rj[3] = {px[gj], py[gj], pz[gj]};
    const double ej[3] = {ox[gj], oy[gj], oz[gj]};
    const double ro[3] = {px[gk], py[gk], pz[gk]};
    const double eo[3] = {ox[gk], oy[gk], oz[gk]};
    const double rn[3] = {tnx[gk], tny[gk], tnz[gk]};
    const double en[3] = {tux[gk], tuy[gk], tuz[gk]};
    BigPair b;
    double d[3];
    double q2 = dist_fold(ro[0], ro[1], ro[2], rj[0], rj[1], rj[2], p.L, d);
    const bool i0 = q2 < p.k.rc2;
    b.e0 = i0 ? pair64_t<SPEC21>(p.k, q2, d, eo, ej) : 0.0;
    q2 = dist_fold(rn[0], rn[1], rn[2], rj[0], rj[1], rj[2], p.L, d);
    const bool i1 = q2 < p.k.rc2;
    b.e1 = i1 ? pair64_t<SPEC21>(p.k, q2, d, en, ej) : 0.0;
    b.n = (int)i0 + (int)i1;
    return b;
}

template <int NT, int AMAX, int SEG, int LW>
struct FastSmem {
    static constexpr int NW = NT / 32;
    static constexpr int NPAIR = AMAX * (AMAX - 1) / 2;
    float4 cpos[NW * SEG];     // x, y, z, ux of the static candidates (segment per warp)
    float2 cori[NW * SEG];     // uy, uz
    unsigned short cidx[NW * SEG]; // flat stencil index of each (to find its FP64 state for a large term)
    // in-cell pair terms rounded to FP32: C - A, B - A, D - C (for a later particle the scan adds
    // D - C if the earlier partner moved, B - A if it stayed)
    float pCA[NPAIR], pBA[NPAIR], pDC[NPAIR];
    // old (a) and trial (b) state of each active particle, relative to the cell
    // origin: [0] = (ax, ay, az, aux), [1] = (auy, auz, bx, by), [2] = (bz, bux, buy, buz)
    float4 pst[AMAX][3];
    float rad2[AMAX];
    double Sold[AMAX], Snew[AMAX];
    double tdU[AMAX], tlu[AMAX]; // colloid dU of the trial, log of the Metropolis draw
    int pid[AMAX];        // particle id (outcome slot)
    unsigned char hard[AMAX];
    int acc[AMAX];
    unsigned short wlist[NW][2][LW]; // per warp: candidate lists of the task's two particles
    // pairs whose FP32 term is above f_big (overlaps), evaluated in FP64 by the
    // fix-up pass after the task queue: static pairs (particle k << 16 | staged
    // candidate) and in-cell pairs (pair index)
    static constexpr int BIGCAP = 32;
    unsigned int bigs[BIGCAP];
    unsigned short bigp[BIGCAP];
    int nbigs, nbigp;
    int st_start[27], st_cnt[27], st_pre[28];
    int segcnt[NW];
    int task;
    int overflow;
    int big; // a pair term above f_big (or clamped, or non-finite): attempt the cell in FP64
    unsigned long long pairs;
};

// Hand a cell over to the FP64 phase kernel (k_phase_rescue, launched after
// this one in the same colour phase); it writes the cell's results.
__device__ __forceinline__ void hand_over(const DevView &v, int ci, int cell, int mode)
{
    const int i = atomicAdd(&v.resc_count[ci], 1);
    v.resc_list[(size_t)ci * v.ctot + i] = cell * 4 + mode;
}



// FP64 pair term of particles at ri (orientation ei) and rj (ej), one-fold
// minimum image, 0 beyond the cutoff.
template <bool SPEC21>
__device__ __forceinline__ double term64(const Replica &p, const double ri[3], const double ei[3], const double rj[3],
                                         const double ej[3])
{
    double d[3];
    const double r2 = dist_fold(ri[0], ri[1], ri[2], rj[0], rj[1], rj[2], p.L, d);
    return r2 < p.k.rc2 ? pair64_t<SPEC21>(p.k, r2, d, ei, ej) : 0.0;
}

// FP64 fix-up of the pairs whose FP32 term is above f_big (overlaps), after
// the task queue, with every thread of the block:
//   in-cell pairs (thread per listed pair): the four terms phi(o/n_q, o/n_p)
//     in FP64 from the master arrays; the differences C - A, B - A, D - C
//     replace the FP32 ones (rounded to FP32 once: below 1e5 eps0 that keeps
//     them within 0.01 eps0); a larger term (the overlap clamp and its
//     neighbourhood) sends the cell to the FP64 hand-over kernel;
//   static pairs (thread per particle): the particle's listed pairs in
//     ascending staged order, both states in FP64, added to its static sums
//     (a fixed order: the bits do not depend on scheduling).
template <int NT, typename SM, bool SPEC21>
__device__ __noinline__ void fixup_big(const DevView *__restrict__ vp, int r, int g0, int na, SM &sm)
{
    const DevView &v = *vp;
    const Replica &p = v.rep[r];
    const int t = threadIdx.x;
    const int nbp = min(sm.nbigp, SM::BIGCAP), nbs = min(sm.nbigs, SM::BIGCAP);
    for (int e = t; e < nbp; e += NT) {
        const int idx = sm.bigp[e];
        int q = (int)((1.0f + sqrtf(1.0f + 8.0f * (float)idx)) * 0.5f);
        while (q * (q - 1) / 2 > idx) q--;
        while ((q + 1) * q / 2 <= idx) q++;
        const int pp = idx - q * (q - 1) / 2;
        const int gq = g0 + q, gp = g0 + pp;
        const double oq[3] = {v.px[gq], v.py[gq], v.pz[gq]}, uq[3] = {v.ox[gq], v.oy[gq], v.oz[gq]};
        const double nq[3] = {v.tnx[gq], v.tny[gq], v.tnz[gq]}, wq[3] = {v.tux[gq], v.tuy[gq], v.tuz[gq]};
        const double op[3] = {v.px[gp], v.py[gp], v.pz[gp]}, up[3] = {v.ox[gp], v.oy[gp], v.oz[gp]};
        const double np_[3] = {v.tnx[gp], v.tny[gp], v.tnz[gp]}, wp[3] = {v.tux[gp], v.tuy[gp], v.tuz[gp]};
        // A = (o_q, o_p), B = (n_q, o_p), C = (o_q, n_p), D = (n_q, n_p)
        double term[4] = {term64<SPEC21>(p, op, up, oq, uq), term64<SPEC21>(p, op, up, nq, wq),
                          term64<SPEC21>(p, np_, wp, oq, uq), term64<SPEC21>(p, np_, wp, nq, wq)};
        // terms with the trial state of a particle that cannot move are never used
        const bool hp = sm.hard[pp] != 0, hq = sm.hard[q] != 0;
        if (hq) term[1] = term[3] = 0.0;
        if (hp) term[2] = term[3] = 0.0;
        if (hp && hq) term[0] = 0.0;
        if (!(fabs(term[0]) <= 1e5 && fabs(term[1]) <= 1e5 && fabs(term[2]) <= 1e5 && fabs(term[3]) <= 1e5)) {
            sm.big = 1;
        } else {
            sm.pCA[idx] = (float)(term[2] - term[0]);
            sm.pBA[idx] = (float)(term[1] - term[0]);
            sm.pDC[idx] = (float)(term[3] - term[2]);
        }
    }
    unsigned long long extra = 0ull;
    for (int k = t; k < na; k += NT) {
        double so = 0.0, sn = 0.0;
        bool any = false;
        int last = -1;
        for (;;) { // this particle's listed candidates in ascending staged order
            int best = 1 << 30;
            for (int e = 0; e < nbs; e++) {
                const unsigned u = sm.bigs[e];
                const int j = (int)(u & 0xFFFFu);
                if ((int)(u >> 16) == k && j > last && j < best) best = j;
            }
            if (best == (1 << 30)) break;
            last = best;
            const int f = sm.cidx[best];
            int sl = 0, hi = 27;
            while (hi - sl > 1) {
                const int mid = (sl + hi) >> 1;
                if (sm.st_pre[mid] <= f) sl = mid;
                else hi = mid;
            }
            const BigPair b = big_pair64<SPEC21>(v.px, v.py, v.pz, v.ox, v.oy, v.oz, v.tnx, v.tny, v.tnz, v.tux,
                                                 v.tuy, v.tuz, v.rep + r, g0 + k, sm.st_start[sl] + (f - sm.st_pre[sl]));
            so += b.e0;
            sn += b.e1;
            extra += (unsigned long long)b.n;
            any = true;
        }
        if (any) {
            sm.Sold[k] += so;
            sm.Snew[k] += sn;
        }
    }
    if (extra) atomicAdd(&sm.pairs, extra);
}

// resident CTAs per SM the register budget is sized for: the 48-particle
// class (36.9 KB of shared memory) fits six per SM at 80 registers, the
// 56-particle class (44.5 KB) five at 102, the 64-particle class is limited to
// three by its shared memory
template <int AMAX> struct FastMinBlocks { static constexpr int value = AMAX <= 48 ? 6 : (AMAX <= 56 ? 5 : 3); };

template <int NT, int AMAX, int SEG, int LW, bool SPEC21>
__global__ void __launch_bounds__(NT, FastMinBlocks<AMAX>::value) k_phase_fast(const __grid_constant__ DevView v, int ci)
{
    using SM = FastSmem<NT, AMAX, SEG, LW>;
    constexpr int NW = SM::NW;
    static_assert(AMAX <= 64, "the scan warp holds two particles per lane");
    static_assert(AMAX + 32 <= NT, "threads 32 .. 32 + AMAX - 1 write the particles back");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SM &sm = *reinterpret_cast<SM *>(smem_raw);
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const int *off = v.act_off + ci * (v.R + 1);
    const int total = off[v.r_hi]; // this launch's replicas: active cells [off[r_lo], off[r_hi])

    for (int a = off[v.r_lo] + blockIdx.x; a < total; a += gridDim.x) {
        const int r = find_replica_f(off, v.R, a);
        const Replica &p = v.rep[r];
        if (!p.use_fast) continue; // uniform across the block
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
        const double w0 = p.w[0], w1 = p.w[1], w2 = p.w[2];
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
            sm.big = 0;
            sm.nbigs = 0;
            sm.nbigp = 0;
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
        if (na > AMAX || na > p.cap) { // above capacity: the whole cell in FP64
            if (t == 0) hand_over(v, ci, cell, 2);
            __syncthreads();
            continue;
        }

        // ---- 2 active particles: phase-start state and precomputed trial ----
        const float rcf = (float)p.k.rc;
        for (int k = t; k < na; k += NT) {
            const int g = g0 + k;
            const float4 c4 = v.cl4[g]; // relative to this cell's origin
            const float2 c2 = v.cl2[g];
            const float dx = v.tdx[g], dy = v.tdy[g], dz = v.tdz[g];
            sm.pst[k][0] = c4;
            sm.pst[k][1] = make_float4(c2.x, c2.y, c4.x + dx, c4.y + dy);
            float tux, tuy, tuz; // the trial orientation as the FP32 state copy will hold it
            unit_f32(v.tux[g], v.tuy[g], v.tuz[g], tux, tuy, tuz);
            sm.pst[k][2] = make_float4(c4.z + dz, tux, tuy, tuz);
            const float rr = rcf + sqrtf(dx * dx + dy * dy + dz * dz) + 1e-3f;
            const unsigned char hd = v.thard[g];
            sm.rad2[k] = hd ? -1.0f : rr * rr;
            sm.hard[k] = hd;
            sm.tdU[k] = v.tdU[g];
            sm.tlu[k] = v.tlu[g];
            sm.pid[k] = v.id[g];
        }

        // ---- 3 staging: warp w takes a contiguous quarter of the 26 static cells'
        //      particles and compacts the kept ones into its own segment ----
        {
            const float wx = (float)w0, wy = (float)w1, wz = (float)w2;
            const float hb = 0.5f * (float)p.k.max_disp + 1e-3f;
            const float prune2 = K.rc2 * 1.0002f + 1e-3f;
            const int fb = (int)(((long long)S26 * w) / NW), fe = (int)(((long long)S26 * (w + 1)) / NW);
            int cnt = 0;
            // two candidates per lane per round, all six coordinates loaded at
            // once: the global loads of a round are independent of each other
            for (int base = fb; base < fe; base += 64) {
                float x[2], y[2], z[2], ux[2], uy[2], uz[2];
                bool keep[2];
                int fi[2];
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int f = base + 32 * h + lane;
                    fi[h] = f;
                    keep[h] = false;
                    x[h] = y[h] = z[h] = ux[h] = uy[h] = uz[h] = 0.0f;
                    if (f < fe) {
                        // largest stencil slot whose prefix is <= f (slot 13 has an empty range;
                        // an empty slot's prefix is the end of the previous range, so it is never picked)
                        int sl = 0, hi = 27;
                        while (hi - sl > 1) {
                            const int mid = (sl + hi) >> 1;
                            if (sm.st_pre[mid] <= f) sl = mid;
                            else hi = mid;
                        }
                        const int g = sm.st_start[sl] + (f - sm.st_pre[sl]);
                        const float4 c4 = v.cl4[g]; // relative to its own cell's origin
                        const float2 c2 = v.cl2[g];
                        // stencil offset of slot sl is (sl % 3, sl / 3 % 3, sl / 9) - 1 cells
                        x[h] = c4.x + (float)(sl % 3 - 1) * wx;
                        y[h] = c4.y + (float)((sl / 3) % 3 - 1) * wy;
                        z[h] = c4.z + (float)(sl / 9 - 1) * wz;
                        const float qx = fmaxf(fmaxf(-hb - x[h], x[h] - (wx + hb)), 0.0f);
                        const float qy = fmaxf(fmaxf(-hb - y[h], y[h] - (wy + hb)), 0.0f);
                        const float qz = fmaxf(fmaxf(-hb - z[h], z[h] - (wz + hb)), 0.0f);
                        keep[h] = qx * qx + qy * qy + qz * qz < prune2;
                        ux[h] = c4.w;
                        uy[h] = c2.x;
                        uz[h] = c2.y;
                    }
                }
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const unsigned bal = __ballot_sync(0xffffffffu, keep[h]);
                    const int pos = cnt + __popc(bal & lt);
                    if (keep[h] && pos < SEG) {
                        sm.cpos[w * SEG + pos] = make_float4(x[h], y[h], z[h], ux[h]);
                        sm.cori[w * SEG + pos] = make_float2(uy[h], uz[h]);
                        sm.cidx[w * SEG + pos] = (unsigned short)fi[h];
                    }
                    cnt += __popc(bal);
                }
            }
            if (lane == 0) {
                sm.segcnt[w] = cnt < SEG ? cnt : SEG;
                if (cnt > SEG) sm.overflow = 2;
            }
        }
        __syncthreads();
        if (sm.overflow) { // staged candidates above a warp segment's capacity
            if (t == 0) hand_over(v, ci, cell, 2);
            __syncthreads();
            continue;
        }
        // ---- 4 task queue: particle tasks (two particles each: cutoff test +
        //      pair sums) and in-cell pair tasks ----
        const int nptask = (na + 1) >> 1;
        const int npair = na * (na - 1) / 2;
        const int ntask = nptask + (npair + 31) / 32;
        unsigned long long npairs = 0ull;
        for (;;) {
            int task = 0;
            if (lane == 0) task = *(volatile int *)&sm.big ? ntask : atomicAdd(&sm.task, 1);
            task = __shfl_sync(0xffffffffu, task, 0);
            if (task >= ntask) break;
            if (task < nptask) {
                const int ka = 2 * task, kb = 2 * task + 1;
                const bool has_b = kb < na;
                const float R2a = sm.rad2[ka];
                const float R2b = has_b ? sm.rad2[kb] : -1.0f;
                double soa = 0.0, sna = 0.0, sob = 0.0, snb = 0.0;
                int np = 0;
                if (R2a > 0.0f || R2b > 0.0f) {
                    const float4 qa = sm.pst[ka][0];
                    const float4 qb = has_b ? sm.pst[kb][0] : qa;
                    int ca = 0, cb = 0;
                    // cutoff test of every staged candidate, warp segment by warp segment
#pragma unroll 1
                    for (int i = 0; i < NW; i++) {
                        const int s0 = i * SEG, sc = sm.segcnt[i];
                        for (int base = 0; base < sc; base += 64) {
                            bool pa[2], pb[2];
#pragma unroll
                            for (int h = 0; h < 2; h++) {
                                const int j = base + 32 * h + lane;
                                pa[h] = pb[h] = false;
                                if (j < sc) {
                                    const float4 c = sm.cpos[s0 + j];
                                    float dx = c.x - qa.x, dy = c.y - qa.y, dz = c.z - qa.z;
                                    pa[h] = dx * dx + dy * dy + dz * dz < R2a;
                                    dx = c.x - qb.x;
                                    dy = c.y - qb.y;
                                    dz = c.z - qb.z;
                                    pb[h] = dx * dx + dy * dy + dz * dz < R2b;
                                }
                            }
#pragma unroll
                            for (int h = 0; h < 2; h++) {
                                const unsigned ba = __ballot_sync(0xffffffffu, pa[h]);
                                const unsigned bb = __ballot_sync(0xffffffffu, pb[h]);
                                const int pa_ = ca + __popc(ba & lt), pb_ = cb + __popc(bb & lt);
                                const unsigned short sl = (unsigned short)(s0 + base + 32 * h + lane);
                                if (pa[h] && pa_ < LW) sm.wlist[w][0][pa_] = sl;
                                if (pb[h] && pb_ < LW) sm.wlist[w][1][pb_] = sl;
                                ca += __popc(ba);
                                cb += __popc(bb);
                            }
                        }
                    }
                    if (ca > LW || cb > LW) {
                        if (lane == 0) sm.overflow = 1;
                        ca = ca < LW ? ca : LW;
                        cb = cb < LW ? cb : LW;
                    }
                    __syncwarp();
                    // FP64 lane sums of the FP32 terms.  Entries [0, ca) belong to
                    // particle a, [ca, ca + cb) to particle b.  An entry with a term
                    // FP32 cannot carry is listed for the FP64 fix-up pass.
                    for (int q = lane; q < ca + cb; q += 32) {
                        const bool isa = q < ca;
                        const int j = isa ? sm.wlist[w][0][q] : sm.wlist[w][1][q - ca];
                        const int k = isa ? ka : kb;
                        const float4 P0 = sm.pst[k][0], P1 = sm.pst[k][1], P2 = sm.pst[k][2];
                        const float4 c = sm.cpos[j];
                        const float2 u = sm.cori[j];
                        float dx = c.x - P0.x, dy = c.y - P0.y, dz = c.z - P0.z;
                        float r2 = dx * dx + dy * dy + dz * dz;
                        const float e0 = pair_fast_t<SPEC21>(K, dx, dy, dz, r2, P0.w, P1.x, P1.y, c.w, u.x, u.y);
                        const bool in0 = r2 < K.rc2;
                        dx = c.x - P1.z;
                        dy = c.y - P1.w;
                        dz = c.z - P2.x;
                        r2 = dx * dx + dy * dy + dz * dz;
                        const float e1 = pair_fast_t<SPEC21>(K, dx, dy, dz, r2, P2.y, P2.z, P2.w, c.w, u.x, u.y);
                        const bool in1 = r2 < K.rc2;
                        int nin = (int)in0 + (int)in1;
                        double d0 = in0 ? (double)e0 : 0.0, d1 = in1 ? (double)e1 : 0.0;
                        if ((in0 && !(fabsf(e0) <= K.big)) || (in1 && !(fabsf(e1) <= K.big))) {
                            const int slot = atomicAdd(&sm.nbigs, 1);
                            if (slot < SM::BIGCAP) sm.bigs[slot] = ((unsigned)k << 16) | (unsigned)j;
                            else sm.overflow = 1;
                            d0 = d1 = 0.0;
                            nin = 0;
                        }
                        if (isa) {
                            soa += d0;
                            sna += d1;
                        } else {
                            sob += d0;
                            snb += d1;
                        }
                        np += nin;
                    }
                    __syncwarp();
                }
#pragma unroll
                for (int o = 16; o >= 1; o >>= 1) {
                    soa += __shfl_xor_sync(0xffffffffu, soa, o);
                    sna += __shfl_xor_sync(0xffffffffu, sna, o);
                    sob += __shfl_xor_sync(0xffffffffu, sob, o);
                    snb += __shfl_xor_sync(0xffffffffu, snb, o);
                    np += __shfl_xor_sync(0xffffffffu, np, o);
                }
                if (lane == 0) {
                    sm.Sold[ka] = soa;
                    sm.Snew[ka] = sna;
                    if (has_b) {
                        sm.Sold[kb] = sob;
                        sm.Snew[kb] = snb;
                    }
                }
                npairs += (unsigned long long)np;
            } else {
                const int idx = (task - nptask) * 32 + lane;
                int npin = 0;
                if (idx < npair) {
                    int q = (int)((1.0f + sqrtf(1.0f + 8.0f * (float)idx)) * 0.5f);
                    while (q * (q - 1) / 2 > idx) q--;
                    while ((q + 1) * q / 2 <= idx) q++;
                    const int pp = idx - q * (q - 1) / 2;
                    float A, B, Cc, D;
                    const float4 Q0 = sm.pst[q][0], Q1 = sm.pst[q][1], Q2 = sm.pst[q][2];
                    const float4 R0 = sm.pst[pp][0], R1 = sm.pst[pp][1], R2 = sm.pst[pp][2];
                    // a(.) = (X0.x, X0.y, X0.z), u_a = (X0.w, X1.x, X1.y); b(.) = (X1.z, X1.w, X2.x), u_b = (X2.y, X2.z, X2.w)
                    {
                        float dx = Q0.x - R0.x, dy = Q0.y - R0.y, dz = Q0.z - R0.z;
                        float r2 = dx * dx + dy * dy + dz * dz;
                        A = pair_fast_t<SPEC21>(K, dx, dy, dz, r2, R0.w, R1.x, R1.y, Q0.w, Q1.x, Q1.y);
                        A = r2 < K.rc2 ? A : 0.0f;
                        npin += 2 * (r2 < K.rc2);
                    }
                    {
                        float dx = Q1.z - R0.x, dy = Q1.w - R0.y, dz = Q2.x - R0.z;
                        float r2 = dx * dx + dy * dy + dz * dz;
                        B = pair_fast_t<SPEC21>(K, dx, dy, dz, r2, R0.w, R1.x, R1.y, Q2.y, Q2.z, Q2.w);
                        B = r2 < K.rc2 ? B : 0.0f;
                        npin += (r2 < K.rc2);
                    }
                    {
                        float dx = Q0.x - R1.z, dy = Q0.y - R1.w, dz = Q0.z - R2.x;
                        float r2 = dx * dx + dy * dy + dz * dz;
                        Cc = pair_fast_t<SPEC21>(K, dx, dy, dz, r2, R2.y, R2.z, R2.w, Q0.w, Q1.x, Q1.y);
                        Cc = r2 < K.rc2 ? Cc : 0.0f;
                        npin += (r2 < K.rc2);
                    }
                    {
                        float dx = Q1.z - R1.z, dy = Q1.w - R1.w, dz = Q2.x - R2.x;
                        float r2 = dx * dx + dy * dy + dz * dz;
                        D = pair_fast_t<SPEC21>(K, dx, dy, dz, r2, R2.y, R2.z, R2.w, Q2.y, Q2.z, Q2.w);
                        D = r2 < K.rc2 ? D : 0.0f;
                    }
                    // a particle that cannot move (colloid hard core, or a trial out of the cell) keeps
                    // its old state: terms with its trial state are never used, so they are dropped
                    // before the size test (p hard: C and D unused; q hard: B and D unused)
                    const bool hp = sm.hard[pp] != 0, hq = sm.hard[q] != 0;
                    if (hq) B = D = 0.0f;
                    if (hp) Cc = D = 0.0f;
                    if (hp && hq) A = 0.0f;
                    if (!(fabsf(A) <= K.big && fabsf(B) <= K.big && fabsf(Cc) <= K.big && fabsf(D) <= K.big)) {
                        const int slot = atomicAdd(&sm.nbigp, 1); // the fix-up pass rewrites this pair
                        if (slot < SM::BIGCAP) sm.bigp[slot] = (unsigned short)idx;
                        else sm.overflow = 1;
                    }
                    // differences in FP64, then rounded (each term is at most f_big here)
                    const double a = A, b = B, c = Cc, d = D;
                    sm.pCA[idx] = (float)(c - a);
                    sm.pBA[idx] = (float)(b - a);
                    sm.pDC[idx] = (float)(d - c);
                }
#pragma unroll
                for (int o = 16; o >= 1; o >>= 1) npin += __shfl_xor_sync(0xffffffffu, npin, o);
                npairs += (unsigned long long)npin;
            }
        }
        if (lane == 0 && npairs) atomicAdd(&sm.pairs, npairs);
        __syncthreads();
        if (!sm.overflow && (sm.nbigs | sm.nbigp)) { // (uniform) FP64 fix-up of the listed pairs
            fixup_big<NT, SM, SPEC21>(&v, r, g0, na, sm);
            __syncthreads();
        }
        if (sm.overflow || sm.big) { // a capacity exceeded, or an in-cell term too large to keep in FP32
            if (t == 0) hand_over(v, ci, cell, sm.overflow ? 2 : 1);
            __syncthreads();
            continue;
        }

        // ---- 5+6 warp 0: decision-independent part of dE (thread per particle),
        //      then the Metropolis decisions in id order; meanwhile thread
        //      32 + k loads the FP64 trial state of particle k for step 7 ----
        const int kw = t - 32; // write-back particle of this thread
        double wn[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        if (w != 0 && kw < na) {
            const int g = g0 + kw;
            wn[0] = v.tnx[g];
            wn[1] = v.tny[g];
            wn[2] = v.tnz[g];
            wn[3] = v.tux[g];
            wn[4] = v.tuy[g];
            wn[5] = v.tuz[g];
        }
        if (w == 0) {
            // decision-independent part of dE_k: static cells, colloid, and the
            // in-cell partners after k (still at their old state when k is tried)
            double e0 = 0.0, e1 = 0.0;
            for (int h = 0; h < 2; h++) {
                const int k = lane + 32 * h;
                if (k >= na) break;
                double sc = 0.0, sd = 0.0;
                int m = k + 1;
                for (; m + 1 < na; m += 2) {
                    sc += (double)sm.pCA[tri(k, m)];
                    sd += (double)sm.pCA[tri(k, m + 1)];
                }
                if (m < na) sc += (double)sm.pCA[tri(k, m)];
                const double d = (sm.Snew[k] - sm.Sold[k]) + (sc + sd) + sm.tdU[k];
                if (h == 0) e0 = d;
                else e1 = d;
            }
            // Metropolis decisions in id order.  dE_k = base_k + sum over earlier
            // m of (D - C if m accepted, else B - A): a triangular system, solved
            // by fixed-point rounds in parallel.  Each round recomputes every
            // dE_k from the current guess of the earlier decisions, adding the
            // terms in increasing m exactly as a sequential scan would; after
            // pass r the first r decisions are final, and a pass that changes
            // no decision has reached the unique solution (usually the second
            // or third pass), so the decisions and dE_k equal the sequential
            // scan's bits.
            const double beta = p.k.beta;
            const bool v0 = lane < na, v1 = lane + 32 < na;
            const unsigned hd0 = __ballot_sync(0xffffffffu, v0 && sm.hard[lane]);
            const unsigned hd1 = __ballot_sync(0xffffffffu, v1 && sm.hard[lane + 32]);
            const double lu0 = v0 ? sm.tlu[lane] : 0.0, lu1 = v1 ? sm.tlu[lane + 32] : 0.0;
            unsigned acc0 = 0u, acc1 = 0u;
            double x0 = e0, x1 = e1;
            for (int round = 0; round <= na; round++) {
                x0 = e0;
                x1 = e1;
                if (v0) {
                    const int kb = tri(0, lane);
                    for (int m = 0; m < lane; m++) x0 += (double)((acc0 >> m) & 1u ? sm.pDC[kb + m] : sm.pBA[kb + m]);
                }
                if (v1) {
                    const int k = lane + 32, kb = tri(0, k);
                    for (int m = 0; m < 32; m++) x1 += (double)((acc0 >> m) & 1u ? sm.pDC[kb + m] : sm.pBA[kb + m]);
                    for (int m = 32; m < k; m++)
                        x1 += (double)((acc1 >> (m - 32)) & 1u ? sm.pDC[kb + m] : sm.pBA[kb + m]);
                }
                const bool a0 = v0 && !((hd0 >> lane) & 1u) && ((x0 <= 0.0) || (lu0 <= -beta * x0));
                const bool a1 = v1 && !((hd1 >> lane) & 1u) && ((x1 <= 0.0) || (lu1 <= -beta * x1));
                const unsigned n0 = __ballot_sync(0xffffffffu, a0), n1 = __ballot_sync(0xffffffffu, a1);
                if (n0 == acc0 && n1 == acc1) break;
                acc0 = n0;
                acc1 = n1;
            }
            if (v0) sm.acc[lane] = (acc0 >> lane) & 1u;
            if (v1) sm.acc[lane + 32] = (acc1 >> lane) & 1u;
            if (v.rec_dE) {
                if (v0) {
                    v.rec_dE[p.p_off + sm.pid[lane]] = ((hd0 >> lane) & 1u) ? 0.0 : x0;
                    v.rec_lu[p.p_off + sm.pid[lane]] = lu0;
                }
                if (v1) {
                    v.rec_dE[p.p_off + sm.pid[lane + 32]] = ((hd1 >> lane) & 1u) ? 0.0 : x1;
                    v.rec_lu[p.p_off + sm.pid[lane + 32]] = lu1;
                }
            }
            // accepted dE summed in a fixed (butterfly) order
            double dsum = ((acc0 >> lane) & 1u ? x0 : 0.0) + ((acc1 >> lane) & 1u ? x1 : 0.0);
            double dabs = ((acc0 >> lane) & 1u ? fabs(x0) : 0.0) + ((acc1 >> lane) & 1u ? fabs(x1) : 0.0);
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1) {
                dsum += __shfl_xor_sync(0xffffffffu, dsum, o);
                dabs += __shfl_xor_sync(0xffffffffu, dabs, o);
            }
            // colloid hard-core rejects (code 1) counted apart from moves that leave their cell (code 3)
            const unsigned hc0 = __ballot_sync(0xffffffffu, v0 && sm.hard[lane] == 1);
            const unsigned hc1 = __ballot_sync(0xffffffffu, v1 && sm.hard[lane + 32] == 1);
            const int nacc = __popc(acc0) + __popc(acc1), nhard = __popc(hc0) + __popc(hc1);
            if (lane == 0) {
                if (!(dsum - dsum == 0.0)) atomicOr(&v.stats[r].flags, F_NONFINITE);
                v.cell_e0[cell] = dsum;
                v.cell_abs[cell] = dabs;
                v.cell_fp64[cell] = 0;
                v.cell_n0[cell] = nacc;
                v.cell_n1[cell] = nhard;
                v.cell_pairs[cell] = sm.pairs;
                v.cell_cands[cell] = (unsigned long long)na * (unsigned long long)(S26 + na - 1);
            }
        }
        __syncthreads();

        // ---- 7 write-back ----
        if (w != 0 && kw < na) {
            const int k = kw, g = g0 + k;
            const int acc = sm.acc[k];
            if (acc) {
                v.px[g] = wn[0];
                v.py[g] = wn[1];
                v.pz[g] = wn[2];
                v.ox[g] = wn[3];
                v.oy[g] = wn[4];
                v.oz[g] = wn[5];
                const float4 P1 = sm.pst[k][1], P2 = sm.pst[k][2];
                v.cl4[g] = make_float4(P1.z, P1.w, P2.x, P2.y);
                v.cl2[g] = make_float2(P2.z, P2.w);
            }
            v.outcome[p.p_off + sm.pid[k]] = sm.hard[k] == 1 ? 2 : acc;
        }
        __syncthreads();
    }
}

// FP64 attempts of the cells the FP32 phase kernel handed over in colour phase
// ci (a pair term above f_big: an overlap, where FP32 rounding of R^12
// exceeds every energy scale; or a cell above the kernel's capacity), block
// per cell, sequentially in the in-cell order (ascending id) from the
// phase-start state, with the trial moves the gather drew (tn*, tu*, tdU, tlu,
// thard): E_old and E_new of each attempt are sums of the FP64 pair term
// (pair_exact; its lighter form for mu = 2, nu = 1, sigma0 = 1) over the 27
// stencil cells' particles read from the FP64 master arrays (earlier accepted
// in-cell moves already written), one-fold minimum image, every thread of the
// block over the candidates, then a fixed-order block sum.
// dE = (E_new - E_old) + dU_colloid, accepted if dE <= 0 or ln u <= -beta dE
// (MCnptColloid.c:2491-2574).  The FP32 state copy of an accepted particle is
// written exactly as the FP32 kernel writes it.  The stencil's FP64 states
// are staged in shared memory once per cell (the own cell's entries updated
// as moves are accepted) when they fit in RESCUE_CAP particles; a larger
// stencil is read from global memory, so any cell count works.  The other
// cells of the colour do not interact with these, so running them after the
// FP32 kernel changes nothing in the chain.
constexpr int RESCUE_CAP = 1024; // particles of a staged stencil (48 KB of shared memory)

template <int NT, bool SPEC21>
__global__ void __launch_bounds__(NT) k_phase_rescue(DevView v, int ci)
{
    constexpr int NW = NT / 32;
    extern __shared__ double sx[]; // [6][RESCUE_CAP]: x, y, z, ux, uy, uz of the staged stencil
    __shared__ int st_start[27], st_cnt[27], pre[28];
    __shared__ double spo[NW], spn[NW];
    __shared__ int snp[NW];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int count = v.resc_count[ci];
    for (int e = blockIdx.x; e < count; e += gridDim.x) {
        const int code = v.resc_list[(size_t)ci * v.ctot + e];
        const int cell = code >> 2, mode = code & 3;
        const int r = v.p2c[cell];
        const Replica &p = v.rep[r];
        const int nc0 = p.nc[0], nc1 = p.nc[1], nc2 = p.nc[2];
        const int loc = cell - p.cell_off;
        const int cx = loc % nc0, cy = (loc / nc0) % nc1, cz = loc / (nc0 * nc1);
        if (t < 27) {
            int x = cx + t % 3 - 1, y = cy + (t / 3) % 3 - 1, z = cz + t / 9 - 1;
            x += x < 0 ? nc0 : (x >= nc0 ? -nc0 : 0);
            y += y < 0 ? nc1 : (y >= nc1 ? -nc1 : 0);
            z += z < 0 ? nc2 : (z >= nc2 ? -nc2 : 0);
            const int c = p.cell_off + (z * nc1 + y) * nc0 + x;
            st_start[t] = v.cell_start[c];
            st_cnt[t] = v.cell_start[c + 1] - v.cell_start[c];
        }
        __syncthreads();
        if (t < 32) {
            const int c = t < 27 ? st_cnt[t] : 0;
            int inc = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += y;
            }
            if (t < 27) pre[t] = inc - c;
            if (t == 26) pre[27] = inc;
        }
        __syncthreads();
        const int total = pre[27];
        const int g0 = st_start[13], na = st_cnt[13];
        const bool staged = total <= RESCUE_CAP;
        if (staged) {
            for (int f = t; f < total; f += NT) {
                int sl = 0, hi = 27;
                while (hi - sl > 1) {
                    const int mid = (sl + hi) >> 1;
                    if (pre[mid] <= f) sl = mid;
                    else hi = mid;
                }
                const int j = st_start[sl] + (f - pre[sl]);
                sx[f] = v.px[j];
                sx[RESCUE_CAP + f] = v.py[j];
                sx[2 * RESCUE_CAP + f] = v.pz[j];
                sx[3 * RESCUE_CAP + f] = v.ox[j];
                sx[4 * RESCUE_CAP + f] = v.oy[j];
                sx[5 * RESCUE_CAP + f] = v.oz[j];
            }
            __syncthreads();
        }
        double dsum = 0.0, dabs = 0.0;
        int nacc = 0, nhard = 0;
        unsigned long long npairs = 0ull;
        for (int k = 0; k < na; k++) {
            const int g = g0 + k;
            const int id = v.id[g];
            const unsigned char code = v.thard[g];
            if (code) { // colloid hard-core reject (1) or a move out of the cell (3): no energy evaluation
                if (t == 0) {
                    v.outcome[p.p_off + id] = code == 1 ? 2 : 0;
                    if (v.rec_dE) {
                        v.rec_dE[p.p_off + id] = 0.0;
                        v.rec_lu[p.p_off + id] = v.tlu[g];
                    }
                }
                nhard += code == 1;
                continue;
            }
            const double ro[3] = {v.px[g], v.py[g], v.pz[g]};
            const double eo[3] = {v.ox[g], v.oy[g], v.oz[g]};
            const double rn[3] = {v.tnx[g], v.tny[g], v.tnz[g]};
            const double en[3] = {v.tux[g], v.tuy[g], v.tuz[g]};
            double po = 0.0, pn = 0.0;
            int np = 0;
            const int fk = pre[13] + k; // this particle's own entry
            for (int f = t; f < total; f += NT) {
                if (f == fk) continue;
                double rj[3], ej[3];
                if (staged) {
                    rj[0] = sx[f], rj[1] = sx[RESCUE_CAP + f], rj[2] = sx[2 * RESCUE_CAP + f];
                    ej[0] = sx[3 * RESCUE_CAP + f], ej[1] = sx[4 * RESCUE_CAP + f], ej[2] = sx[5 * RESCUE_CAP + f];
                } else {
                    int sl = 0, hi = 27;
                    while (hi - sl > 1) {
                        const int mid = (sl + hi) >> 1;
                        if (pre[mid] <= f) sl = mid;
                        else hi = mid;
                    }
                    const int j = st_start[sl] + (f - pre[sl]);
                    rj[0] = v.px[j], rj[1] = v.py[j], rj[2] = v.pz[j];
                    ej[0] = v.ox[j], ej[1] = v.oy[j], ej[2] = v.oz[j];
                }
                double d[3];
                double r2 = dist_fold(ro[0], ro[1], ro[2], rj[0], rj[1], rj[2], p.L, d);
                if (r2 < p.k.rc2) {
                    po += SPEC21 ? pair_energy64_21(p.k, r2, d, eo, ej) : pair_exact(p.k, r2, d, eo, ej);
                    np++;
                }
                r2 = dist_fold(rn[0], rn[1], rn[2], rj[0], rj[1], rj[2], p.L, d);
                if (r2 < p.k.rc2) {
                    pn += SPEC21 ? pair_energy64_21(p.k, r2, d, en, ej) : pair_exact(p.k, r2, d, en, ej);
                    np++;
                }
            }
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1) {
                po += __shfl_xor_sync(0xffffffffu, po, o);
                pn += __shfl_xor_sync(0xffffffffu, pn, o);
                np += __shfl_xor_sync(0xffffffffu, np, o);
            }
            if (lane == 0) {
                spo[w] = po;
                spn[w] = pn;
                snp[w] = np;
            }
            __syncthreads();
            if (t == 0) {
                double so = spo[0], sn = spn[0];
                int sp = snp[0];
                for (int q = 1; q < NW; q++) {
                    so += spo[q];
                    sn += spn[q];
                    sp += snp[q];
                }
                const double dE = (sn - so) + v.tdU[g];
                const double lu = v.tlu[g];
                const bool acc = (dE <= 0.0) || (lu <= -p.k.beta * dE);
                if (acc) {
                    v.px[g] = rn[0];
                    v.py[g] = rn[1];
                    v.pz[g] = rn[2];
                    v.ox[g] = en[0];
                    v.oy[g] = en[1];
                    v.oz[g] = en[2];
                    if (staged) {
                        const int fk = pre[13] + k;
                        sx[fk] = rn[0], sx[RESCUE_CAP + fk] = rn[1], sx[2 * RESCUE_CAP + fk] = rn[2];
                        sx[3 * RESCUE_CAP + fk] = en[0], sx[4 * RESCUE_CAP + fk] = en[1], sx[5 * RESCUE_CAP + fk] = en[2];
                    }
                    const float4 c4 = v.cl4[g];
                    float tux, tuy, tuz;
                    unit_f32(en[0], en[1], en[2], tux, tuy, tuz);
                    v.cl4[g] = make_float4(c4.x + v.tdx[g], c4.y + v.tdy[g], c4.z + v.tdz[g], tux);
                    v.cl2[g] = make_float2(tuy, tuz);
                    dsum += dE;
                    dabs += fabs(dE);
                    nacc++;
                }
                v.outcome[p.p_off + id] = acc ? 1 : 0;
                if (v.rec_dE) {
                    v.rec_dE[p.p_off + id] = dE;
                    v.rec_lu[p.p_off + id] = lu;
                }
                npairs += (unsigned long long)sp;
            }
            __syncthreads(); // the accepted state is visible to the next attempt
        }
        if (t == 0) {
            if (!(dsum - dsum == 0.0)) atomicOr(&v.stats[r].flags, F_NONFINITE);
            v.cell_e0[cell] = dsum;
            v.cell_abs[cell] = dabs;
            v.cell_n0[cell] = nacc;
            v.cell_n1[cell] = nhard;
            v.cell_pairs[cell] = npairs;
            v.cell_cands[cell] = (unsigned long long)na * (unsigned long long)(total > 0 ? total - 1 : 0);
            v.cell_fp64[cell] = mode;
        }
        __syncthreads();
    }
}

} // namespace lcmc

#include "lcmc_launch.h"

namespace lcmc {

// (threads, active capacity, staged candidates per warp segment, per-warp list capacity)
// the shared memory of the 48- and 56-particle classes lets six and five
// blocks share an SM's 228 KB (1 KB of it reserved per block)
static_assert(sizeof(FastSmem<128, 48, 160, 160>) + 1024 <= 233472 / 6, "48-class: six blocks per SM");
static_assert(sizeof(FastSmem<128, 56, 176, 192>) + 1024 <= 233472 / 5, "56-class: five blocks per SM");
static const FastVariant kVariants[] = {{128, 48, 160, 160}, {128, 56, 176, 192}, {128, 64, 288, 384}};

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
    cudaFuncSetAttribute(k_phase_fast<NT, AMAX, SEG, LW, S21>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         cudaSharedmemCarveoutMaxShared);
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_phase_fast<NT, AMAX, SEG, LW, S21>, NT, bytes);
    return n > 0 ? n : 1;
}

// variant = 2 * capacity class + (mu = 2, nu = 1, sigma0 = 1 specialisation)
void launch_phase_fast(int variant, const DevView &v, cudaStream_t s, int ci, int grid)
{
    switch (variant) {
    case 0: launch_v<128, 48, 160, 160, false>(v, s, ci, grid); break;
    case 1: launch_v<128, 48, 160, 160, true>(v, s, ci, grid); break;
    case 2: launch_v<128, 56, 176, 192, false>(v, s, ci, grid); break;
    case 3: launch_v<128, 56, 176, 192, true>(v, s, ci, grid); break;
    case 4: launch_v<128, 64, 288, 384, false>(v, s, ci, grid); break;
    default: launch_v<128, 64, 288, 384, true>(v, s, ci, grid); break;
    }
}

void launch_phase_rescue(bool spec21, const DevView &v, cudaStream_t s, int ci, int grid)
{
    const int bytes = 6 * RESCUE_CAP * (int)sizeof(double);
    if (spec21) k_phase_rescue<256, true><<<grid, 256, bytes, s>>>(v, ci);
    else k_phase_rescue<256, false><<<grid, 256, bytes, s>>>(v, ci);
}

// Opts the hand-over kernel in to its dynamic shared memory (call once).
void rescue_init()
{
    const int bytes = 6 * RESCUE_CAP * (int)sizeof(double);
    cudaFuncSetAttribute(k_phase_rescue<256, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    cudaFuncSetAttribute(k_phase_rescue<256, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

// Also opts the variant in to its dynamic shared memory size: call once
// before the first launch of a variant.
int fast_blocks_per_sm(int variant)
{
    switch (variant) {
    case 0: return occupancy_v<128, 48, 160, 160, false>();
    case 1: return occupancy_v<128, 48, 160, 160, true>();
    case 2: return occupancy_v<128, 56, 176, 192, false>();
    case 3: return occupancy_v<128, 56, 176, 192, true>();
    case 4: return occupancy_v<128, 64, 288, 384, false>();
    default: return occupancy_v<128, 64, 288, 384, true>();
    }
}

} // namespace lcmc
