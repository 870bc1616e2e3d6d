// lcmc_rebin.cu - per-sweep grid set-up and the integer counting-sort rebin.
//
// The reference keeps a Verlet list rebuilt by an O(N^2) double loop
// (build_neighbor_lists, MCnptColloid.c:1395-1468) and, in its MPI path,
// scatters particles to 2x2x2 subcells of each rank's block
// (dist_batch_to_cells, MCnptColloid.c:4942).  Here every sweep re-bins all
// particles of all replicas into a cell grid (width >= rc + max_displacement)
// with a randomly shifted origin:
//   k_sweep_setup  grid size, shift and colour order per replica (Philox)
//   k_bin          cell of every particle + arrival rank (atomics)
//   k_scan_*       exclusive scan of the cell counts (3 kernels)
//   k_scatter      slot of every particle
//   k_sort_cells   inside every cell, ascending particle id (deterministic)
//   k_gather       permute the SoA state into the other buffer
// The result is bit-identical to the CPU oracle's grid (cell-major, id order).
#include <cuda_runtime.h>

#include "lcmc_internal.h"
#include "lcmc_reduce.cuh"
#include "lcmc_rng.cuh"
#include "lcmc_trial.cuh"

namespace lcmc {

// Cells per axis: the largest count whose cells are at least wmin wide; an
// even count (8-colour checkerboard) unless the replica takes the fine grid,
// which keeps an odd count of 3 or more (3 colours on that axis).
__device__ __forceinline__ int grid_dim(double L, double wmin, int nc_max, int fine, int *flags)
{
    int m = (int)floor(L / wmin);
    int nc = m >= 2 ? ((fine && m >= 3) ? m : m - (m & 1)) : 1;
    if (nc > nc_max) {
        nc = nc_max;
        atomicOr(flags, F_GRIDCAP);
    }
    return nc;
}

// One block; thread r sets up replica r.  Then a thread per colour phase
// scans the phase's active-cell counts over replicas.
__global__ void k_sweep_setup(DevView v)
{
    for (int r = threadIdx.x; r < v.R; r += blockDim.x) {
        Replica &p = v.rep[r];
        for (int a = 0; a < 3; a++) {
            p.nc[a] = grid_dim(p.L[a], p.wmin, p.nc_max, p.fine, &v.stats[r].flags);
            p.w[a] = p.L[a] / (double)p.nc[a];
            p.kc[a] = (p.nc[a] & 1) && p.nc[a] >= 3 ? 3 : 2;
        }
        p.ncol = p.kc[0] * p.kc[1] * p.kc[2];
        U4 s = draw(p.key, SWEEP_ID, p.sweep, TAG_SHIFT);
        p.shift[0] = u01(s.x) * p.w[0];
        p.shift[1] = u01(s.y) * p.w[1];
        p.shift[2] = u01(s.z) * p.w[2];
        // colour c = bx + kc0 (by + kc1 bz); with 8 colours c = bx + 2 by + 4 bz,
        // drawn and shuffled exactly as before the fine grid existed
        const int K = p.ncol;
        uint32_t rr[LCMC_MAX_COLOURS + 1];
        U4 c0 = draw(p.key, SWEEP_ID, p.sweep, TAG_COLOUR);
        U4 c1 = draw(p.key, SWEEP_ID, p.sweep, TAG_COLOUR + 1);
        rr[0] = c0.x, rr[1] = c0.y, rr[2] = c0.z, rr[3] = c0.w, rr[4] = c1.x, rr[5] = c1.y, rr[6] = c1.z, rr[7] = c1.w;
        for (int m = 0; 8 + 4 * m < K - 1; m++) {
            const U4 e = draw(p.key, SWEEP_ID, p.sweep, TAG_COLOUR_EXT + (uint32_t)m);
            rr[8 + 4 * m] = e.x, rr[9 + 4 * m] = e.y, rr[10 + 4 * m] = e.z, rr[11 + 4 * m] = e.w;
        }
        int perm[LCMC_MAX_COLOURS];
        for (int i = 0; i < K; i++) perm[i] = i;
        for (int i = K - 1; i >= 1; i--) { // Fisher-Yates (the reference shuffles its subcells, 646-648)
            int j = (int)(rr[K - 1 - i] % (uint32_t)(i + 1));
            int t = perm[i];
            perm[i] = perm[j];
            perm[j] = t;
        }
        for (int i = 0; i < LCMC_MAX_COLOURS; i++) p.perm[i] = i < K ? perm[i] : -1;
        p.use_fast = (p.kernel == 1) && p.nc[0] >= 4 && p.nc[1] >= 4 && p.nc[2] >= 4;
        p.vol_state = 0;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < v.nphase * v.ngroup; i += blockDim.x) v.resc_count[i] = 0;
    if ((int)threadIdx.x < v.nphase) {
        int ci = threadIdx.x;
        int *off = v.act_off + ci * (v.R + 1);
        int acc = 0;
        for (int r = 0; r < v.R; r++) {
            off[r] = acc;
            const Replica &p = v.rep[r];
            const int col = p.perm[ci];
            if (col < 0) continue; // this replica has fewer colours
            const int b[3] = {col % p.kc[0], (col / p.kc[0]) % p.kc[1], col / (p.kc[0] * p.kc[1])};
            int cnt = 1;
            for (int a = 0; a < 3; a++) cnt *= axis_colour_count(p.nc[a], p.kc[a], b[a]);
            acc += cnt;
        }
        off[v.R] = acc;
    }
}

__device__ __forceinline__ int cell_of(double x, double shift, double w, int nc, double L)
{
    double t = x - shift;
    if (t < 0.0) t += L;
    int c = (int)(t / w);
    if (c >= nc) c = nc - 1;
    if (c < 0) c = 0;
    return c;
}

__global__ void k_bin(DevView v)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < v.ntot; i += gridDim.x * blockDim.x) {
        const Replica &p = v.rep[v.p2r[i]];
        int cx = cell_of(v.px[i], p.shift[0], p.w[0], p.nc[0], p.L[0]);
        int cy = cell_of(v.py[i], p.shift[1], p.w[1], p.nc[1], p.L[1]);
        int cz = cell_of(v.pz[i], p.shift[2], p.w[2], p.nc[2], p.L[2]);
        int c = p.cell_off + (cz * p.nc[1] + cy) * p.nc[0] + cx;
        v.cid[i] = c;
        v.rank[i] = atomicAdd(&v.cell_count[c], 1);
    }
}

// --- three-pass exclusive scan of cell_count -> cell_start (ctot + 1 entries) ---
constexpr int SCAN_BLOCK = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;

__device__ __forceinline__ int block_excl_scan(int x, int *sh, int *total)
{
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) sh[w] = inc;
    __syncthreads();
    if (w == 0) {
        int s = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0;
        int si = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, si, o);
            if (lane >= o) si += y;
        }
        sh[lane] = si - s;
        if (lane == 31) sh[32] = si;
    }
    __syncthreads();
    int r = inc - x + sh[w];
    *total = sh[32];
    __syncthreads();
    return r;
}

__global__ void k_scan_tiles(DevView v)
{
    __shared__ int sh[33];
    int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    int s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) s += (base + k < v.ctot) ? v.cell_count[base + k] : 0;
    int tot;
    block_excl_scan(s, sh, &tot);
    if (threadIdx.x == 0) v.block_sums[blockIdx.x] = tot;
}

__global__ void k_scan_sums(DevView v, int nblocks)
{
    __shared__ int sh[33];
    // nblocks <= SCAN_BLOCK * SCAN_ITEMS (ctot <= 16.7 M cells)
    int base = threadIdx.x * SCAN_ITEMS;
    int loc[SCAN_ITEMS];
    int s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        loc[k] = (base + k < nblocks) ? v.block_sums[base + k] : 0;
        s += loc[k];
    }
    int tot;
    int ex = block_excl_scan(s, sh, &tot);
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        if (base + k < nblocks) v.block_sums[base + k] = ex;
        ex += loc[k];
    }
    if (threadIdx.x == 0) v.cell_start[v.ctot] = tot; // end sentinel = all particles
}

__global__ void k_scan_apply(DevView v)
{
    __shared__ int sh[33];
    int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    int loc[SCAN_ITEMS];
    int s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        loc[k] = (base + k < v.ctot) ? v.cell_count[base + k] : 0;
        s += loc[k];
    }
    int tot;
    int ex = block_excl_scan(s, sh, &tot) + v.block_sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        if (base + k < v.ctot) v.cell_start[base + k] = ex;
        ex += loc[k];
    }
}

__global__ void k_scatter(DevView v)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < v.ntot; i += gridDim.x * blockDim.x)
        v.perm[v.cell_start[v.cid[i]] + v.rank[i]] = i;
}

// Warp per cell: order the cell's slots by particle id (ids are unique inside
// a replica).  Writes the gather source of every destination slot to `rank`
// (reused as the second permutation buffer).
__global__ void k_sort_cells(DevView v)
{
    int lane = threadIdx.x & 31;
    int warps = (gridDim.x * blockDim.x) >> 5;
    for (int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < v.ctot; c += warps) {
        int s = v.cell_start[c], e = v.cell_start[c + 1], n = e - s;
        for (int a = lane; a < n; a += 32) {
            int src = v.perm[s + a];
            int my = v.id[src];
            int rk = 0;
            for (int b = 0; b < n; b++) rk += v.id[v.perm[s + b]] < my;
            v.rank[s + rk] = src;
        }
    }
}

// Permute into the other buffer and, for systems on the FP32 kernel, build
// this sweep's trial move of every particle (a particle is attempted once per
// sweep from its sweep-start state, so the trial is known now): new state,
// displacement, colloid-term change, log of the Metropolis draw, hard-core flag.
__global__ void k_gather(DevView v)
{
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < v.ntot; g += gridDim.x * blockDim.x) {
        int src = v.rank[g];
        const double ro[3] = {v.px[src], v.py[src], v.pz[src]};
        const double eo[3] = {v.ox[src], v.oy[src], v.oz[src]};
        const int id = v.id[src];
        v.qx[g] = ro[0];
        v.qy[g] = ro[1];
        v.qz[g] = ro[2];
        v.qux[g] = eo[0];
        v.quy[g] = eo[1];
        v.quz[g] = eo[2];
        v.qid[g] = id;
        v.scid[g] = v.cid[src];
        const Replica &p = v.rep[v.p2r[g]];
        if (!p.use_fast) continue;
        double rn[3], en[3], dsp[3], u;
        const int ok = make_trial(p, (uint32_t)id, ro, eo, rn, en, dsp, &u);
        const int cl = v.cid[src] - p.cell_off;
        const int cx = cl % p.nc[0], cy = (cl / p.nc[0]) % p.nc[1], cz = cl / (p.nc[0] * p.nc[1]);
        // 0 trial to evaluate, 1 colloid hard-core reject, 3 leaves its cell (rejected)
        const unsigned char code = !ok ? 1 : (leaves_cell(p, cx, cy, cz, ro, dsp) ? 3 : 0);
        double dU = 0.0;
        if (code == 0 && p.k.coll_on) dU = colloid_rod(p.k, rn, en, p.L) - colloid_rod(p.k, ro, eo, p.L);
        v.tnx[g] = rn[0];
        v.tny[g] = rn[1];
        v.tnz[g] = rn[2];
        v.tux[g] = en[0];
        v.tuy[g] = en[1];
        v.tuz[g] = en[2];
        v.tdx[g] = (float)dsp[0];
        v.tdy[g] = (float)dsp[1];
        v.tdz[g] = (float)dsp[2];
        v.tdU[g] = dU;
        v.tlu[g] = log_unit(u);
        v.thard[g] = code;
        // FP32 copy relative to the particle's own cell origin
        const double lx = fold_rel(ro[0], p.shift[0] + (double)cx * p.w[0], 0.5 * p.w[0], p.L[0], 1.0 / p.L[0]);
        const double ly = fold_rel(ro[1], p.shift[1] + (double)cy * p.w[1], 0.5 * p.w[1], p.L[1], 1.0 / p.L[1]);
        const double lz = fold_rel(ro[2], p.shift[2] + (double)cz * p.w[2], 0.5 * p.w[2], p.L[2], 1.0 / p.L[2]);
        float ux, uy, uz;
        unit_f32(eo[0], eo[1], eo[2], ux, uy, uz);
        v.cl4[g] = make_float4((float)lx, (float)ly, (float)lz, ux);
        v.cl2[g] = make_float2(uy, uz);
    }
}

// Per-cell results of a sweep in chunks of LCMC_RED_CHUNK cells (blocks:
// chunk, replica): dE, accepted, hard-core rejections, in-cutoff pairs,
// stencil candidates, sum of |dE| accepted, cells attempted in FP64 by the
// FP32 kernel and, of those, cells above its capacity (counts are exact in
// FP64).
__global__ void __launch_bounds__(256) k_cell_chunk_sums(DevView v)
{
    const int c = blockIdx.x, r = blockIdx.y;
    const Replica &p = v.rep[r];
    const int ncell = p.nc[0] * p.nc[1] * p.nc[2];
    const int i0 = c * LCMC_RED_CHUNK;
    if (i0 >= ncell) return;
    const int i1 = min(ncell, i0 + LCMC_RED_CHUNK);
    double s[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int i = i0 + (int)threadIdx.x; i < i1; i += blockDim.x) {
        const int g = p.cell_off + i;
        s[0] += v.cell_e0[g];
        s[1] += (double)v.cell_n0[g];
        s[2] += (double)v.cell_n1[g];
        s[3] += (double)v.cell_pairs[g];
        s[4] += (double)v.cell_cands[g];
        s[5] += v.cell_abs[g];
        const int m = v.cell_fp64[g];
        s[6] += m != 0 ? 1.0 : 0.0;
        s[7] += m == 2 ? 1.0 : 0.0;
    }
    __shared__ double sh[8][8];
    block_sums<8>(s, sh);
    if (threadIdx.x == 0)
        for (int k = 0; k < 8; k++) v.red_part[((size_t)r * v.red_nchunk + c) * LCMC_RED_K + k] = s[k];
}

// Block per replica: add the chunk sums of the colour phases into the
// statistics and the running energy.  Runs before the volume move, whose exact
// U(V) is the energy of the configuration the phases left (the running energy
// must include their dE when the move compares or replaces it).
__global__ void __launch_bounds__(256) k_sweep_stats(DevView v)
{
    const int r = blockIdx.x;
    Replica &p = v.rep[r];
    double s[8];
    finish_sums<8>(v, r, p.nc[0] * p.nc[1] * p.nc[2], s);
    if (threadIdx.x == 0) {
        DevStats &st = v.stats[r];
        st.attempted += (unsigned long long)p.n;
        st.accepted += (unsigned long long)s[1];
        st.hard += (unsigned long long)s[2];
        st.pairs += (unsigned long long)s[3];
        st.cands += (unsigned long long)s[4];
        st.abs_dE += s[5];
        st.fp64_cells += (unsigned long long)s[6];
        st.overcap_cells += (unsigned long long)s[7];
        st.energy += s[0];
        if (!(s[0] == s[0]) || s[0] - s[0] != 0.0) st.flags |= F_NONFINITE;
        p.adapt_att += p.adapt_on ? (unsigned long long)p.n : 0ull;
        p.adapt_acc += p.adapt_on ? (unsigned long long)s[1] : 0ull;
    }
}

// One thread per replica, after the volume move (which draws from this
// sweep's counter): count the sweep, and the adaptive step.
__global__ void k_sweep_advance(DevView v)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < v.R; r += gridDim.x * blockDim.x) {
        Replica &p = v.rep[r];
        p.sweep += 1ull;
        // adaptive step (MCnptColloid.c:987-1031) per block of >= 10,000
        // attempts: -5 % below 30 % acceptance, +5 % above 55 %, with the
        // reference's resets at 1e-4 and 1.5 min_thick; never above the cap the
        // cell grid was built for (the checkerboard needs width >= rc + d)
        if (p.adapt_on) {
            if (p.adapt_att >= 10000ull) {
                const double ratio = (double)p.adapt_acc / (double)p.adapt_att;
                p.adapt_att = 0ull;
                p.adapt_acc = 0ull;
                double d = p.k.max_disp, a = p.k.max_rot;
                if (ratio < 0.3) {
                    d -= d * 0.05;
                    if (d < 0.0001 * p.min_thick) {
                        d = 0.01 * p.min_thick;
                        if (a > 0.000001) a -= 0.5 * a;
                    }
                } else if (ratio > 0.55) {
                    d += d * 0.05;
                    if (d > 1.5 * p.min_thick) {
                        d = 0.75 * p.min_thick;
                        if (a < 0.7) a += 0.5 * a;
                    }
                }
                p.k.max_disp = d < p.d_cap ? d : p.d_cap;
                p.k.max_rot = a;
            }
        }
    }
}

} // namespace lcmc

#include "lcmc_launch.h"

namespace lcmc {

void launch_rebin(const DevView &v, cudaStream_t s, int grid)
{
    k_sweep_setup<<<1, 1024, 0, s>>>(v);
    cudaMemsetAsync(v.cell_count, 0, sizeof(int) * (size_t)v.ctot, s);
    k_bin<<<grid, 256, 0, s>>>(v);
    const int tiles = (v.ctot + SCAN_TILE - 1) / SCAN_TILE;
    k_scan_tiles<<<tiles, SCAN_BLOCK, 0, s>>>(v);
    k_scan_sums<<<1, SCAN_BLOCK, 0, s>>>(v, tiles);
    k_scan_apply<<<tiles, SCAN_BLOCK, 0, s>>>(v);
    k_scatter<<<grid, 256, 0, s>>>(v);
    k_sort_cells<<<grid, 256, 0, s>>>(v);
    k_gather<<<grid, 256, 0, s>>>(v);
}

void launch_sweep_stats(const DevView &v, cudaStream_t s)
{
    k_cell_chunk_sums<<<dim3(v.red_nchunk, v.R), 256, 0, s>>>(v);
    k_sweep_stats<<<v.R, 256, 0, s>>>(v);
}

void launch_sweep_advance(const DevView &v, cudaStream_t s)
{
    k_sweep_advance<<<(v.R + 127) / 128, 128, 0, s>>>(v);
}

} // namespace lcmc
