// lcmc_noalloc.cu - FP64 total energy of a caller-owned device configuration
// without any device allocation (lcmc_total_energy_noalloc).
//
// Who needs it: a host program that already owns the GPU's memory (its own
// pool reserves it) or that runs this library inside a time step where the
// device-wide synchronisation of cudaMalloc/cudaFree is not acceptable.  The
// energy computation needs scratch (a cell list and per-particle energies);
// here it lives in one file-scope __device__ array of fixed size, present on
// every GPU that loads liblcmc.so until the process exits.  No cudaMalloc,
// cudaFree or allocating library call is made on this path.
//
// Compiled without FMA contraction, like the FP64 sweep kernel.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/lcmc.h"
#include "lcmc_gb.cuh"
#include "lcmc_internal.h"

namespace lcmc {

constexpr int NA_MAX_N = LCMC_NOALLOC_MAX_PARTICLES;
constexpr int NA_MAX_C = LCMC_NOALLOC_MAX_CELLS;

struct NoAllocScratch {
    int count[NA_MAX_C];
    int start[NA_MAX_C + 1];
    int fill[NA_MAX_C];
    int cid[NA_MAX_N];
    int order[NA_MAX_N];
    int sorted[NA_MAX_N];
    double e[NA_MAX_N];
};

// The scratch area.  In host code this name is only a stand-in for the symbol:
// its device address comes from cudaGetSymbolAddress (noalloc_scratch below).
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

struct NAArgs {
    GBConsts k;
    double L[3], w[3];
    int nc[3];
    int n, ncell;
    const double *px, *py, *pz, *ox, *oy, *oz;
};

__global__ void k_na_zero(NoAllocScratch *s, int ncell)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
        s->count[c] = 0;
        s->fill[c] = 0;
    }
}

__device__ __forceinline__ int na_cell_axis(double x, double w, int nc)
{
    int c = (int)(x / w);
    return c < 0 ? 0 : (c >= nc ? nc - 1 : c);
}

__global__ void k_na_bin(NoAllocScratch *s, NAArgs a)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const int cx = na_cell_axis(a.px[i], a.w[0], a.nc[0]);
        const int cy = na_cell_axis(a.py[i], a.w[1], a.nc[1]);
        const int cz = na_cell_axis(a.pz[i], a.w[2], a.nc[2]);
        const int c = (cz * a.nc[1] + cy) * a.nc[0] + cx;
        s->cid[i] = c;
        atomicAdd(&s->count[c], 1);
    }
}

// One block of 1024 threads, up to 32 cells per thread.
__global__ void k_na_scan(NoAllocScratch *s, int ncell)
{
    __shared__ int sh[33];
    const int per = (ncell + 1023) / 1024;
    const int b = threadIdx.x * per;
    int loc = 0;
    for (int k = 0; k < per; k++)
        if (b + k < ncell) loc += s->count[b + k];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int inc = loc;
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) sh[w] = inc;
    __syncthreads();
    if (w == 0) {
        int v = sh[lane], vi = v;
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, vi, o);
            if (lane >= o) vi += y;
        }
        sh[lane] = vi - v;
        if (lane == 31) sh[32] = vi;
    }
    __syncthreads();
    int ex = inc - loc + sh[w];
    for (int k = 0; k < per; k++)
        if (b + k < ncell) {
            s->start[b + k] = ex;
            ex += s->count[b + k];
        }
    if (threadIdx.x == 0) s->start[ncell] = sh[32];
}

__global__ void k_na_scatter(NoAllocScratch *s, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int c = s->cid[i];
        s->order[s->start[c] + atomicAdd(&s->fill[c], 1)] = i;
    }
}

// Warp per cell: particles of a cell in ascending index (deterministic sums).
__global__ void k_na_sort(NoAllocScratch *s, int ncell)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < ncell; c += warps) {
        const int b = s->start[c], n = s->start[c + 1] - b;
        for (int q = lane; q < n; q += 32) {
            const int my = s->order[b + q];
            int rk = 0;
            for (int u = 0; u < n; u++) rk += s->order[b + u] < my;
            s->sorted[b + rk] = my;
        }
    }
}

// Warp per particle: 1/2 sum over the 27-cell stencil (duplicates dropped,
// one-fold minimum image, r < rc) of the FP64 pair term, plus the colloid term.
__global__ void k_na_energy(NoAllocScratch *s, NAArgs a)
{
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    __shared__ int s_cell[8][27];
    __shared__ int s_base[8][28];
    for (int i = blockIdx.x * nw + wib; i < a.n; i += gridDim.x * nw) {
        const int cell = s->cid[i];
        const int cx = cell % a.nc[0], cy = (cell / a.nc[0]) % a.nc[1], cz = cell / (a.nc[0] * a.nc[1]);
        int c = -1;
        if (lane < 27) {
            const int x = (cx + lane % 3 - 1 + a.nc[0]) % a.nc[0];
            const int y = (cy + (lane / 3) % 3 - 1 + a.nc[1]) % a.nc[1];
            const int z = (cz + lane / 9 - 1 + a.nc[2]) % a.nc[2];
            c = (z * a.nc[1] + y) * a.nc[0] + x;
        }
        const unsigned same = __match_any_sync(0xffffffffu, c);
        const bool keep = lane < 27 && (__ffs(same) - 1) == lane;
        const unsigned kb = __ballot_sync(0xffffffffu, keep);
        const int ncl = __popc(kb);
        if (keep) s_cell[wib][__popc(kb & ((1u << lane) - 1u))] = c;
        __syncwarp();
        int cnt = lane < ncl ? s->start[s_cell[wib][lane] + 1] - s->start[s_cell[wib][lane]] : 0;
        int inc = cnt;
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane < ncl) s_base[wib][lane] = inc - cnt;
        if (lane == 31) s_base[wib][ncl] = inc;
        __syncwarp();
        const double ri[3] = {a.px[i], a.py[i], a.pz[i]};
        const double ei[3] = {a.ox[i], a.oy[i], a.oz[i]};
        double acc = 0.0;
        for (int sc = 0; sc < ncl; sc++) {
            const int B = s_base[wib][sc], ns = s_base[wib][sc + 1] - B;
            const int g0 = s->start[s_cell[wib][sc]];
            for (int q = B + ((lane - B) & 31); q < B + ns; q += 32) {
                const int j = s->sorted[g0 + (q - B)];
                if (j == i) continue;
                const double rj[3] = {a.px[j], a.py[j], a.pz[j]};
                const double ej[3] = {a.ox[j], a.oy[j], a.oz[j]};
                double d[3];
                const double r2 = dist_fold(ri[0], ri[1], ri[2], rj[0], rj[1], rj[2], a.L, d);
                if (r2 < a.k.rc2) acc += pair_exact(a.k, r2, d, ei, ej);
            }
        }
        for (int o = 16; o >= 1; o >>= 1) acc = acc + __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) {
            double u = 0.5 * acc;
            if (a.k.coll_on) u += colloid_rod(a.k, ri, ei, a.L);
            s->e[i] = u;
        }
        __syncwarp();
    }
}

// One block: sum of the per-particle energies in a fixed order -> *out.
__global__ void k_na_reduce(const NoAllocScratch *s, int n, double *out)
{
    __shared__ double sh[256];
    double v = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) v += s->e[i];
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

// Device address of the scratch area, looked up once per device with that
// device current (cudaGetSymbolAddress does not allocate).
static int noalloc_scratch(NoAllocScratch **out, char *msg, size_t len)
{
    static std::mutex mu;
    static NoAllocScratch *addr[64] = {nullptr};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) {
        snprintf(msg, len, "cudaGetDevice: %s", cudaGetErrorString(e));
        return LCMC_ENODEV;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            snprintf(msg, len, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
            return LCMC_ECUDA;
        }
        addr[dev] = (NoAllocScratch *)p;
    }
    *out = addr[dev];
    return LCMC_OK;
}

int total_energy_noalloc(const GBConsts &k, int n, const double *px, const double *py, const double *pz,
                         const double *ox, const double *oy, const double *oz, const double box[3], double *d_out,
                         cudaStream_t st, char *msg, size_t len)
{
    NAArgs a;
    a.k = k;
    a.n = n;
    a.ncell = 1;
    if (n > NA_MAX_N) {
        snprintf(msg, len, "n = %d above the allocation-free limit of %d particles", n, NA_MAX_N);
        return LCMC_EINVAL;
    }
    // every size check runs before the first launch; the cell count per axis
    // and their product are formed in 64 bits from finite boxes only, so a
    // huge or non-finite box cannot wrap into a small (or negative) count
    for (int d = 0; d < 3; d++) {
        if (!std::isfinite(box[d])) {
            snprintf(msg, len, "box edge %d is not finite", d);
            return LCMC_EINVAL;
        }
    }
    if (!(box[0] >= 2.0 * k.rc && box[1] >= 2.0 * k.rc && box[2] >= 2.0 * k.rc)) {
        snprintf(msg, len, "box shorter than twice the cutoff");
        return LCMC_EBOX;
    }
    long long ncell = 1;
    for (int d = 0; d < 3; d++) {
        const double m = std::floor(box[d] / k.rc);
        if (!(m <= (double)NA_MAX_C)) {
            snprintf(msg, len, "box edge %d gives more than %d cells per axis (allocation-free limit %d cells)", d,
                     NA_MAX_C, NA_MAX_C);
            return LCMC_EINVAL;
        }
        a.nc[d] = m < 1.0 ? 1 : (int)m;
        a.L[d] = box[d];
        a.w[d] = box[d] / (double)a.nc[d];
        ncell *= (long long)a.nc[d];
    }
    if (ncell > (long long)NA_MAX_C) {
        snprintf(msg, len, "%d x %d x %d cells above the allocation-free limit of %d", a.nc[0], a.nc[1], a.nc[2],
                 NA_MAX_C);
        return LCMC_EINVAL;
    }
    a.ncell = (int)ncell;
    a.px = px;
    a.py = py;
    a.pz = pz;
    a.ox = ox;
    a.oy = oy;
    a.oz = oz;
    NoAllocScratch *s = nullptr;
    int rc = noalloc_scratch(&s, msg, len);
    if (rc) return rc;
    if (n <= 0) {
        k_na_reduce<<<1, 256, 0, st>>>(s, 0, d_out);
        cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? LCMC_OK : LCMC_ECUDA;
    }
    k_na_zero<<<(a.ncell + 255) / 256, 256, 0, st>>>(s, a.ncell);
    k_na_bin<<<(n + 255) / 256, 256, 0, st>>>(s, a);
    k_na_scan<<<1, 1024, 0, st>>>(s, a.ncell);
    k_na_scatter<<<(n + 255) / 256, 256, 0, st>>>(s, n);
    k_na_sort<<<(a.ncell + 7) / 8, 256, 0, st>>>(s, a.ncell);
    k_na_energy<<<(n + 7) / 8, 256, 0, st>>>(s, a);
    k_na_reduce<<<1, 256, 0, st>>>(s, n, d_out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        snprintf(msg, len, "launch: %s", cudaGetErrorString(e));
        return LCMC_ECUDA;
    }
    return LCMC_OK;
}

} // namespace lcmc
