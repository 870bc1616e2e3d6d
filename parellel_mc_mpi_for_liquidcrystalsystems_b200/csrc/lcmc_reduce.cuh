// lcmc_reduce.cuh - fixed-order block reductions over a replica's chunk
// partial sums (DevView::red_part, written by the chunk-sum kernels).
#pragma once
#include "lcmc_internal.h"

namespace lcmc {

// Block sum of K values (blockDim.x a multiple of 32, at most 256); warp
// butterflies, then thread 0 adds the warp results in warp order and holds
// the sums.
template <int K>
__device__ __forceinline__ void block_sums(double (&s)[K], double (*sh)[8])
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; k++) {
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) s[k] += __shfl_xor_sync(0xffffffffu, s[k], o);
        if (lane == 0) sh[k][w] = s[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < K; k++) {
            double t = sh[k][0];
            for (int q = 1; q < (int)(blockDim.x >> 5); q++) t += sh[k][q];
            s[k] = t;
        }
    }
    __syncthreads();
}

// Sum of replica r's chunk partials over `count` items (particles by
// default; call from every thread of one block; thread 0 holds the result).
template <int K>
__device__ __forceinline__ void finish_sums(const DevView &v, int r, int count, double (&s)[K])
{
    const int nc = (count + LCMC_RED_CHUNK - 1) / LCMC_RED_CHUNK;
#pragma unroll
    for (int k = 0; k < K; k++) s[k] = 0.0;
    for (int c = threadIdx.x; c < nc; c += blockDim.x)
        for (int k = 0; k < K; k++) s[k] += v.red_part[((size_t)r * v.red_nchunk + c) * LCMC_RED_K + k];
    __shared__ double sh[K][8];
    block_sums<K>(s, sh);
}

template <int K>
__device__ __forceinline__ void finish_sums(const DevView &v, int r, double (&s)[K])
{
    finish_sums<K>(v, r, v.rep[r].n, s);
}

} // namespace lcmc
