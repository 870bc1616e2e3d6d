// lcmc_launch.h - host-side launchers exported by the kernel translation units.
#pragma once
#include <cuda_runtime.h>

#include "lcmc_internal.h"

namespace lcmc {

// lcmc_rebin.cu
void launch_rebin(const DevView &v, cudaStream_t s, int grid);
// per-cell results of the colour phases into the statistics and the running
// energy (before the volume move); then the sweep counter and adaptive step
void launch_sweep_stats(const DevView &v, cudaStream_t s);
void launch_sweep_advance(const DevView &v, cudaStream_t s);

// lcmc_sweep_exact.cu (FP64, bit-identical to the CPU oracle)
void launch_phase_exact(const DevView &v, cudaStream_t s, int ci, int grid);
void launch_energy_exact(const DevView &v, cudaStream_t s, double *e0, double *e1, int *hard, int scaled, int grid);
int energy_exact_blocks_per_sm(); // resident blocks of 128 threads per SM

// lcmc_sweep_fast.cu (FP32)
struct FastVariant {
    int threads, amax, seg, lcap; // active-cell capacity, staged candidates per warp, list capacity
};
int fast_variant_count();
FastVariant fast_variant(int i);
void launch_phase_fast(int variant, const DevView &v, cudaStream_t s, int ci, int grid);
// FP64 attempts of the cells the FP32 kernel handed over in colour phase ci
void launch_phase_rescue(bool spec21, const DevView &v, cudaStream_t s, int ci, int grid);
void rescue_init(); // once per process before the first hand-over launch
int fast_blocks_per_sm(int variant);

// lcmc_misc.cu
void launch_q_chunk_sums(const DevView &v, cudaStream_t s); // Q-tensor chunk sums of every replica
// chunk sums of (e0, e1, hard) of the NPT replicas not rejected at stage 1
void launch_chunk_sums_volume(const DevView &v, cudaStream_t s, const double *e0, const double *e1, const int *hard);
// FP32-pair screen of the volume move: energies at V and V', chunk sums, stage 1
void launch_screen(const DevView &v, cudaStream_t s, double *e0, double *e1, int *hard, int grid, bool spec21);
int screen_blocks_per_sm();
void launch_energy_reduce(const DevView &v, cudaStream_t s, const double *e0, int replica_only);
// FP64 energy check of the due replicas (all = every replica) from per-particle energies e0
void launch_energy_check(const DevView &v, cudaStream_t s, const double *e0, int all);
void launch_volume(const DevView &v, cudaStream_t s, double *e0, double *e1, int *hard, int grid);
void launch_order_sums(const DevView &v, cudaStream_t s, int r, double *out);
void launch_to_id_order(const DevView &v, cudaStream_t s, int r, int grid);
void launch_validate_upload(const double *const x[6], int *id, int n, const double L[3], double R2, int *flag,
                            cudaStream_t s, int grid);

} // namespace lcmc
struct lcmc_mlp;
namespace lcmc {
// lcmc_mlp.cu (in-sweep surrogate inference)
void *mlp_input(lcmc_mlp *m);
int mlp_ld(lcmc_mlp *m);
int mlp_bmax(lcmc_mlp *m);
int mlp_n_in(lcmc_mlp *m);
const float *mlp_forward_device(lcmc_mlp *m, int B, cudaStream_t s);
int *mlp_err(lcmc_mlp *m);

// lcmc_da.cu (surrogate features, delayed acceptance, recordings)
void launch_features(const DevView &v, cudaStream_t s, void *X, int ldx, int grid);
void launch_da_stage1(const DevView &v, cudaStream_t s, const float *y);
void launch_record_samples(const DevView &v, cudaStream_t s);
void launch_hist_record(const DevView &v, cudaStream_t s);
void launch_volume_propose(const DevView &v, cudaStream_t s);
void launch_volume_finish(const DevView &v, cudaStream_t s, double *e0, double *e1, int *hard, int grid);

// lcmc_noalloc.cu (allocation-free FP64 total energy on a caller's stream)
int total_energy_noalloc(const GBConsts &k, int n, const double *px, const double *py, const double *pz,
                         const double *ox, const double *oy, const double *oz, const double box[3], double *d_out,
                         cudaStream_t st, char *msg, size_t len);

// lcmc_pairtest.cu / lcmc_pairtest64.cu (pair term on given inputs)
void launch_pair_terms32(const GBConsts &k, int n, const double *d, const double *ei, const double *ej, double *out,
                         cudaStream_t s);
void launch_pair_terms64(const GBConsts &k, int n, const double *d, const double *ei, const double *ej, double *out,
                         cudaStream_t s);

} // namespace lcmc
